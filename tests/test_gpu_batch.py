"""Batched ensembles (hamr_batch_*) against the same blocks stepped one by one
through their own contexts.

The batch launches run the very per-item bodies the single-block kernels run,
so with the strict build (no multiply-add contraction, identical rounding in
every inlined copy) the results must be bit for bit the same; the production
build may contract differently in the batched copies, so it is held to 1e-12
of each field's scale.
"""
import numpy as np
import pytest

from hamr_gamma_wind_b200 import problems
from hamr_gamma_wind_b200.api import Batch, Block
from tests._gpu import plant

pytestmark = pytest.mark.gpu


def _members(precision="fp64", strict=True, with_2d=True, planted=False, **kw):
    pbs, _ = problems.torus_ensemble(4, 16, 26, seed=7)
    if with_2d:
        pbs.append(problems.fm_torus(40, 32, 1, rout=40.0))   # reflective poles, 2-D
    blocks = []
    for k, pb in enumerate(pbs):
        if planted:
            plant(pb, seed=100 + k)
        b = Block(**pb.block_kwargs(), precision=precision, strict=strict, **kw)
        b.set_geometry(pb.geo)
        b.upload(pb.p, pb.ps)
        b.bound()
        blocks.append(b)
    return pbs, blocks


def _rel(a, b):
    a = a.reshape(a.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return float((np.abs(a - b).max(axis=1) / scale).max())


def _close(blocks):
    for b in blocks:
        b.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_step_matches_single_blocks_bitwise(precision):
    pbs, solo = _members(precision)
    _, mem = _members(precision)
    batch = Batch(mem)
    dts = np.array([0.2 * min(pb.dx[:2]) for pb in pbs])
    for _ in range(3):
        dn_solo = np.array([b.step(dt) for b, dt in zip(solo, dts)])
        dn_batch = batch.step(dts)
        np.testing.assert_array_equal(dn_solo, dn_batch)
        dts = np.minimum(dn_solo, 1.3 * dts)
    for a, b in zip(solo, mem):
        pa, sa = a.download()
        pb_, sb = b.download()
        np.testing.assert_array_equal(pa, pb_)
        np.testing.assert_array_equal(sa, sb)
    batch.close()
    _close(solo + mem)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_bulk_copy_update_matches_single_blocks_bitwise(precision, monkeypatch):
    """Members 3-D with 32 or more zones along x3: the batch's conserved update
    runs the single-block row kernel with its fluxes staged by bulk copies,
    one CTA per row of each member (forced for FP64, where the tiled update
    is the default), and its x3 fluxes the single-block slot kernel with the
    centre EMFs; the members must match the members stepped alone bit for
    bit, before and after the autotuner has timed the update's forms."""
    monkeypatch.setenv("HAMR_BATCH_CONS_TMA", "1")
    pbs, _ = problems.torus_ensemble(3, 32, 40, seed=11)
    assert all(pb.n3 >= 32 for pb in pbs)

    def blocks():
        out = []
        for pb in pbs:
            b = Block(**pb.block_kwargs(), precision=precision, strict=True)
            b.set_geometry(pb.geo)
            b.upload(pb.p, pb.ps)
            b.bound()
            out.append(b)
        return out

    solo, mem = blocks(), blocks()
    batch = Batch(mem)
    tun = batch.tuning()
    assert tun["update"]["tile"] == 0   # the row kernel is in use
    assert tun["flux3"]["tile"] == 0    # and the x3 slot kernel (with the centre EMFs)
    dts = np.array([0.2 * min(pb.dx[:2]) for pb in pbs])
    for s in range(4):
        if s == 2:
            batch.autotune(dts, reps=1)
        dn_solo = np.array([b.step(dt) for b, dt in zip(solo, dts)])
        np.testing.assert_array_equal(dn_solo, batch.step(dts))
        dts = np.minimum(dn_solo, 1.3 * dts)
    for a, b in zip(solo, mem):
        for x, y in zip(a.download(), b.download()):
            np.testing.assert_array_equal(x, y)
    batch.close()
    _close(solo + mem)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_bulk_copy_update_with_failed_zones_bitwise(precision, monkeypatch):
    """The same members with planted failed and near-vacuum zones and no
    floors: the batch's bulk-copy update and one-pass inversion phase against
    the members stepped alone (whose update runs the primary inversion
    inside and leaves the failed zones to the fallback pass over a list);
    one step, flags and failure counters included."""
    monkeypatch.setenv("HAMR_BATCH_CONS_TMA", "1")
    pbs, _ = problems.torus_ensemble(3, 32, 40, seed=11, rho_atm=1e-8, u_atm=1e-10)
    for k, pb in enumerate(pbs):
        nfail, _ = plant(pb, seed=200 + k)
        assert nfail > 0

    def blocks():
        out = []
        for pb in pbs:
            b = Block(**pb.block_kwargs(), precision=precision, strict=True)
            b.set_geometry(pb.geo)
            b.upload(pb.p, pb.ps)
            b.bound()
            out.append(b)
        return out

    solo, mem = blocks(), blocks()
    batch = Batch(mem)
    dts = np.array([0.2 * min(pb.dx[:2]) for pb in pbs])
    dn_solo = np.array([b.step(dt) for b, dt in zip(solo, dts)])
    np.testing.assert_array_equal(dn_solo, batch.step(dts))
    for a, b in zip(solo, mem):
        for x, y in zip((*a.download(), *a.download_flags()), (*b.download(), *b.download_flags())):
            assert np.array_equal(x, y, equal_nan=True)
        assert a.download_flags()[1].any()   # the fallback pass had zones to count
    batch.close()
    _close(solo + mem)


def test_batch_production_build_close_to_single_blocks():
    pbs, solo = _members(strict=False)
    _, mem = _members(strict=False)
    batch = Batch(mem)
    dts = np.array([0.2 * min(pb.dx[:2]) for pb in pbs])
    for _ in range(2):
        for b, dt in zip(solo, dts):
            b.step(dt)
        batch.step(dts)
    for a, b in zip(solo, mem):
        assert _rel(a.active(a.download()[0]), b.active(b.download()[0])) <= 1e-12
    batch.close()
    _close(solo + mem)


def test_batch_graph_advance_matches_step_loop_and_single_advance():
    """advance (captured graph, per-member step-size refresh every 2 steps)
    against the same steps taken through hamr_batch_step, and against each
    member's own hamr_advance."""
    pbs, a = _members()
    _, b = _members()
    _, solo = _members()
    ba, bb = Batch(a), Batch(b)
    dt0 = np.array([0.2 * min(pb.dx[:2]) for pb in pbs])
    dt_graph = ba.advance(6, dt0, interval=2)
    dt_solo = np.array([s.step_ch(6, d, interval=2) for s, d in zip(solo, dt0)])
    np.testing.assert_array_equal(dt_graph, dt_solo)
    dt = dt0.copy()
    for n in range(6):
        dn = bb.step(dt)
        if (n + 1) % 2 == 0:
            dt = np.minimum(dn, 1.3 * dt)
    np.testing.assert_array_equal(dt, dt_graph)
    for x, y, z in zip(a, b, solo):
        px, py, pz = x.download()[0], y.download()[0], z.download()[0]
        np.testing.assert_array_equal(px, py)
        np.testing.assert_array_equal(px, pz)
    ba.close()
    bb.close()
    _close(a + b + solo)


def test_autotuned_batch_gives_identical_results():
    """The autotuner only changes launch shapes (tiles, grid, schedule order):
    state after tuning is untouched and the tuned batch steps bit for bit
    like the untuned one."""
    pbs, a = _members()
    _, b = _members()
    ba, bb = Batch(a), Batch(b)
    dts = np.array([0.2 * min(pb.dx[:2]) for pb in pbs])
    p_before = [x.download()[0] for x in a]
    tun = ba.autotune(dts, reps=1)
    assert set(tun) == {"flux3", "flux2", "flux1", "fix_flux", "emf_centre", "emf_edge", "pole_average",
                        "face_update", "update", "invert", "bound_x1", "bound_x3", "bound_x2"}
    assert tun["flux1"]["ms"] > 0 and tun["flux1"]["tile"] >= 128
    for x, p0 in zip(a, p_before):
        np.testing.assert_array_equal(x.download()[0], p0)
    for _ in range(2):
        np.testing.assert_array_equal(ba.step(dts), bb.step(dts))
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x.download()[0], y.download()[0])
        np.testing.assert_array_equal(x.download_flags()[1], y.download_flags()[1])
    ba.close()
    bb.close()
    _close(a + b)


def test_batch_rejects_mixed_kinds():
    pbs, blocks = _members(with_2d=False)
    pb = pbs[0]
    other = Block(**pb.block_kwargs(), precision="mixed", strict=True)
    other.set_geometry(pb.geo)
    with pytest.raises(Exception):
        Batch(blocks + [other])
    with pytest.raises(Exception):
        Batch([blocks[0], blocks[0]])
    other.close()
    _close(blocks)


@pytest.mark.parametrize("variant", [dict(riemann="hllc"), dict(recon="mc")])
def test_batch_variants_match_single_blocks_bitwise(variant):
    """HLLC and MC members run the same per-item bodies in the batch."""
    pbs, solo = _members(**variant)
    _, mem = _members(**variant)
    batch = Batch(mem)
    dts = np.array([0.2 * min(pb.dx[:2]) for pb in pbs])
    for _ in range(2):
        dn_solo = np.array([b.step(dt) for b, dt in zip(solo, dts)])
        np.testing.assert_array_equal(dn_solo, batch.step(dts))
        dts = np.minimum(dn_solo, 1.3 * dts)
    for a, b in zip(solo, mem):
        np.testing.assert_array_equal(a.download()[0], b.download()[0])
    batch.close()
    _close(solo + mem)


@pytest.mark.parametrize("floors,repair", [(True, "none"), (False, "reset"), (True, "reset")])
def test_batch_with_floors_and_reset_matches_single_blocks_bitwise(floors, repair):
    """Members with planted failed and near-vacuum zones (negative energies,
    rho = 1e-24): the batched inversion phase with the opt-in floors and the
    reset of failed zones is the single-block kernel's body, bit for bit,
    flags and failure counters included."""
    pbs, solo = _members(planted=True, floors=floors, repair=repair)
    _, mem = _members(planted=True, floors=floors, repair=repair)
    batch = Batch(mem)
    dts = np.array([0.2 * min(pb.dx[:2]) for pb in pbs])
    for _ in range(2):
        dn_solo = np.array([b.step(dt) for b, dt in zip(solo, dts)])
        dn_batch = batch.step(dts)
        np.testing.assert_array_equal(dn_solo, dn_batch)
        dts = np.minimum(dn_solo, 1.3 * dts)
    nflag = 0
    for a, b in zip(solo, mem):
        np.testing.assert_array_equal(a.download()[0], b.download()[0])
        np.testing.assert_array_equal(a.download()[1], b.download()[1])
        fa, fb = a.download_flags(), b.download_flags()
        np.testing.assert_array_equal(fa[0], fb[0])
        np.testing.assert_array_equal(fa[1], fb[1])
        nflag += int(fa[1].sum())
    assert nflag > 0
    batch.close()
    _close(solo)
    _close(mem)


def test_batch_refuses_mixed_opt_ins_and_the_neighbour_repair():
    from hamr_gamma_wind_b200 import _lib
    _, a = _members(with_2d=False, floors=True)
    _, b = _members(with_2d=False)
    with pytest.raises(_lib.HamrError):
        Batch(a[:2] + b[:2])
    _, c = _members(with_2d=False, repair="neighbours")
    with pytest.raises(_lib.HamrError):
        Batch(c)
    _close(a + b + c)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_persistent_batch_matches_phase_launches(precision):
    """One persistent cooperative launch per sub-step (every phase in one
    kernel, grid-wide barriers between dependent phases) against one launch
    per phase: bit for bit, stepwise and through the captured advance, with
    the ensemble's 3-D members and the 2-D member with reflective poles (the
    polar flux fix as an extra phase), after autotuning the tile maps."""
    pbs, a = _members(precision)
    _, b = _members(precision)
    ba, bb = Batch(a), Batch(b)
    dts = np.array([0.2 * min(pb.dx[:2]) for pb in pbs])
    ba.autotune(dts, reps=1)
    ba.set_persistent(True)
    for _ in range(2):
        np.testing.assert_array_equal(ba.step(dts), bb.step(dts))
    np.testing.assert_array_equal(ba.advance(4, dts, interval=2), bb.advance(4, dts, interval=2))
    for x, y in zip(a, b):
        px, sx = x.download()
        py, sy = y.download()
        np.testing.assert_array_equal(px, py)
        np.testing.assert_array_equal(sx, sy)
        np.testing.assert_array_equal(x.download_flags()[1], y.download_flags()[1])
    ba.set_persistent(False)   # back to per-phase launches: still identical
    np.testing.assert_array_equal(ba.step(dts), bb.step(dts))
    ba.close()
    bb.close()
    _close(a + b)


def test_persistent_batch_refuses_other_solvers():
    pbs, a = _members(with_2d=False, riemann="hllc")
    ba = Batch(a)
    with pytest.raises(Exception):
        ba.set_persistent(True)
    ba.close()
    _close(a)
