"""CUDA step against the oracle on the same inputs and metric tables.

Tolerances:
  * strict build (no FMA contraction, the oracle's operation order): 1e-14 of
    each field's scale on every problem -- only pow() roundings may differ;
  * production build (multiply-adds contracted into FMAs): 1e-12 of each
    field's scale on the smooth problems (Orszag-Tang, entropy wave). On the
    torus the step itself amplifies round-off (see the torus-body test), so
    the production build is held to L1 bounds over the torus body there.
"""
import numpy as np
import pytest

from hamr_gamma_wind_b200 import problems
from tests._gpu import field_rel_err, make_pair, oracle_step

pytestmark = pytest.mark.gpu

CASES = {
    "torus3d": lambda: problems.fm_torus(32, 16, 8, rout=40.0),
    "torus2d": lambda: problems.fm_torus(48, 48, 1, rout=40.0),
    "ot": lambda: problems.orszag_tang(64),
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("strict,tol", [(True, 1e-14), (False, 1e-12)])
def test_one_step(case, strict, tol):
    if not strict and case.startswith("torus"):
        pytest.skip("torus: production build is checked against the round-off envelope below")
    pb = CASES[case]()
    blk, s = make_pair(pb, strict=strict)
    dt = 0.2 * min(pb.dx[:2])
    dn_gpu = blk.step(dt)
    dn_orc = oracle_step(s, dt)
    p, ps = blk.download()
    e = field_rel_err(blk, p, s, "p")
    assert e.max() <= tol, f"primitives: {e}"
    eb = field_rel_err(blk, ps, s, "ps")
    assert eb.max() <= tol, f"face field: {eb}"
    assert abs(dn_gpu - dn_orc) <= tol * dn_orc
    blk.close()


@pytest.mark.parametrize("case", ["torus3d", "torus2d"])
def test_production_build_on_torus_body(case):
    """Production build against the oracle over two steps, in the torus body
    (rho > 1e-2 rho_max). Outside it the step is ill-conditioned: in the
    1e-16-density atmosphere the inversion's velocities move by up to 1e-2 of
    their scale when the oracle's own inputs are perturbed by 1e-15. Inside it,
    the equatorial plane of the symmetric torus carries a mass flux that is
    zero up to round-off, and the upwinded corner EMF switches branch on its
    sign, so theta-velocity and field see isolated O(1e-6) relative changes
    when multiply-adds are contracted. Measured: hydrodynamic fields <= 2e-11,
    u2 and field <= 3e-6 (L1 relative over the body)."""
    pb = CASES[case]()
    dt = 0.2 * min(pb.dx[:2])
    blk, s = make_pair(pb, strict=False)
    rho0 = pb.active(pb.p)[0]
    body = rho0 > 1e-2 * rho0.max()
    for _ in range(2):
        blk.step(dt)
        oracle_step(s, dt)
    p, ps = blk.download()
    a, b = blk.active(p), s.blk.active("p")
    for k, tol in ((0, 1e-9), (1, 1e-9), (2, 1e-9), (4, 1e-9), (3, 1e-4), (5, 1e-4), (6, 1e-4), (7, 1e-4)):
        l1 = np.abs(a[k][body] - b[k][body]).sum() / max(np.abs(b[k][body]).sum(), 1e-300)
        assert l1 <= tol, (k, l1)
    A, B = blk.active(ps), s.blk.active("ps")
    for k in range(3):
        l1 = np.abs(A[k][body] - B[k][body]).sum() / max(np.abs(B[k][body]).sum(), 1e-300)
        assert l1 <= 1e-4, (k, l1)
    blk.close()


def test_entropy_wave_second_order():
    """Advected density wave after one crossing time: L1 error falls by ~4x
    per doubling of resolution (second order in space and time)."""
    errs = []
    for n in (32, 64, 128):
        pb = problems.entropy_wave(n, amp=1e-6)
        blk, s = make_pair(pb, strict=False)
        rho0 = problems_active_rho(pb)
        v0 = 0.5
        t_end = 1.0 / v0
        dt = 0.5 * (1.0 / n) / 1.0
        nsteps = int(np.ceil(t_end / dt))
        dt = t_end / nsteps
        for _ in range(nsteps):
            blk.step(dt)
        p, _ = blk.download()
        rho = blk.active(p)[0]
        errs.append(np.abs(rho - rho0).mean())
        blk.close()
    order = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert (order > 1.8).all(), (errs, order)


def problems_active_rho(pb):
    return pb.active(pb.p)[0].copy()


@pytest.mark.parametrize("case", ["torus3d", "ot"])
def test_many_steps_strict(case):
    pb = CASES[case]()
    blk, s = make_pair(pb, strict=True)
    dt = 0.2 * min(pb.dx[:2])
    for _ in range(10):
        dn = blk.step(dt)
        dn_o = oracle_step(s, dt)
        dt = min(dn, 1.3 * dt)
    p, ps = blk.download()
    assert field_rel_err(blk, p, s, "p").max() <= 1e-12
    assert field_rel_err(blk, ps, s, "ps").max() <= 1e-12
    blk.close()


def test_divb_roundoff():
    pb = problems.fm_torus(32, 16, 8, rout=40.0)
    blk, s = make_pair(pb, strict=False)
    dt = 0.2 * min(pb.dx[:2])
    d0 = blk.divb_max()
    for _ in range(20):
        dt = min(blk.step(dt), 1.3 * dt)
    d1 = blk.divb_max()
    _, ps = blk.download()
    bmax = np.abs(blk.active(ps)).max()
    assert d1 <= 1e-12 * bmax / min(pb.dx) + d0, (d0, d1)
    blk.close()


@pytest.mark.parametrize("case", list(CASES))
def test_divb_matches_oracle(case):
    """hamr_divb_max against the oracle's divb_calc restatement (diag.c:153-199,
    with its 0.25 factor) on the same face field: the field after three
    strict-build steps (div B at round-off, so both sides get the GPU's field
    bit for bit), then that field with seeded noise, whose divergence is of
    order noise / dx. Strict build: the same sums in the same order."""
    pb = CASES[case]()
    from oracle import oracle as O
    blk, s = make_pair(pb, strict=True)
    dt = 0.2 * min(pb.dx[:2])
    for _ in range(3):
        dt = min(blk.step(dt), 1.3 * dt)
    p, ps = blk.download()
    rng = np.random.default_rng(11)
    noisy = ps * (1.0 + 1e-3 * rng.standard_normal(ps.shape))
    for field in (ps, noisy):
        blk.upload(p, field)
        s.blk.arrays["ps"][:] = field
        d_gpu = blk.divb_max()
        d_orc = O.divb_max(s)
        assert abs(d_gpu - d_orc) <= 1e-14 * d_orc, (d_gpu, d_orc)
    assert d_orc > 1e-6 * np.abs(noisy).max() / max(pb.dx)
    blk.close()


def test_graph_advance_matches_step_loop():
    pb = problems.fm_torus(32, 16, 8, rout=40.0)
    a, _ = make_pair(pb, strict=False)
    b, _ = make_pair(pb, strict=False)
    dt0 = 0.2 * min(pb.dx[:2])
    dt_a = a.step_ch(8, dt0, interval=1)
    dt = dt0
    for _ in range(8):
        dn = b.step(dt)
        dt = min(dn, 1.3 * dt)
    pa, _ = a.download()
    pb_, _ = b.download()
    assert np.array_equal(pa, pb_)
    assert dt_a == dt
    a.close()
    b.close()


def test_bench_size_torus_strict():
    """The 192 x 96 x 64 torus of the benchmark (r_out = 1000), one step of the
    strict build against the oracle: the kernels' index arithmetic and launch
    shapes at a production block size, not only at the small test sizes."""
    pb = problems.fm_torus(192, 96, 64, rout=1000.0)
    blk, s = make_pair(pb, strict=True)
    dt = 0.2 * min(pb.dx[:2])
    dn_gpu = blk.step(dt)
    dn_orc = oracle_step(s, dt)
    p, ps = blk.download()
    assert field_rel_err(blk, p, s, "p").max() <= 1e-14
    assert field_rel_err(blk, ps, s, "ps").max() <= 1e-14
    assert abs(dn_gpu - dn_orc) <= 1e-14 * dn_orc
    blk.close()


@pytest.mark.parametrize("case", ["torus3d", "torus2d"])
def test_newman_hamlin_inversion_strict(case):
    """Newman-Hamlin as the primary inversion (the reference's NEWMAN builds),
    fallbacks unchanged: strict build against the oracle over three steps.
    Tolerance 1e-12: the solver's cubic root goes through acos and cos, whose
    last bit differs between CUDA's and the host's libm, and acos is
    ill-conditioned where its argument nears 1 (weakly magnetised zones)."""
    pb = CASES[case]()
    blk, s = make_pair(pb, strict=True, inversion="nm")
    dt = 0.2 * min(pb.dx[:2])
    for _ in range(3):
        dn = blk.step(dt)
        dn_o = oracle_step(s, dt)
        assert abs(dn - dn_o) <= 1e-12 * dn_o
        dt = min(dn, 1.3 * dt)
    p, ps = blk.download()
    assert field_rel_err(blk, p, s, "p").max() <= 1e-12
    assert field_rel_err(blk, ps, s, "ps").max() <= 1e-12
    blk.close()


@pytest.mark.parametrize("ng", [3, 2])
@pytest.mark.parametrize("case", ["torus3d", "torus2d"])
def test_mc_reconstruction_strict(case, ng):
    """Linear MC reconstruction (the reference's PPM = 0 builds, which run with
    two ghost layers) against the oracle, strict build, three steps. The
    atmosphere is 1e-8 here: with floors off, as shipped, the 1e-14 one next
    to the magnetised torus surface runs away to NaN in the first step under
    MC, in the oracle exactly as on the GPU. Tolerance 1e-11: in 3-D more
    zones reach the entropy fallbacks under MC, whose pow() differs in the
    last bit between CUDA and the host libm; moving the oracle's pow by one
    ulp moves these velocities by 5e-12 of their scale (1e-15 with PPM)."""
    n1, n2, n3 = (32, 16, 8) if case == "torus3d" else (48, 48, 1)
    pb = problems.fm_torus(n1, n2, n3, rout=40.0, ng=ng, rho_atm=1e-8, u_atm=1e-10)
    blk, s = make_pair(pb, strict=True, recon="mc")
    dt = 0.2 * min(pb.dx[:2])
    for _ in range(3):
        dn = blk.step(dt)
        dn_o = oracle_step(s, dt)
        assert abs(dn - dn_o) <= 1e-11 * dn_o
        dt = min(dn, 1.3 * dt)
    p, ps = blk.download()
    assert field_rel_err(blk, p, s, "p").max() <= 1e-11
    assert field_rel_err(blk, ps, s, "ps").max() <= 1e-11
    blk.close()


@pytest.mark.parametrize("case", ["torus3d", "torus2d"])
def test_hllc_strict(case):
    """HLLC in the orthonormal face frame (the reference's HLLC = 1 builds,
    fluxcalc2D_FT), strict build against the oracle, three steps. The frame's
    x^-1/2 is correctly rounded on the GPU (Newton step with an fma residual)
    as the host pow(x, -0.5) is, so the faces agree bit for bit except where
    the host pow misrounds. Inside the torus body (density above 1e-6 of its
    peak) every field within 1e-12 of its scale; over all zones 1e-10: the
    1e-16 atmosphere amplifies last-bit flux differences into its poloidal
    velocity (moving every pow of the oracle itself by one ulp moves that
    velocity by 1e-10 to 3e-8 of its scale)."""
    pb = CASES[case]()
    blk, s = make_pair(pb, strict=True, riemann="hllc")
    dt = 0.2 * min(pb.dx[:2])
    for _ in range(3):
        dn = blk.step(dt)
        dn_o = oracle_step(s, dt)
        assert abs(dn - dn_o) <= 1e-14 * dn_o
        dt = min(dn, 1.3 * dt)
    p, ps = blk.download()
    assert field_rel_err(blk, p, s, "p").max() <= 1e-10
    assert field_rel_err(blk, ps, s, "ps").max() <= 1e-12
    a, b = blk.active(p), s.blk.active("p")
    body = b[0] > 1e-6 * b[0].max()
    for k in range(8):
        assert np.abs(a[k] - b[k])[body].max() <= 1e-12 * np.abs(b[k][body]).max()
    blk.close()


@pytest.mark.parametrize("case", ["torus3d", "torus2d"])
def test_hllc_production_body(case):
    """Production (fma) build with HLLC: inside the torus body (density above
    1e-6 of its peak) every field within 1e-8 of its scale after three steps.
    Measured (B200): 3.5e-9 on the 3-D torus, where the contracted
    multiply-adds of the face-frame solver move one field by that much at a
    few faces; the strict build holds the reference's roundings (above)."""
    pb = CASES[case]()
    blk, s = make_pair(pb, strict=False, riemann="hllc")
    dt = 0.2 * min(pb.dx[:2])
    for _ in range(3):
        dn = blk.step(dt)
        dn_o = oracle_step(s, dt)
        assert abs(dn - dn_o) <= 1e-13 * dn_o
        dt = min(dn, 1.3 * dt)
    a = blk.active(blk.download()[0])
    b = s.blk.active("p")
    body = b[0] > 1e-6 * b[0].max()
    for k in range(8):
        assert np.abs(a[k] - b[k])[body].max() <= 1e-8 * np.abs(b[k][body]).max()
    blk.close()


@pytest.mark.parametrize("case", ["torus3d", "torus2d"])
def test_hlld_strict(case):
    """HLLD (the reference's HLLD = 1 builds: calc_HLLD with its HLLC and HLL
    fallbacks) in the same face frame, strict build against the oracle, three
    steps, under the HLLC test's bounds: torus body within 1e-12 of each
    field's scale, all zones within 1e-10."""
    pb = CASES[case]()
    blk, s = make_pair(pb, strict=True, riemann="hlld")
    dt = 0.2 * min(pb.dx[:2])
    for _ in range(3):
        dn = blk.step(dt)
        dn_o = oracle_step(s, dt)
        assert abs(dn - dn_o) <= 1e-14 * dn_o
        dt = min(dn, 1.3 * dt)
    p, ps = blk.download()
    assert field_rel_err(blk, p, s, "p").max() <= 1e-10
    assert field_rel_err(blk, ps, s, "ps").max() <= 1e-12
    a, b = blk.active(p), s.blk.active("p")
    body = b[0] > 1e-6 * b[0].max()
    for k in range(8):
        assert np.abs(a[k] - b[k])[body].max() <= 1e-12 * np.abs(b[k][body]).max()
    blk.close()


@pytest.mark.parametrize("case", ["torus3d", "torus2d"])
def test_hlld_production_body(case):
    """Production (fma) build with HLLD: inside the torus body every field
    within 3e-8 of its scale after three steps (measured: 6.0e-9 at most on
    the 3-D torus, after the face-frame solvers' shared-divisor quotients
    changed which operations the compiler contracts; the contracted Newton
    residuals of the pressure solve carry more round-off than HLLC's closed
    form)."""
    pb = CASES[case]()
    blk, s = make_pair(pb, strict=False, riemann="hlld")
    dt = 0.2 * min(pb.dx[:2])
    for _ in range(3):
        dn = blk.step(dt)
        dn_o = oracle_step(s, dt)
        assert abs(dn - dn_o) <= 1e-13 * dn_o
        dt = min(dn, 1.3 * dt)
    a = blk.active(blk.download()[0])
    b = s.blk.active("p")
    body = b[0] > 1e-6 * b[0].max()
    for k in range(8):
        assert np.abs(a[k] - b[k])[body].max() <= 3e-8 * np.abs(b[k][body]).max()
    blk.close()


@pytest.mark.parametrize("case,recon,riemann", [("torus3d", "ppm", "hll"), ("torus3d", "mc", "hll"),
                                                ("torus2d", "ppm", "hllc"), ("torus2d", "ppm", "hlld"),
                                                ("ot", "ppm", "hll")])
def test_row_flux_kernels_strict(case, recon, riemann, monkeypatch):
    """The x1/x2 row kernels (each zone reconstructed once, 12 faces per
    thread; used on large blocks) forced on small ones: bit for bit the
    face-by-face kernels, so the oracle bounds of the other tests hold."""
    pb = CASES[case]() if recon == "ppm" else problems.fm_torus(32, 16, 8, rout=40.0, rho_atm=1e-8, u_atm=1e-10)
    blk_f, _ = make_pair(pb, strict=True, recon=recon, riemann=riemann)
    monkeypatch.setenv("HAMR_FLUX_ROWS_MIN", "0")
    blk_r, _ = make_pair(pb, strict=True, recon=recon, riemann=riemann)
    dt = 0.2 * min(pb.dx[:2])
    for _ in range(3):
        dn_f = blk_f.step(dt)
        dn_r = blk_r.step(dt)
        assert dn_f == dn_r
        dt = min(dn_f, 1.3 * dt)
    pf, psf = blk_f.download()
    pr, psr = blk_r.download()
    np.testing.assert_array_equal(blk_f.active(pf), blk_r.active(pr))
    np.testing.assert_array_equal(blk_f.active(psf), blk_r.active(psr))
    blk_f.close()
    blk_r.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_column_staged_update_matches(precision, monkeypatch):
    """The conserved update with the metric and connection staged per CTA
    (blocks with n3 >= 64) against the zone-by-zone loads: the same values,
    so bit for bit in either precision (production build)."""
    from hamr_gamma_wind_b200.api import Block
    pb = problems.fm_torus(96, 48, 64, rout=1000.0)
    blks = []
    for cols in ("0", "1"):
        monkeypatch.setenv("HAMR_CONS_COLS", cols)
        b = Block(**pb.block_kwargs(), precision=precision)
        b.set_geometry(pb.geo)
        b.upload(pb.p, pb.ps)
        b.bound()
        blks.append(b)
    dt = 0.2 * min(pb.dx[:2])
    for _ in range(2):
        d0, d1 = blks[0].step(dt), blks[1].step(dt)
        assert d0 == d1
        dt = min(d0, 1.3 * dt)
    p0, s0 = blks[0].download()
    p1, s1 = blks[1].download()
    np.testing.assert_array_equal(p0, p1)
    np.testing.assert_array_equal(s0, s1)
    for b in blks:
        b.close()


def test_production_build_all_zones_c2():
    """The contracted (FMA) build against the oracle over every active zone of
    the 192 x 96 x 64 benchmark torus, three steps. It does not keep the
    reference's roundings, and the step switches branch on a few near-ties:
    measured here (B200), the largest face-field changes sit at four x1 faces
    at the edge of the magnetised loop (density 0.2-0.4 of its peak, where
    the loop's vector potential switches on), and the toroidal field, built
    from zero by cancellation in the first steps, moves by up to 5e-5 of its
    (small) scale. Injecting relative noise up to 1e-12 into the oracle's own
    state at every sub-step moves it far less (B1 L1 2e-11), so these are
    discrete switches, not smooth round-off growth. The strict build, which
    is the one benchmarked for FP64, keeps the reference's roundings and is
    held to 1e-14 above. Bounds: ten times the measured differences (L1 and
    max relative to each field's scale, all zones)."""
    pb = problems.fm_torus(192, 96, 64, rout=1000.0)
    blk, s = make_pair(pb, strict=False)
    dt = 0.2 * min(pb.dx[:2])
    for _ in range(3):
        blk.step(dt)
        oracle_step(s, dt)
    p, ps = blk.download()
    a, b = blk.active(p), s.blk.active("p")
    A, B = blk.active(ps), s.blk.active("ps")
    # (L1, max) bounds per field
    bounds = {0: (2e-12, 2e-10), 1: (6e-11, 3e-7), 2: (3e-11, 6e-9), 3: (2e-9, 1e-7), 4: (3e-12, 3e-9),
              5: (3e-8, 4e-5), 6: (3e-8, 3e-5), 7: (6e-6, 3e-4)}
    for k, (tl1, tmax) in bounds.items():
        d, r = np.abs(a[k] - b[k]), np.abs(b[k])
        l1, mx = d.sum() / r.sum(), d.max() / r.max()
        assert l1 <= tl1 and mx <= tmax, (k, l1, mx)
    for k, (tl1, tmax) in enumerate([(3e-8, 8e-5), (3e-8, 6e-5), (7e-6, 5e-4)]):
        d, r = np.abs(A[k] - B[k]), np.abs(B[k])
        l1, mx = d.sum() / r.sum(), d.max() / r.max()
        assert l1 <= tl1 and mx <= tmax, ("face", k, l1, mx)
    blk.close()


def test_benchmark_size_strict_c3_one_step():
    """One strict-build step of the full 384 x 192 x 192 benchmark torus
    against the oracle (about 20 GB of host memory for both sides): every
    primitive and face field within 1e-14 of its scale, the CFL step within
    1e-14."""
    pb = problems.fm_torus(384, 192, 192, rout=1000.0)
    blk, s = make_pair(pb, strict=True)
    dt = 0.2 * min(pb.dx[:2])
    dn_gpu = blk.step(dt)
    dn_orc = oracle_step(s, dt)
    p, ps = blk.download()
    assert field_rel_err(blk, p, s, "p").max() <= 1e-14
    assert field_rel_err(blk, ps, s, "ps").max() <= 1e-14
    assert abs(dn_gpu - dn_orc) <= 1e-14 * dn_orc
    blk.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("shape", [(24, 16, 8), (64, 40, 48), (50, 18, 70)])
def test_fused_ct_matches_separate_kernels(precision, shape, monkeypatch):
    """The fused constrained-transport kernel (centre EMFs, edge EMFs and the
    face update in one pass, polar rows after the phi average; selected with
    HAMR_CT_FUSED=1) against the three separate kernels: bit for bit, over
    blocks that span several (j, z) tiles and x1 chunks, with ragged tile
    edges. Strict build: with multiply-add contraction the compiler may fuse
    the same expression differently in two kernels, so only the build without
    it is bitwise comparable."""
    from hamr_gamma_wind_b200.api import Block
    pb = problems.fm_torus(*shape, rout=40.0)
    out = {}
    for fused in ("1", "0"):
        monkeypatch.setenv("HAMR_CT_FUSED", fused)
        blk = Block(**pb.block_kwargs(), precision=precision, strict=True)
        blk.set_geometry(pb.geo)
        blk.upload(pb.p, pb.ps)
        blk.bound()
        dt = 0.2 * min(pb.dx[:2])
        for _ in range(3):
            dt = min(blk.step(dt), 1.3 * dt)
        out[fused] = blk.download()
        blk.close()
    assert np.array_equal(out["1"][0], out["0"][0])
    assert np.array_equal(out["1"][1], out["0"][1])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("shape", [(24, 16, 32), (20, 12, 300), (16, 10, 38)])
def test_tma_staged_update_matches_direct_loads(precision, shape, monkeypatch):
    """The conserved update with its flux operands staged by bulk copies (one
    row of zones per CTA, rows longer than 256 zones in equal pieces, ragged
    16-byte windows) against the update that loads them directly: bit for
    bit over three steps (strict build, as above). The 1e-8 atmosphere of the
    MC tests: on these coarse, long-phi blocks the mixed step runs the 1e-14
    one away to NaN with either update."""
    from hamr_gamma_wind_b200.api import Block
    pb = problems.fm_torus(*shape, rout=40.0, rho_atm=1e-8, u_atm=1e-10)
    out = {}
    for tma in ("1", "0"):
        monkeypatch.setenv("HAMR_CONS_TMA", tma)
        blk = Block(**pb.block_kwargs(), precision=precision, strict=True)
        blk.set_geometry(pb.geo)
        blk.upload(pb.p, pb.ps)
        blk.bound()
        dt = 0.2 * min(pb.dx)   # long phi rows: the x3 zone width is the smallest
        for _ in range(3):
            dt = min(blk.step(dt), 1.3 * dt)
        out[tma] = blk.download()
        blk.close()
    assert np.isfinite(pb.active(out["0"][0])).all()
    assert np.array_equal(out["1"][0], out["0"][0])
    assert np.array_equal(out["1"][1], out["0"][1])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["torus3d", "torus2d"])
def test_concurrent_substep_matches_serial(precision, case, monkeypatch):
    """The sub-step with its independent kernels on side streams (x2 and x1
    fluxes and the centre EMFs beside the x3 fluxes, the CT chain beside the
    conserved update) against the same kernels in one stream: bit for bit,
    stepwise and through the graph-captured advance, with the CFL step sizes
    (each direction keeps its own step-size slot). The x1/x2 row kernels are
    forced so that their shared-memory stencil windows run as well."""
    from hamr_gamma_wind_b200.api import Block
    pb = (problems.fm_torus(40, 24, 32, rout=40.0) if case == "torus3d"
          else problems.fm_torus(48, 48, 1, rout=40.0))
    monkeypatch.setenv("HAMR_FLUX_ROWS_MIN", "0")
    out = {}
    for conc in ("1", "0"):
        monkeypatch.setenv("HAMR_CONCURRENT", conc)
        blk = Block(**pb.block_kwargs(), precision=precision, strict=True)
        blk.set_geometry(pb.geo)
        blk.upload(pb.p, pb.ps)
        blk.bound()
        dt = 0.2 * min(pb.dx[:2])
        dts = []
        for _ in range(3):
            dt = min(blk.step(dt), 1.3 * dt)
            dts.append(dt)
        dts.append(blk.step_ch(4, dt, interval=2))
        out[conc] = (*blk.download(), dts)
        blk.close()
    assert np.isfinite(pb.active(out["0"][0])).all()
    assert np.array_equal(out["1"][0], out["0"][0])
    assert np.array_equal(out["1"][1], out["0"][1])
    assert out["1"][2] == out["0"][2]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("shape", [(24, 16, 32), (20, 12, 130), (16, 10, 38)])
def test_centre_emfs_in_x3_kernel_match_separate_kernel(precision, shape, monkeypatch):
    """The centre EMFs computed by the x3 flux kernel (its slots are the
    centre-EMF zones; a slot shared by two CTAs, and the last slot, done
    once) against k_emf_centre: bit for bit over three steps, rows longer and
    shorter than a CTA's 127 slots."""
    from hamr_gamma_wind_b200.api import Block
    pb = problems.fm_torus(*shape, rout=40.0, rho_atm=1e-8, u_atm=1e-10)
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("HAMR_EMF_IN_X3", flag)
        blk = Block(**pb.block_kwargs(), precision=precision, strict=True)
        blk.set_geometry(pb.geo)
        blk.upload(pb.p, pb.ps)
        blk.bound()
        dt = 0.2 * min(pb.dx)
        for _ in range(3):
            dt = min(blk.step(dt), 1.3 * dt)
        out[flag] = blk.download()
        blk.close()
    assert np.isfinite(pb.active(out["0"][0])).all()
    assert np.array_equal(out["1"][0], out["0"][0])
    assert np.array_equal(out["1"][1], out["0"][1])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("inversion", ["2d", "nm"])
def test_inversion_inside_update_matches_separate_kernels(precision, inversion, monkeypatch):
    """The primary inversion run inside the TMA-staged update kernel (the
    guess from the state the update read, W written only for zones whose
    primary solver fails, which then take the fallback pass) against the
    update kernel followed by k_invert_primary: bit for bit over three steps
    of fixed size, flags and failure counters included, on a torus with
    planted failed and near-vacuum zones so that the fallback list is used."""
    from hamr_gamma_wind_b200.api import Block
    from tests._gpu import plant
    pb = problems.fm_torus(24, 16, 40, rout=40.0, rho_atm=1e-8, u_atm=1e-10)
    nfail, _ = plant(pb)
    assert nfail > 0
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("HAMR_FUSE_INV", flag)
        blk = Block(**pb.block_kwargs(), precision=precision, strict=True, inversion=inversion)
        blk.set_geometry(pb.geo)
        blk.upload(pb.p, pb.ps)
        blk.bound()
        dt = 0.2 * min(pb.dx)
        for _ in range(3):   # fixed sub-steps: a failed zone without floors may stay unphysical
            blk.advance_stage(0, 0.5 * dt, dt)
            blk.advance_stage(1, dt, dt)
        out[flag] = (*blk.download(), *blk.download_flags())
        blk.close()
    assert out["0"][3].any()   # the fallback pass had zones to count
    for a, b in zip(out["1"], out["0"]):
        assert np.array_equal(a, b, equal_nan=True)
