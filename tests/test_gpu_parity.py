"""CUDA step against the oracle on the same inputs and metric tables.

Tolerances: the strict build (no FMA contraction) reproduces the oracle's
operation order, so it must agree to 1e-14 of each field's scale (only pow()
roundings differ); the production build contracts multiply-adds and must
agree to 1e-12 of each field's scale after one step -- the FP64 parity bar.
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
