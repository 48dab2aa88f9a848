"""The oracle (C restatement) against golden outputs of the reference's own
kernel code, committed under tests/golden/ (written by
tests/golden/make_golden.py from the host build of the reference sources).
Needs neither the reference sources nor a GPU: the inputs are rebuilt here
(seeded synthetic state, metric tables from the library's host geometry
builder) and confirmed identical to the reference run's by SHA-256 digest.
Every comparison is bit for bit.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests._setups import clone, make_setup
from tests.golden.make_golden import SEED, digest

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(HERE, name))


def _setup(v, f):
    return make_setup(v, seed=SEED, dims=(f["dims"], float(f["gam"])), geometry="product")


@pytest.mark.parametrize("v", ["t3", "t2", "ot"])
def test_inputs_rebuilt_exactly(v):
    f = load(f"ref_{v}.npz")
    s = _setup(v, f)
    g = s.geo
    assert digest(g.gcov, g.gcon, g.gdet, g.conn) == str(f["geo_sha"]), "metric tables differ"
    assert digest(s.blk.arrays["p"], s.blk.arrays["ps"]) == str(f["in_sha"]), "initial state differs"


@pytest.mark.parametrize("v", ["t3", "t2", "ot"])
def test_half_stage_golden(v):
    f = load(f"ref_{v}.npz")
    s = _setup(v, f)
    dt = float(f["dt"])
    d = O.oracle_stage(s, 0, 0.5 * dt, dt, True)
    np.testing.assert_array_equal(s.blk.active("ph"), f["half_ph"])
    np.testing.assert_array_equal(s.blk.active("psh"), f["half_psh"])
    np.testing.assert_array_equal(d, f["half_dtdir"])


@pytest.mark.parametrize("v", ["t3", "t2", "ot"])
def test_two_rk2_steps_golden(v):
    f = load(f"ref_{v}.npz")
    s = clone(_setup(v, f))
    dt = float(f["dt"])
    stage = lambda s_, fl, Dt, dd, c: O.oracle_stage(s_, fl, Dt, dd, c)
    bound = lambda s_, a, b: O.oracle_bound(s_, a, b)
    dts = []
    for _ in range(2):
        n = O.step(stage, bound, s, dt)
        dts.append(n)
        dt = min(n, 1.3 * dt)
    np.testing.assert_array_equal(s.blk.active("p"), f["steps_p"])
    np.testing.assert_array_equal(s.blk.active("ps"), f["steps_ps"])
    np.testing.assert_array_equal(np.asarray(dts), f["steps_dt"])


def test_para_golden():
    f = load("ref_cells.npz")
    for x, lr in zip(f["para_x"], f["para_lr"]):
        assert O.para(x) == (lr[0], lr[1])


def test_primtoflux_golden():
    f = load("ref_cells.npz")
    gam = float(f["gam"])
    for n in range(len(f["ptf_dir"])):
        flux, v = np.zeros(9), np.zeros(2)
        O.lib().ho_primtoflux(gam, O._ptr(f["ptf_pr"][n].copy()), O._ptr(f["ptf_gcov"][n].copy()),
                              O._ptr(f["ptf_gcon"][n].copy()), float(f["ptf_gdet"][n]), int(f["ptf_dir"][n]),
                              O._ptr(flux), O._ptr(v[:1]), O._ptr(v[1:]))
        np.testing.assert_array_equal(flux, f["ptf_flux"][n])
        np.testing.assert_array_equal(v, f["ptf_v"][n])


@pytest.mark.parametrize("name", ["2d", "1dvsq2fix1", "1dfix1", "nm"])
def test_inversions_golden(name):
    f = load("ref_cells.npz")
    gam = float(f["gam"])
    k = f"inv_{name}_"
    rets = f[k + "ret"]
    assert (rets == 0).sum() > 10 and (rets != 0).sum() > 10
    for n in range(len(rets)):
        r, p = O.utoprim(name, gam, f[k + "U"][n].copy(), f[k + "gcov"][n].copy(), f[k + "gcon"][n].copy(),
                         float(f[k + "gdet"][n]), f[k + "guess"][n].copy())
        assert r == rets[n], (n, r, rets[n])
        np.testing.assert_array_equal(p, f[k + "prim"][n])


@pytest.mark.parametrize("v", ["t3", "t2"])
def test_neighbour_repair_golden(v):
    """The oracle's fixup_utoprim against the reference's CPU routine's
    output on seeded random states and flag patterns."""
    from tests.golden.make_golden import REPAIR_DENSITIES, flag_pattern_setup
    f = load("ref_repair.npz")
    dims, gam = f[f"{v}_dims"], float(f[f"{v}_gam"])
    for k, dens in enumerate(REPAIR_DENSITIES):
        s = flag_pattern_setup(dims, gam, dens, SEED + k)
        assert digest(s.blk.arrays["p"], s.blk.arrays["pflag"]) == str(f[f"{v}_nb{k}_in_sha"])
        before = s.blk.active("p").copy()
        O.oracle_fixup_utoprim(s, "p")
        np.testing.assert_array_equal(s.blk.active("p")[:5], f[f"{v}_nb{k}_p"])
        np.testing.assert_array_equal(s.blk.active("p")[5:], before[5:])
        np.testing.assert_array_equal(s.blk.active("failimage")[4], f[f"{v}_nb{k}_fi4"])
        assert not s.blk.pflag.any()


@pytest.mark.parametrize("v", ["t3", "t2"])
def test_failed_zone_reset_golden(v):
    """A half sub-step with planted failed zones and the reset of failed
    zones (repair 1) against the reference's fixup and fixuputoprim kernels."""
    from tests._setups import plant_failures
    f = load("ref_repair.npz")
    dims, gam = f[f"{v}_dims"], float(f[f"{v}_gam"])
    s = make_setup(v, seed=7, dims=(dims, gam), geometry="product")
    plant_failures(s, frac=0.08, seed=11)
    assert digest(s.blk.arrays["p"], s.blk.arrays["ps"]) == str(f[f"{v}_reset_in_sha"])
    s.repair = 1
    O.oracle_stage(s, 0, 0.0005, 0.001)
    np.testing.assert_array_equal(s.blk.active("ph")[:5], f[f"{v}_reset_ph"])
    np.testing.assert_array_equal(s.blk.active("pflag", 1)[0], f[f"{v}_reset_pflag"])
