"""Opt-in floors and failed-zone repair on the B200 against the oracle.

The torus gets planted trouble before the first step: zones with a negative
internal energy, where every solver of the inversion chain fails (pflag 6),
in a random scatter and in one solid patch (failed zones bordering each
other, so the neighbour repair's order matters), and zones of vanishing
density and energy inside the magnetised torus, which the floors lift in
the drift frame. Strict build: flags and failure counters agree exactly,
primitives to 1e-13 of each field's scale (the strict build's bound is 1e-14;
pow() roundings of the planted extreme states carry one more digit).

Without floors the repaired zones can be left unphysical (a neighbour
average of negative energies, a reset to rho = u = 1e-20 next to a dense
torus), and in the next step the inversion's outcome there turns on the
last bit of its input: measured, after three sub-steps bit-tight to 1e-15, a
fourth in which three zones of the 3-D torus failed on one side only. Those
runs are compared over one step; with floors over two.
"""
import numpy as np
import pytest

from hamr_gamma_wind_b200 import problems
from tests._gpu import field_rel_err, make_pair, oracle_step, plant

pytestmark = pytest.mark.gpu

CASES = {
    "torus3d": lambda: problems.fm_torus(32, 16, 8, rout=40.0),
    "torus2d": lambda: problems.fm_torus(48, 48, 1, rout=40.0),
}


def run_pair(case, floors, repair, steps=2, strict=True, patch=3):
    pb = CASES[case]()
    nfail, nthin = plant(pb, patch=patch)
    assert nfail > 0 and nthin > 0
    blk, s = make_pair(pb, strict=strict, floors=floors, repair=repair)
    dt = 0.2 * min(pb.dx[:2])
    out = []
    for _ in range(steps):
        blk.step(dt)
        oracle_step(s, dt)
        p, ps = blk.download()
        pflag, fail = blk.download_flags()
        out.append((field_rel_err(blk, p, s, "p").max(), field_rel_err(blk, ps, s, "ps").max(),
                    pflag, fail, s.blk.pflag.copy(), s.blk.failimage.copy(), blk.active(p)))
    blk.close()
    return out


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("floors,repair", [(True, "none"), (False, "reset"), (True, "reset"),
                                           (False, "neighbours"), (True, "neighbours")])
def test_floors_and_repairs_strict(case, floors, repair):
    for ep, eps, pflag, fail, opflag, ofail, p in run_pair(case, floors, repair, steps=2 if floors else 1):
        np.testing.assert_array_equal(pflag, opflag)
        np.testing.assert_array_equal(fail, ofail)
        assert ep <= 1e-13 and eps <= 1e-13, (ep, eps)
        assert np.isfinite(p).all()
    if floors:
        assert np.abs(p).max() < 1e30
    if repair == "neighbours":
        assert not pflag.any()                       # every failed zone repaired


def test_neighbour_repair_of_a_large_cluster_strict():
    """A solid 8 x 8 x 8 patch of failed zones: chains of dependent zones
    many waves long in the one-CTA repair kernel."""
    for ep, eps, pflag, fail, opflag, ofail, p in run_pair("torus3d", True, "neighbours", steps=1, patch=8):
        np.testing.assert_array_equal(pflag, opflag)
        np.testing.assert_array_equal(fail, ofail)
        assert ep <= 1e-13 and eps <= 1e-13, (ep, eps)


def test_floors_and_repair_production_build():
    """The FMA build on the same planted tori. Contracted multiply-adds move
    the planted zones' inversion across its failure boundary in a few zones
    (measured: 4 of 236 in the first sub-step), after which the repaired
    values differ outright, so this build is held to what the opt-ins
    guarantee rather than to the oracle's values: after two steps every zone
    is finite, no failed zone is left, the density floor holds, and the
    failure counts stay within 20 % of the oracle's (measured: within 11 %). (The energy need not be
    positive: the repair runs after the floors and may average in ghost
    values that still hold the planted negative energies, as the reference's
    order of fixup, fixup_utoprim, bound_prim has it.)"""
    for case in CASES:
        for ep, eps, pflag, fail, opflag, ofail, p in run_pair(case, True, "neighbours", strict=False):
            ks = pflag.size
            assert np.isfinite(p).all()
            assert not pflag.any()
            assert p[0].min() >= 1e-20 * (1 - 1e-12)
            f, of = fail.reshape(5, ks).sum(axis=1), ofail.reshape(5, ks).sum(axis=1)
            assert np.all(np.abs(f - of) <= 0.2 * np.maximum(of, 20)), (f, of)
