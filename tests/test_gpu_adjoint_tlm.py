"""The adjoint's gradient against an FP64 reference gradient: the oracle
compiled on forward-mode dual numbers (oracle/oracle_dual.py), a
tangent-linear model of the reference step that shares no code with the CUDA
library's hand-written reverse sweep. For seeded directions v of the initial
internal-energy field, <dJ/du0, v> from the adjoint must equal the oracle's
directional derivative dJ(u0; v), and dJ/dgamma its gamma tangent. Unlike
finite differences this check has no step size: it is immune to the
limiter and upwind switches that limit difference quotients of J.

The CUDA forward runs the strict build, so both sides take the same branches.
Remaining differences: the adjoint differentiates the converged inversion by
the implicit-function theorem, the dual oracle differentiates the Newton
iterates as iterated, and the sums run in different orders."""
import numpy as np
import pytest

from tests._adjoint import TorusRun, tangent_errors

pytestmark = pytest.mark.gpu

TOL = 1e-9


@pytest.mark.parametrize("radius", [None, 12.0])
def test_adjoint_matches_tangent_linear_oracle(radius):
    """48 x 48 torus, 10 steps; objective through the horizon (None) or through
    the sphere at the pressure maximum r = 12; 21 directions and gamma."""
    run = TorusRun(48, 48, nsteps=10, every=4, strict=True, radius=radius)
    u0 = run.u0()
    J, gu, gg, _, _ = run.grad(u0, run.pb.gam)
    assert J != 0.0
    errs, gerr = tangent_errors(run, u0, run.pb.gam, gu, gg, ndir=21)
    assert errs.max() <= TOL, errs
    assert gerr <= TOL, gerr


def test_adjoint_matches_tangent_linear_oracle_c5():
    """The adjoint workload: 2-D torus 256 x 256 (a = 0.9375, beta_min = 100),
    200 steps, checkpoint every 20, J = sum_n dt Mdot_n through the sphere at
    the torus's pressure maximum r = 12 (matter crosses it from the first
    step); 7 directions and gamma."""
    run = TorusRun(256, 256, nsteps=200, every=20, strict=True, radius=12.0)
    u0 = run.u0()
    J, gu, gg, _, _ = run.grad(u0, run.pb.gam)
    assert J > 0.0
    errs, gerr = tangent_errors(run, u0, run.pb.gam, gu, gg, ndir=7)
    assert errs.max() <= TOL, errs
    assert gerr <= TOL, gerr
