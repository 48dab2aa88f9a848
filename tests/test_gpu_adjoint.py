"""Hand-written adjoint of the RK2 step (C-ABI backward, checkpointed driver)
against central finite differences of the forward objective.

Objective: J = sum_n dt_n Mdot_n, the mass flux through the x1 face column
at r = 12 (the torus's pressure maximum, which matter crosses from the first
step) of a magnetised 2-D torus (48 x 48 here), steps of fixed size; the
gamma derivative and the checkpoint-interval test also use the horizon
column. The gradient is taken w.r.t. the initial internal-energy field (the
pressure perturbation) and gamma, through torch.autograd with the adjoint as
the backward of a torch.autograd.Function (tests/_adjoint.py).
Finite differences: central differences, relative step 1e-6, on seeded
random directions. J's relative sensitivity to round-off of the state is
about 3e-13 (limiter and upwind switches react to last-bit changes), so the
quotient's round-off error falls as the step grows; measured on this run
(B200, production build, median / worst of eight directions): step 1e-8
2.9e-5 / 1.9e-4, 1e-7 7.5e-6 / 1.2e-5, 1e-6 3.6e-7 / 2.4e-6. Through the
horizon column J is 4e-15 of atmosphere and the quotients do not settle
(1.6e-6 median at 1e-7, 1.2e-4 at 1e-6). The exact check of the gradient is
the tangent-linear one (tests/test_gpu_adjoint_tlm.py).
The adjoint differentiates the limiter and
upwind branches the forward takes, so the state must not sit exactly on a
branch switch: the torus is built with `generic` seeded noise, which removes
the exact ties of the textbook state (flat atmosphere, mirror symmetry, zero
field and velocities outside the torus) where J has kinks.
"""
import numpy as np
import pytest
import torch

from tests._adjoint import MdotObjective, TorusRun

pytestmark = pytest.mark.gpu

FD_REL = 1e-6
FD_WORST = 1e-4


def _fd(run, u0, gam, v, eps):
    """central difference of J along v"""
    return (run.J(u0 + eps * v, gam) - run.J(u0 - eps * v, gam)) / (2 * eps)


@pytest.fixture(scope="module")
def run():
    """objective through the horizon column"""
    return TorusRun(48, 48, nsteps=10, every=4)


@pytest.fixture(scope="module")
def run12():
    """objective through the column at r = 12"""
    return TorusRun(48, 48, nsteps=10, every=4, radius=12.0)


def test_autograd_gradient_matches_central_differences(run12):
    run = run12
    u0 = torch.from_numpy(run.u0()).requires_grad_(True)
    gam = torch.tensor(run.pb.gam, dtype=torch.float64, requires_grad=True)
    J = MdotObjective.apply(u0, gam, run)
    J.backward()
    assert J.item() != 0.0
    rng = np.random.default_rng(11)
    u = run.u0()
    errs = []
    for _ in range(8):
        v = rng.standard_normal(u.shape) * u          # relative perturbation of the pressure
        dd_ad = float((u0.grad.numpy() * v).sum())
        dd_fd = _fd(run, u, run.pb.gam, v, 1e-6)
        errs.append(abs(dd_ad - dd_fd) / max(abs(dd_fd), 1e-300))
    # the median direction agrees to FD_REL; a direction whose +-eps runs cross
    # one of the (dense, but measure-zero) limiter or upwind switches of the
    # step can differ more, so the worst direction is held to FD_WORST
    assert np.median(errs) <= FD_REL and max(errs) <= FD_WORST, errs


def test_gamma_derivative_matches_central_difference(run):
    """dJ/dgamma of the horizon objective against a central difference with
    step 1e-7 in gamma."""
    u = run.u0()
    g = run.pb.gam
    J, _, gg, _, _ = run.grad(u, g)
    assert J != 0.0
    dg_fd = (run.J(u, g + 1e-7) - run.J(u, g - 1e-7)) / 2e-7
    assert abs(gg - dg_fd) <= FD_REL * abs(dg_fd), (gg, dg_fd)


def test_checkpoint_interval_does_not_change_the_gradient(run):
    u = run.u0()
    J1, g1, gg1, _, _ = run.grad(u, run.pb.gam, every=1)
    J2, g2, gg2, _, _ = run.grad(u, run.pb.gam, every=4)
    J3, g3, gg3, _, _ = run.grad(u, run.pb.gam, every=10)
    assert J1 == J2 == J3
    scale = np.abs(g1).max()
    assert np.abs(g1 - g2).max() <= 1e-12 * scale and np.abs(g1 - g3).max() <= 1e-12 * scale
    assert abs(gg1 - gg2) <= 1e-12 * abs(gg1) and abs(gg1 - gg3) <= 1e-12 * abs(gg1)
