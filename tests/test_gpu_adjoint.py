"""Hand-written adjoint of the RK2 step (C-ABI backward, checkpointed driver)
against central finite differences of the forward objective.

Objective: J = sum_n dt_n Mdot_n, the accretion rate through the x1 face
column at the horizon of a magnetised 2-D torus (48 x 48 here), steps of fixed
size. The gradient is taken w.r.t. the initial internal-energy field (the
pressure perturbation) and gamma, through torch.autograd with the adjoint as
the backward of a torch.autograd.Function (tests/_adjoint.py).
Finite differences: central differences, relative step 1e-8, on seeded
random directions (a smaller step crosses fewer limiter and upwind
switches; round-off of J stays near 1e-8 relative of the quotient). With
1e-7, after the forward's divisions were rewritten (strict build unchanged
bit for bit, tangent-linear check still at 1e-13), the production build's
quotients crossed switches in about half of the directions: median 1.2e-6
over eight. The adjoint differentiates the limiter and
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
    return TorusRun(48, 48, nsteps=10, every=4)


def test_autograd_gradient_matches_central_differences(run):
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
        dd_fd = _fd(run, u, run.pb.gam, v, 1e-8)
        errs.append(abs(dd_ad - dd_fd) / max(abs(dd_fd), 1e-300))
    # the median direction agrees to FD_REL; a direction whose +-eps runs cross
    # one of the (dense, but measure-zero) limiter or upwind switches of the
    # step can differ more, so the worst direction is held to FD_WORST
    assert np.median(errs) <= FD_REL and max(errs) <= FD_WORST, errs
    g = run.pb.gam
    dg_fd = (run.J(u, g + 1e-7) - run.J(u, g - 1e-7)) / 2e-7
    assert abs(gam.grad.item() - dg_fd) <= FD_REL * abs(dg_fd), (gam.grad.item(), dg_fd)


def test_checkpoint_interval_does_not_change_the_gradient(run):
    u = run.u0()
    J1, g1, gg1, _, _ = run.grad(u, run.pb.gam, every=1)
    J2, g2, gg2, _, _ = run.grad(u, run.pb.gam, every=4)
    J3, g3, gg3, _, _ = run.grad(u, run.pb.gam, every=10)
    assert J1 == J2 == J3
    scale = np.abs(g1).max()
    assert np.abs(g1 - g2).max() <= 1e-12 * scale and np.abs(g1 - g3).max() <= 1e-12 * scale
    assert abs(gg1 - gg2) <= 1e-12 * abs(gg1) and abs(gg1 - gg3) <= 1e-12 * abs(gg1)
