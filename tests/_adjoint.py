"""Test-harness wrapper of the C-ABI adjoint as a torch.autograd.Function:
J(u0, gamma) = accretion-rate objective of a 2-D torus run whose initial
internal-energy field is u0 (active zones), with gamma the adiabatic index.
Forward: hamr_mdot_forward; backward: hamr_adjoint_run (checkpointed)."""
import numpy as np
import torch

from hamr_gamma_wind_b200 import problems
from hamr_gamma_wind_b200.api import Adjoint, Block


def horizon_face(pb, spin):
    """x1 face column closest to the outer horizon r_H = 1 + sqrt(1 - a^2),
    inside the active range."""
    rh = 1.0 + np.sqrt(1.0 - spin * spin)
    rin = 0.9 * rh
    faces = np.arange(pb.ng + 1, pb.ng + pb.n1)
    r = np.exp(np.log(rin) + (faces - pb.ng) * pb.dx[0])
    return int(faces[np.argmin(np.abs(r - rh))])


class TorusRun:
    def __init__(self, n1=48, n2=48, nsteps=10, spin=0.9375, every=4, cfl=0.2, rout=40.0, strict=False,
                 generic=1e-3):
        self.pb = problems.fm_torus(n1, n2, 1, spin=spin, rout=rout, generic=generic)
        self.ih = horizon_face(self.pb, spin)
        self.dts = np.full(nsteps, cfl * min(self.pb.dx[:2]))
        self.every = every
        self.strict = strict

    def u0(self):
        return self.pb.active(self.pb.p)[1][:, :, 0].copy()

    def _block(self, u0, gam):
        p = self.pb.p.copy()
        v = self.pb.active(p)   # view into p
        v[1][:, :, 0] = u0
        kw = self.pb.block_kwargs()
        kw["gam"] = float(gam)
        b = Block(**kw, strict=self.strict)
        b.set_geometry(self.pb.geo)
        b.upload(p, self.pb.ps)
        return b

    def J(self, u0, gam):
        b = self._block(u0, gam)
        a = Adjoint(b, self.ih)
        J = a.forward(self.dts)
        a.close()
        b.close()
        return J

    def grad(self, u0, gam, every=None):
        b = self._block(u0, gam)
        a = Adjoint(b, self.ih)
        J, gp, gs, gg = a.gradient(self.dts, every or self.every)
        gu = b.active(gp)[1][:, :, 0].copy()
        a.close()
        b.close()
        return J, gu, gg, gp, gs


class MdotObjective(torch.autograd.Function):
    @staticmethod
    def forward(ctx, u0, gam, run):
        ctx.run = run
        ctx.save_for_backward(u0, gam)
        return torch.tensor(run.J(u0.numpy(), float(gam)), dtype=torch.float64)

    @staticmethod
    def backward(ctx, gJ):
        u0, gam = ctx.saved_tensors
        _, gu, gg, _, _ = ctx.run.grad(u0.numpy(), float(gam))
        return gJ * torch.from_numpy(gu), gJ * torch.tensor(gg, dtype=torch.float64), None
