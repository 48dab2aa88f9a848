"""Test-harness wrapper of the C-ABI adjoint as a torch.autograd.Function:
J(u0, gamma) = accretion-rate objective of a 2-D torus run whose initial
internal-energy field is u0 (active zones), with gamma the adiabatic index.
Forward: hamr_mdot_forward; backward: hamr_adjoint_run (checkpointed)."""
import numpy as np
import torch

from hamr_gamma_wind_b200 import problems
from hamr_gamma_wind_b200.api import Adjoint, Block


def face_at_radius(pb, spin, r):
    """x1 face column closest to Boyer-Lindquist radius r, inside the active
    range (log-r grid from 0.9 r_H)."""
    rin = 0.9 * (1.0 + np.sqrt(1.0 - spin * spin))
    faces = np.arange(pb.ng + 1, pb.ng + pb.n1)
    rf = np.exp(np.log(rin) + (faces - pb.ng) * pb.dx[0])
    return int(faces[np.argmin(np.abs(rf - r))])


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
                 generic=1e-3, radius=None):
        """radius: the objective's surface (Boyer-Lindquist r); None: the horizon"""
        self.pb = problems.fm_torus(n1, n2, 1, spin=spin, rout=rout, generic=generic)
        self.ih = horizon_face(self.pb, spin) if radius is None else face_at_radius(self.pb, spin, radius)
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


def tangent_errors(run, u0, gam, gu, gg, ndir, seed=7):
    """The adjoint's gradient (gu w.r.t. the initial internal energy, gg w.r.t.
    gamma) against the FP64 tangent-linear oracle (oracle/oracle_dual.py): for
    ndir seeded relative directions v of u0, |<gu, v> - dJ(v)| / |dJ(v)|, and
    the same for gamma. The oracle's values follow the same step as the CUDA
    forward (strict build: to the last bits), its tangents are the forward-mode
    derivative of that step along v."""
    from oracle import oracle as O, oracle_dual as OD
    from tests._gpu import BCMAP
    pb = run.pb
    rng = np.random.default_rng(seed)
    p0 = pb.p.copy()
    pb.active(p0)[1][:, :, 0] = u0
    errs, gerr = [], None
    left = ndir
    while left > 0 or gerr is None:
        nv = min(left, OD.NT - 1)
        ob = O.Block(pb.n1, pb.n2, pb.n3, pb.ng, pb.ksize, pb.gsize)
        ob.arrays["p"][:] = p0
        ob.arrays["ps"][:] = pb.ps
        geo = O.Geometry(pb.geo.gsize, pb.geo.gcov, pb.geo.gcon, pb.geo.gdet, pb.geo.conn)
        s = O.Setup(ob, geo, pb.dx, float(gam), pb.cour, pb.poles[0], pb.poles[1], tuple(BCMAP[b] for b in pb.bc),
                    int(pb.ct_upwind))
        tr = OD.TangentRun(s, gam_tangents=[0.0] * (OD.NT - 1) + [1.0])
        seed_t = np.zeros((OD.NT, 9 * pb.ksize))
        vs = [rng.standard_normal(u0.shape) * u0 for _ in range(nv)]
        for q, v in enumerate(vs):
            pb.active(seed_t[q])[1][:, :, 0] = v
        tr.seed("p", seed_t)
        _, dJ = tr.objective(run.ih, run.dts)
        for q, v in enumerate(vs):
            ad = float((gu * v).sum())
            errs.append(abs(ad - dJ[q]) / max(abs(dJ[q]), 1e-300))
        gerr = abs(gg - dJ[-1]) / max(abs(dJ[-1]), 1e-300)
        left -= nv
    return np.array(errs), gerr
