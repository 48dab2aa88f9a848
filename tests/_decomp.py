"""The oracle as a slab of a decomposed domain (host arrays; halo messages
packed by numpy in the device layouts, [component][layer][j][z] for x1 sides
and [component][layer][i][z] for x2 sides), for the decomposition tests: the steppers of hamr_gamma_wind_b200.decomp drive it
exactly as they drive the GPU blocks."""
import numpy as np
import torch

from oracle import oracle as O
from tests._gpu import BCMAP


def oracle_setup(pb, halo=0, **kw):
    ob = O.Block(pb.n1, pb.n2, pb.n3, pb.ng, pb.ksize, pb.gsize)
    ob.arrays["p"][:] = pb.p
    ob.arrays["ps"][:] = pb.ps
    geo = O.Geometry(pb.geo.gsize, pb.geo.gcov, pb.geo.gcon, pb.geo.gdet, pb.geo.conn)
    return O.Setup(ob, geo, pb.dx, pb.gam, pb.cour, pb.poles[0], pb.poles[1], tuple(BCMAP[b] for b in pb.bc),
                   int(pb.ct_upwind), halo=halo, **kw)


class OracleSlab:
    def __init__(self, sp, **kw):
        self.sp = sp
        self.s = oracle_setup(sp, halo=getattr(sp, "halo", 0), **kw)
        self.dt3 = None
        b = self.s.blk
        self.count = max(12 * sp.ng * b.g2 * b.g3, 12 * sp.ng * b.g1 * b.g3)

    @staticmethod
    def _names(full):
        return ("p", "ps") if full else ("ph", "psh")

    def stage(self, full, Dt, dt):
        d = O.oracle_stage(self.s, full, Dt, dt, calc_dt=bool(full))
        if full:
            self.dt3 = np.array(d[1:4])

    def bound_dim(self, full, dim):
        O.oracle_bound_dim(self.s, dim, *self._names(full))

    def _layers(self, side, ghost):
        """index of the ng layers next to `side` (0, 1: x1; 2, 3: x2):
        the active ones, or the ghosts beyond it"""
        ng = self.sp.ng
        n = self.sp.n1 if side < 2 else self.sp.n2
        if ghost:
            i0 = ng + n if side & 1 else 0
        else:
            i0 = n if side & 1 else ng
        sl = slice(i0, i0 + ng)
        return (slice(None), sl) if side < 2 else (slice(None), slice(None), sl)

    def pack(self, full, side):
        pn, sn = self._names(full)
        ix = self._layers(side, ghost=False)
        a = np.concatenate([self.s.blk.view(pn, 9)[ix], self.s.blk.view(sn, 3)[ix]])
        if side >= 2:   # [component][layer][i][z], as the device packs it
            a = a.transpose(0, 2, 1, 3)
        return torch.from_numpy(np.ascontiguousarray(a).reshape(-1).copy())

    def recv_buffer(self, side):
        return torch.empty(self.count, dtype=torch.float64)

    def unpack(self, full, side, buf):
        ng = self.sp.ng
        b = self.s.blk
        pn, sn = self._names(full)
        ix = self._layers(side, ghost=True)
        if side < 2:
            a = buf.numpy()[:12 * ng * b.g2 * b.g3].reshape(12, ng, b.g2, b.g3)
        else:
            a = buf.numpy()[:12 * ng * b.g1 * b.g3].reshape(12, ng, b.g1, b.g3).transpose(0, 2, 1, 3)
        b.view(pn, 9)[ix] = a[:9]
        b.view(sn, 3)[ix] = a[9:]

    def cfl_dirs(self):
        return self.dt3

    def state(self):
        return self.s.blk.arrays["p"].copy(), self.s.blk.arrays["ps"].copy()
