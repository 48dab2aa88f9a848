"""Shared helpers of the GPU parity tests: run the CUDA block and the oracle
on the same state and metric tables."""
import numpy as np

from hamr_gamma_wind_b200.api import Block
from oracle import oracle as O

BCMAP = {"periodic": O.BC_PERIODIC, "outflow": O.BC_OUTFLOW, "pole_trans": O.BC_POLE_TRANS,
         "pole_refl": O.BC_POLE_REFL}


def make_pair(pb, strict=True, inversion="2d", recon="ppm", riemann="hll", floors=False, repair="none"):
    """CUDA block and oracle setup holding the same ghost-filled state."""
    blk = Block(**pb.block_kwargs(), strict=strict, inversion=inversion, recon=recon, riemann=riemann,
                floors=floors, repair=repair)
    blk.set_geometry(pb.geo)
    blk.upload(pb.p, pb.ps)
    blk.bound()
    p0, ps0 = blk.download()
    ob = O.Block(pb.n1, pb.n2, pb.n3, pb.ng, blk.ksize, blk.gsize)
    ob.arrays["p"][:] = p0
    ob.arrays["ps"][:] = ps0
    geo = O.Geometry(pb.geo.gsize, pb.geo.gcov, pb.geo.gcon, pb.geo.gdet, pb.geo.conn)
    s = O.Setup(ob, geo, pb.dx, pb.gam, pb.cour, pb.poles[0], pb.poles[1],
                tuple(BCMAP[b] for b in pb.bc), int(pb.ct_upwind), {"2d": 0, "nm": 1}[inversion],
                {"ppm": 0, "mc": 1}[recon], {"hll": 0, "hllc": 1, "hlld": 2}[riemann], 0, int(bool(floors)),
                {"none": 0, "reset": 1, "neighbours": 2}[repair])
    return blk, s


def oracle_step(s, dt):
    return O.step(lambda s_, f, Dt, d, c: O.oracle_stage(s_, f, Dt, d, c),
                  lambda s_, a, b: O.oracle_bound(s_, a, b), s, dt)


def field_rel_err(blk, p_dev, s, name="p"):
    """max over variables of max|a - b| / max|b| on the active zones."""
    a = blk.active(p_dev)
    b = s.blk.active(name)
    errs = []
    for k in range(a.shape[0]):
        scale = np.abs(b[k]).max()
        d = np.abs(a[k] - b[k]).max()
        errs.append(0.0 if d == 0 else d / max(scale, 1e-300))
    return np.array(errs)


def plant(pb, patch=3, frac=0.05, seed=13):
    """Negative energy (inversion fails) and near-vacuum zones (floors)."""
    P = pb.active(pb.p)
    rng = np.random.default_rng(seed)
    fail = rng.random(P[0].shape) < frac
    i0, j0 = P.shape[1] // 3, P.shape[2] // 2
    dz = patch if P.shape[3] > 1 else 1
    fail[i0:i0 + patch, j0:j0 + patch, :dz] = True
    P[1][fail] = -1e-2
    thin = (rng.random(P[0].shape) < frac) & ~fail
    P[0][thin] = 1e-24
    P[1][thin] = 1e-26
    return int(fail.sum()), int(thin.sum())
