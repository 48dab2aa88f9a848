"""Domains split along x1 (or along x2) into slabs, one block per slab: the
reference's multi-block layout with its ghost exchange between neighbouring
blocks (boundcomP.c, GPU_boundcom*.cu, GPU_program2.cu), for one GPU holding
several slabs or one slab per GPU.

A sub-step of a domain split along x1 is, on every slab: the stage (fluxes,
constrained transport, update, inversion), the x1 ghost fill of the physical
sides, the halo exchange with the x1 neighbours, then the x3 and the x2 ghost
fills. Along x2 (slabs of whole (x1, x3) extent, the poles in the first and
the last slab): the x1, x3 and x2 fills (poles and physical sides), then the
x2 halo exchange, whose messages carry the x1 and x3 ghosts just filled.
Either is the order in which an undivided block fills its own ghosts (x1, x3,
x2), and every face shared by two slabs is computed by both from the same
data, so the decomposed step reproduces the undivided block bit for bit (no
EMF synchronisation is needed at a shared face, unlike the reference's
refinement boundaries). The step size is the undivided block's: the
per-direction CFL minima are reduced over all slabs first, then combined as
1/(1/d1 + 1/d2 + 1/d3) (step_ch.c:1320-1331).

A slab is anything with the methods the steppers call
(`stage`, `bound_dim`, `pack`, `unpack`, `cfl_dirs`); `GpuSlab` wraps a
`Block`. `LocalExchange` swaps halos between slabs of one process;
`DistributedExchange` sends them to the neighbouring ranks with
torch.distributed (NCCL between GPUs).
"""
from __future__ import annotations

from dataclasses import replace

import numpy as np

from .api import Block, Geometry
from .problems import Problem

LOWER, UPPER = 0, 1
HALO_LOWER, HALO_UPPER = 1, 2     # halo bits of an x1 split; an x2 split's are 4, 8


def split(pb: Problem, widths, axis: int = 1) -> list:
    """The slabs of `pb` along x1 (axis 1) or x2 (axis 2) with the given
    active widths (summing to n1 or n2; along x1 each at least ng, along x2
    at least ng + 2, so that the reflective pole's near-axis rows stay out of
    the exchanged layers): per slab a Problem holding the slice of the state
    and of the metric tables (ghost layers included, so the tables are the
    undivided block's to the bit), its halo sides (`halo` attribute), its
    offset along the axis and, along x2, its pole flags (the poles stay with
    the first and the last slab)."""
    widths = [int(n) for n in widths]
    if axis not in (1, 2):
        raise ValueError("slabs along x1 or x2")
    ntot, wmin = (pb.n1, pb.ng) if axis == 1 else (pb.n2, pb.ng + 2)
    if sum(widths) != ntot or min(widths) < wmin:
        raise ValueError(f"slab widths {widths} must sum to {ntot}, each at least {wmin}")
    if axis == 2 and pb.bc[1] == "periodic":
        raise ValueError("an x2 split needs non-periodic x2 boundaries")
    g1, g2, g3 = pb.g
    ng = pb.ng
    pv = pb.view(pb.p)
    sv = pb.view(pb.ps)
    out = []
    off = 0
    last = len(widths) - 1
    for k, n in enumerate(widths):
        G1 = n + 2 * ng if axis == 1 else g1
        G2 = g2 if axis == 1 else n + 2 * ng
        sl = (slice(None), slice(off, off + G1)) if axis == 1 else (slice(None), slice(None), slice(off, off + G2))
        ncell = G1 * G2 * g3
        ksize = ncell + (64 - ncell % 64)
        ngeo = G1 * G2
        gsize = ngeo + (64 - ngeo % 64)
        p = np.zeros(9 * ksize)
        ps = np.zeros(3 * ksize)
        p.reshape(9, ksize)[:, :ncell] = pv[sl].reshape(9, ncell)
        ps.reshape(3, ksize)[:, :ncell] = sv[sl].reshape(3, ncell)
        geo = Geometry(gsize)
        for name, planes in (("gcov", 50), ("gcon", 50), ("gdet", 5), ("conn", 40)):
            src = getattr(pb.geo, name).reshape(planes, pb.geo.gsize)[:, :g1 * g2].reshape(planes, g1, g2)
            dst = getattr(geo, name).reshape(planes, gsize)
            dst[:, :ngeo] = src[sl].reshape(planes, ngeo)
        startx = list(pb.startx)
        if len(startx) > axis:
            startx[axis] = startx[axis] + off * pb.dx[axis - 1]
        lo_bit, hi_bit = (HALO_LOWER, HALO_UPPER) if axis == 1 else (4, 8)
        if axis == 1:
            slab = replace(pb, n1=n, ksize=ksize, gsize=gsize, geo=geo, p=p, ps=ps, startx=tuple(startx))
        else:
            poles = (pb.poles[0] if k == 0 else 0, pb.poles[1] if k == last else 0)
            slab = replace(pb, n2=n, ksize=ksize, gsize=gsize, geo=geo, p=p, ps=ps, startx=tuple(startx),
                           poles=poles)
        slab.halo = (lo_bit if k > 0 else 0) | (hi_bit if k < last else 0)
        slab.offset = off
        slab.axis = axis
        out.append(slab)
        off += n
    return out


def join(pb: Problem, slabs, states) -> tuple:
    """The undivided block's (p, ps) assembled from the slabs' active layers
    (states: per slab its (p, ps) in the slab's layout); ghosts of pb kept."""
    p = pb.p.copy()
    ps = pb.ps.copy()
    pv, sv = pb.view(p), pb.view(ps)
    ng = pb.ng
    for sl, (a, b) in zip(slabs, states):
        av, bv = sl.view(a), sl.view(b)
        axis = getattr(sl, "axis", 1)
        n = sl.n1 if axis == 1 else sl.n2
        i0 = ng + sl.offset
        if axis == 1:
            pv[:, i0:i0 + n] = av[:, ng:ng + n]
            sv[:, i0:i0 + n] = bv[:, ng:ng + n]
        else:
            pv[:, :, i0:i0 + n] = av[:, :, ng:ng + n]
            sv[:, :, i0:i0 + n] = bv[:, :, ng:ng + n]
    return p, ps


def cfl_step(dmin) -> float:
    """1/(1/d1 + 1/d2 + 1/d3), in the operation order of the device's
    k_dt_finalize."""
    d1, d2, d3 = (float(x) for x in dmin)
    return 1. / (1. / d1 + 1. / d2 + 1. / d3)


class SlabStepper:
    """RK2 steps of the slabs this process holds, split along `axis` (1 or
    2), halos swapped by `exchange` (an object with `swap(slabs, full,
    axis)` and `min_dirs(d3)`)."""

    def __init__(self, slabs, exchange, axis: int = 1):
        self.slabs = list(slabs)
        self.exchange = exchange
        self.axis = axis

    def fill(self, full: int):
        """Ghost fill of the state the last sub-step wrote (full: p, ps),
        in the undivided block's order."""
        for s in self.slabs:
            s.bound_dim(full, 1)
        if self.axis == 1:
            self.exchange.swap(self.slabs, full, 1)
        for s in self.slabs:
            s.bound_dim(full, 3)
        for s in self.slabs:
            s.bound_dim(full, 2)
        if self.axis == 2:
            self.exchange.swap(self.slabs, full, 2)

    def substep(self, full: int, Dt: float, dt: float):
        for s in self.slabs:
            s.stage(full, Dt, dt)
        self.fill(full)

    def step(self, dt: float) -> float:
        """One RK2 step of size dt; returns the CFL step of its full sub-step
        over the whole domain."""
        self.substep(0, 0.5 * dt, dt)
        self.substep(1, dt, dt)
        d = np.min(np.array([s.cfl_dirs() for s in self.slabs]), axis=0)
        return cfl_step(self.exchange.min_dirs(d))


class GpuSlab:
    """A Block as a slab: halo messages in device buffers (torch tensors on
    the block's device)."""

    def __init__(self, block: Block, device=None):
        import torch
        self.block = block
        n = block.halo_count()
        dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.send = [torch.empty(n, dtype=torch.float64, device=dev) for _ in range(2)]
        self.recv = [torch.empty(n, dtype=torch.float64, device=dev) for _ in range(2)]

    def stage(self, full, Dt, dt):
        self.block.advance_stage(full, Dt, dt)

    def bound_dim(self, full, dim):
        self.block.bound_dim(full, dim)

    def pack(self, full, side):
        """side 0, 1: x1 lower, upper; 2, 3: x2 lower, upper"""
        self.block.halo_pack(full, side, self.send[side & 1].data_ptr())
        return self.send[side & 1]

    def recv_buffer(self, side):
        return self.recv[side & 1]

    def unpack(self, full, side, buf):
        self.block.halo_unpack(full, side, buf.data_ptr())

    def cfl_dirs(self):
        return self.block.cfl_dirs()


class LocalExchange:
    """Halos between consecutive slabs of this process (slab k's upper side
    faces slab k+1's lower side). All slabs must run on one stream, so that
    packs, copies and unpacks are ordered."""

    def swap(self, slabs, full, axis=1):
        o = 2 * (axis - 1)   # side codes of the axis
        msgs = []
        for a, b in zip(slabs[:-1], slabs[1:]):
            msgs.append((a, o + UPPER, b.pack(full, o + LOWER)))
            msgs.append((b, o + LOWER, a.pack(full, o + UPPER)))
        for s, side, buf in msgs:
            s.unpack(full, side, buf)

    def min_dirs(self, d):
        return d


class DistributedExchange:
    """One slab per rank, ranks in x1 order: the upper side of rank r faces
    the lower side of rank r + 1. Messages go by point-to-point
    torch.distributed calls (NCCL: device buffers; gloo: host buffers); the
    CFL minima by an all-reduce (MIN). Every rank takes the same collective
    steps in the same order."""

    def __init__(self, rank: int, world: int, group=None):
        self.rank, self.world, self.group = rank, world, group

    def swap(self, slabs, full, axis=1):
        import torch.distributed as dist
        (s,) = slabs
        o = 2 * (axis - 1)   # side codes of the axis
        ops, recvs = [], []
        for side, peer in ((o + LOWER, self.rank - 1), (o + UPPER, self.rank + 1)):
            if 0 <= peer < self.world:
                buf = s.recv_buffer(side)
                ops.append(dist.P2POp(dist.isend, s.pack(full, side), peer, group=self.group))
                ops.append(dist.P2POp(dist.irecv, buf, peer, group=self.group))
                recvs.append((side, buf))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for side, buf in recvs:
            s.unpack(full, side, buf)

    def min_dirs(self, d):
        import torch
        import torch.distributed as dist
        dev = "cuda" if dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.tensor(np.asarray(d, dtype=np.float64), device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
        return t.cpu().numpy()


def gpu_slabs(slab_problems, stream, strict=False, **block_kwargs):
    """Blocks for the slabs (geometry and state uploaded) wrapped as
    GpuSlab, all on `stream` (a cudaStream_t handle shared by the slabs, so
    that LocalExchange's packs, unpacks and the stages are ordered)."""
    if not stream:
        raise ValueError("slabs on one GPU need one shared stream")
    out = []
    for sp in slab_problems:
        b = Block(**sp.block_kwargs(), halo=sp.halo, stream=stream, strict=strict, **block_kwargs)
        b.set_geometry(sp.geo)
        b.upload(sp.p, sp.ps)
        out.append(GpuSlab(b))
    return out
