"""Domains split along x1 into slabs, one block per slab: the reference's
multi-block layout along r with its ghost exchange between neighbouring
blocks (boundcomP.c, GPU_boundcom*.cu, GPU_program2.cu), for one GPU holding
several slabs or one slab per GPU.

A sub-step of the decomposed domain is, on every slab: the stage (fluxes,
constrained transport, update, inversion), the x1 ghost fill of the physical
sides, the halo exchange with the x1 neighbours, then the x3 and the x2 ghost
fills. That is the order in which an undivided block fills its own ghosts
(x1, x3, x2), and every face shared by two slabs is computed by both from the
same data, so the decomposed step reproduces the undivided block bit for bit
(no EMF synchronisation is needed at a shared face, unlike the reference's
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
HALO_LOWER, HALO_UPPER = 1, 2


def split(pb: Problem, n1s) -> list:
    """The slabs of `pb` along x1 with the given active widths (summing to
    pb.n1, each at least ng): per slab a Problem holding the slice of the
    state and of the metric tables (ghost layers included, so the tables are
    the undivided block's to the bit) and its halo sides (`halo` attribute,
    bit 0 lower, bit 1 upper)."""
    n1s = [int(n) for n in n1s]
    if sum(n1s) != pb.n1 or min(n1s) < pb.ng:
        raise ValueError(f"slab widths {n1s} must sum to n1 = {pb.n1}, each at least ng = {pb.ng}")
    g1, g2, g3 = pb.g
    ng = pb.ng
    pv = pb.view(pb.p)
    sv = pb.view(pb.ps)
    out = []
    off = 0
    for k, n in enumerate(n1s):
        G1 = n + 2 * ng
        ncell = G1 * g2 * g3
        ksize = ncell + (64 - ncell % 64)
        ngeo = G1 * g2
        gsize = ngeo + (64 - ngeo % 64)
        p = np.zeros(9 * ksize)
        ps = np.zeros(3 * ksize)
        p.reshape(9, ksize)[:, :ncell] = pv[:, off:off + G1].reshape(9, ncell)
        ps.reshape(3, ksize)[:, :ncell] = sv[:, off:off + G1].reshape(3, ncell)
        geo = Geometry(gsize)
        for name, planes in (("gcov", 50), ("gcon", 50), ("gdet", 5), ("conn", 40)):
            src = getattr(pb.geo, name).reshape(planes, pb.geo.gsize)[:, :g1 * g2].reshape(planes, g1, g2)
            dst = getattr(geo, name).reshape(planes, gsize)
            dst[:, :ngeo] = src[:, off:off + G1].reshape(planes, ngeo)
        startx = tuple(pb.startx)
        if len(startx) > 1:
            startx = (startx[0], startx[1] + off * pb.dx[0]) + tuple(startx[2:])
        slab = replace(pb, n1=n, ksize=ksize, gsize=gsize, geo=geo, p=p, ps=ps, startx=startx)
        slab.halo = (HALO_LOWER if k > 0 else 0) | (HALO_UPPER if k < len(n1s) - 1 else 0)
        slab.offset = off
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
        i0 = ng + sl.offset
        pv[:, i0:i0 + sl.n1] = av[:, ng:ng + sl.n1]
        sv[:, i0:i0 + sl.n1] = bv[:, ng:ng + sl.n1]
    return p, ps


def cfl_step(dmin) -> float:
    """1/(1/d1 + 1/d2 + 1/d3), in the operation order of the device's
    k_dt_finalize."""
    d1, d2, d3 = (float(x) for x in dmin)
    return 1. / (1. / d1 + 1. / d2 + 1. / d3)


class SlabStepper:
    """RK2 steps of the slabs this process holds, halos swapped by `exchange`
    (an object with `swap(slabs, full)` and `min_dirs(d3)`)."""

    def __init__(self, slabs, exchange):
        self.slabs = list(slabs)
        self.exchange = exchange

    def fill(self, full: int):
        """Ghost fill of the state the last sub-step wrote (full: p, ps),
        in the undivided block's order."""
        for s in self.slabs:
            s.bound_dim(full, 1)
        self.exchange.swap(self.slabs, full)
        for s in self.slabs:
            s.bound_dim(full, 3)
        for s in self.slabs:
            s.bound_dim(full, 2)

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
        self.block.halo_pack(full, side, self.send[side].data_ptr())
        return self.send[side]

    def recv_buffer(self, side):
        return self.recv[side]

    def unpack(self, full, side, buf):
        self.block.halo_unpack(full, side, buf.data_ptr())

    def cfl_dirs(self):
        return self.block.cfl_dirs()


class LocalExchange:
    """Halos between consecutive slabs of this process (slab k's upper side
    faces slab k+1's lower side). All slabs must run on one stream, so that
    packs, copies and unpacks are ordered."""

    def swap(self, slabs, full):
        msgs = []
        for a, b in zip(slabs[:-1], slabs[1:]):
            msgs.append((a, UPPER, b.pack(full, LOWER)))
            msgs.append((b, LOWER, a.pack(full, UPPER)))
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

    def swap(self, slabs, full):
        import torch.distributed as dist
        (s,) = slabs
        ops, recvs = [], []
        for side, peer in ((LOWER, self.rank - 1), (UPPER, self.rank + 1)):
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
