"""Domains decomposed along x1 or x2 (hamr_gamma_wind_b200.decomp), on the
host: the oracle as the slabs, driven by the same steppers the GPU blocks use.

Split into slabs with halo sides and stepped with the halo exchange in the
undivided block's fill order (along x1 between the x1 and x3 ghost fills,
along x2 after the x2 fill, the poles staying with the first and last slab),
the domain must reproduce the undivided block bit for bit, step size
included; over two and three gloo ranks (one slab each, halos by
point-to-point messages, CFL minima by an all-reduce) as well.
"""
import os
import tempfile
from dataclasses import replace

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from hamr_gamma_wind_b200 import decomp, problems
from oracle import oracle as O
from tests._decomp import OracleSlab, oracle_setup
from tests._gpu import oracle_step

CASES = {
    "torus3d": (lambda: problems.fm_torus(32, 16, 8, rout=40.0), [12, 20], 1),
    "torus2d": (lambda: problems.fm_torus(48, 48, 1, rout=40.0), [10, 16, 22], 1),
    # along x2: transmissive poles (3-D) and reflective poles (2-D, with the
    # near-axis row fix) in the first and last slabs
    "torus3d_x2": (lambda: problems.fm_torus(24, 24, 8, rout=40.0), [7, 9, 8], 2),
    "torus2d_x2": (lambda: problems.fm_torus(40, 48, 1, rout=40.0), [20, 28], 2),
}


def bound_problem(pb):
    """pb with its ghost zones filled (the undivided block's fill)."""
    s = oracle_setup(pb)
    O.oracle_bound(s)
    return replace(pb, p=s.blk.arrays["p"].copy(), ps=s.blk.arrays["ps"].copy()), s


def test_split_join_round_trip():
    pb, _ = bound_problem(problems.fm_torus(32, 16, 8, rout=40.0))
    slabs = decomp.split(pb, [7, 12, 13])
    assert [s.halo for s in slabs] == [2, 3, 1]
    assert [s.offset for s in slabs] == [0, 7, 19]
    p, ps = decomp.join(pb, slabs, [(s.p, s.ps) for s in slabs])
    np.testing.assert_array_equal(p, pb.p)
    np.testing.assert_array_equal(ps, pb.ps)
    # a slab's metric tables are the undivided block's rows, ghosts included
    g1, g2, _ = pb.g
    full = pb.geo.gcov.reshape(50, pb.geo.gsize)[:, :g1 * g2].reshape(50, g1, g2)
    s1 = slabs[1]
    G1 = s1.n1 + 2 * pb.ng
    part = s1.geo.gcov.reshape(50, s1.geo.gsize)[:, :G1 * g2].reshape(50, G1, g2)
    np.testing.assert_array_equal(part, full[:, 7:7 + G1])
    with pytest.raises(ValueError):
        decomp.split(pb, [2, 30])
    with pytest.raises(ValueError):
        decomp.split(pb, [10, 10])
    # along x2: halo bits 4 and 8, the poles with the end slabs
    x2 = decomp.split(pb, [5, 6, 5], axis=2)
    assert [s.halo for s in x2] == [8, 12, 4]
    assert [s.poles for s in x2] == [(pb.poles[0], 0), (0, 0), (0, pb.poles[1])]
    p, ps = decomp.join(pb, x2, [(s.p, s.ps) for s in x2])
    np.testing.assert_array_equal(p, pb.p)
    np.testing.assert_array_equal(ps, pb.ps)
    with pytest.raises(ValueError):
        decomp.split(pb, [4, 12], axis=2)   # narrower than ng + 2


@pytest.mark.parametrize("case", list(CASES))
def test_oracle_slabs_match_undivided_block(case):
    make, widths, axis = CASES[case]
    pb, s_full = bound_problem(make())
    slabs = decomp.split(pb, widths, axis=axis)
    stepper = decomp.SlabStepper([OracleSlab(sp) for sp in slabs], decomp.LocalExchange(), axis=axis)
    dt = 0.2 * min(pb.dx[:2])
    for _ in range(3):
        dn_full = oracle_step(s_full, dt)
        dn_slab = stepper.step(dt)
        assert dn_slab == dn_full
        dt = min(dn_full, 1.3 * dt)
    p, ps = decomp.join(pb, slabs, [sl.state() for sl in stepper.slabs])
    np.testing.assert_array_equal(pb.active(p), s_full.blk.active("p"))
    np.testing.assert_array_equal(pb.active(ps), s_full.blk.active("ps"))


WIDTHS = {(2, 1): [14, 18], (3, 1): [10, 9, 13], (2, 2): [7, 9]}


def _rank(rank, world, path, port, axis=1):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        pb, _ = bound_problem(problems.fm_torus(32, 16, 8, rout=40.0))
        slabs = decomp.split(pb, WIDTHS[world, axis], axis=axis)
        me = OracleSlab(slabs[rank])
        stepper = decomp.SlabStepper([me], decomp.DistributedExchange(rank, world), axis=axis)
        dt = 0.2 * min(pb.dx[:2])
        dts = []
        for _ in range(2):
            dn = stepper.step(dt)
            dts.append(dn)
            dt = min(dn, 1.3 * dt)
        p, ps = me.state()
        np.savez(os.path.join(path, f"rank{rank}.npz"), p=p, ps=ps, dts=np.array(dts))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,axis", [(2, 1), (3, 1), (2, 2)])
def test_gloo_ranks_match_undivided_block(world, axis):
    """One slab per rank (the middle rank of three exchanges with both
    neighbours; along x2 each rank holds one pole), halos and the CFL
    minimum over gloo: bit for bit the undivided block, step sizes
    included."""
    with tempfile.TemporaryDirectory() as path:
        port = 29500 + (os.getpid() + 97 * world + 31 * axis) % 2000
        mp.spawn(_rank, args=(world, path, port, axis), nprocs=world, join=True)
        pb, s_full = bound_problem(problems.fm_torus(32, 16, 8, rout=40.0))
        slabs = decomp.split(pb, WIDTHS[world, axis], axis=axis)
        dt = 0.2 * min(pb.dx[:2])
        dts = []
        for _ in range(2):
            dn = oracle_step(s_full, dt)
            dts.append(dn)
            dt = min(dn, 1.3 * dt)
        res = [np.load(os.path.join(path, f"rank{r}.npz")) for r in range(world)]
        for r in res:
            np.testing.assert_array_equal(r["dts"], np.array(dts))
        p, ps = decomp.join(pb, slabs, [(r["p"], r["ps"]) for r in res])
        np.testing.assert_array_equal(pb.active(p), s_full.blk.active("p"))
        np.testing.assert_array_equal(pb.active(ps), s_full.blk.active("ps"))
