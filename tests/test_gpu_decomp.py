"""Domains decomposed along x1 or x2 on one GPU (hamr_gamma_wind_b200.decomp):
slabs as Blocks with halo sides, halos packed and unpacked by the library's
kernels (hamr_halo_pack / hamr_halo_unpack) in the undivided block's fill
order (x1 halos between the x1 and x3 ghost fills, x2 halos after the x2
fill, the poles with the end slabs), against the undivided Block. Every slab runs the same kernels on the
same data as the undivided block (the step-size reduction is a minimum), so
in either build the domain must match it bit for bit, step sizes included."""
import ctypes
from dataclasses import replace

import numpy as np
import pytest
import torch

from hamr_gamma_wind_b200 import _lib, decomp, problems
from hamr_gamma_wind_b200.api import Block

pytestmark = pytest.mark.gpu

CASES = {
    "torus3d": (lambda: problems.fm_torus(32, 16, 8, rout=40.0), [12, 20], 1),
    "torus2d": (lambda: problems.fm_torus(48, 48, 1, rout=40.0), [10, 16, 22], 1),
    "torus3d_x2": (lambda: problems.fm_torus(24, 24, 8, rout=40.0), [7, 9, 8], 2),
    "torus2d_x2": (lambda: problems.fm_torus(40, 48, 1, rout=40.0), [20, 28], 2),
}


def _stream_handle(stream):
    return ctypes.c_void_p(stream.cuda_stream).value


def _undivided(pb, strict, stream, **kw):
    blk = Block(**pb.block_kwargs(), strict=strict, stream=stream, **kw)
    blk.set_geometry(pb.geo)
    blk.upload(pb.p, pb.ps)
    blk.bound()
    p0, ps0 = blk.download()
    return blk, replace(pb, p=p0, ps=ps0)


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("strict,kw", [(True, {}), (False, {}), (True, dict(precision="mixed")),
                                       (True, dict(riemann="hllc"))])
def test_slabs_match_undivided_block(case, strict, kw):
    make, widths, axis = CASES[case]
    stream = torch.cuda.Stream()
    h = _stream_handle(stream)
    blk, pb = _undivided(make(), strict, h, **kw)
    slabs = decomp.split(pb, widths, axis=axis)
    gs = decomp.gpu_slabs(slabs, h, strict=strict, **kw)
    stepper = decomp.SlabStepper(gs, decomp.LocalExchange(), axis=axis)
    dt = 0.2 * min(pb.dx[:2])
    for _ in range(3):
        dn_full = blk.step(dt)
        dn_slab = stepper.step(dt)
        assert dn_slab == dn_full
        dt = min(dn_full, 1.3 * dt)
    p, ps = decomp.join(pb, slabs, [g.block.download() for g in gs])
    pf, psf = blk.download()
    np.testing.assert_array_equal(pb.active(p), pb.active(pf))
    np.testing.assert_array_equal(pb.active(ps), pb.active(psf))
    for g in gs:
        g.block.close()
    blk.close()


def test_halo_block_refuses_whole_steps():
    pb = problems.fm_torus(32, 16, 8, rout=40.0)
    sl = decomp.split(pb, [16, 16])[0]
    b = Block(**sl.block_kwargs(), halo=sl.halo)
    b.set_geometry(sl.geo)
    b.upload(sl.p, sl.ps)
    with pytest.raises(_lib.HamrError):
        b.step(0.01)
    # the larger of an x1 side's (G2 x G3) and an x2 side's (G1 x G3) message
    G1, G2, G3 = sl.n1 + 2 * pb.ng, pb.n2 + 2 * pb.ng, pb.n3 + 2 * pb.ng
    assert b.halo_count() == 12 * pb.ng * max(G1, G2) * G3
    b.close()


def test_x2_halo_side_refuses_a_pole():
    """An x2 side shared with a neighbour cannot be a pole."""
    pb = problems.fm_torus(24, 24, 8, rout=40.0)
    sl = decomp.split(pb, [12, 12], axis=2)[0]
    with pytest.raises(_lib.HamrError):
        Block(**dict(sl.block_kwargs(), poles=(1, 1)), halo=sl.halo)
