"""The allocation-free step, for callers that may not allocate device memory
(inside another component's CUDA graph capture, or under a framework that owns
the whole device memory pool): hamr_step_noalloc advances caller-held device
buffers using only scratch arrays that live inside the library.

Checked through the C ABI against the context-based step (hamr_step) on the
same block, on two calls in a row -- the second call runs on scratch that still
holds the first call's contents. Same kernels in the same order, so the results
must agree to the parity tests' strict tolerance (1e-14 of each field's scale);
they are in fact expected to be identical. Collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from hamr_gamma_wind_b200 import _lib, problems
from hamr_gamma_wind_b200.api import Block

pytestmark = pytest.mark.gpu

TOL = 1e-14


def _params(pb, stream):
    bc = {"periodic": 0, "outflow": 1, "pole_trans": 2, "pole_refl": 3}
    return _lib.HamrParams(pb.n1, pb.n2, pb.n3, pb.ng, pb.ksize, pb.gsize, pb.dx[0], pb.dx[1], pb.dx[2],
                           pb.gam, pb.cour, pb.poles[0], pb.poles[1], bc[pb.bc[0]], bc[pb.bc[1]],
                           bc[pb.bc[2]], int(pb.ct_upwind), 0, stream)


def _rel(a, b):
    a = a.reshape(a.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    scale = np.maximum(np.abs(b).max(axis=1), 1e-300)
    return (np.abs(a - b).max(axis=1) / scale).max()


@pytest.mark.parametrize("case", ["torus3d", "ot"])
def test_noalloc_step_matches_context_step_twice(case):
    import torch
    pb = problems.fm_torus(24, 16, 8, rout=40.0) if case == "torus3d" else problems.orszag_tang(48)
    assert pb.ksize <= _lib.NOALLOC_MAX_CELLS
    L = _lib.load()
    # reference result: the context path
    blk = Block(**pb.block_kwargs())
    blk.set_geometry(pb.geo)
    blk.upload(pb.p, pb.ps)
    blk.bound()
    p0, ps0 = blk.download()
    dt = 0.2 * min(pb.dx[:2])
    dn_ctx = [blk.step(dt)]
    ref_states = [blk.download()]
    dn_ctx.append(blk.step(dt))
    ref_states.append(blk.download())
    blk.close()

    # the allocation-free path on caller-owned device buffers
    dev = torch.device("cuda")
    p_d = torch.from_numpy(p0.copy()).to(dev)
    ps_d = torch.from_numpy(ps0.copy()).to(dev)
    tabs = [torch.from_numpy(getattr(pb.geo, n).copy()).to(dev) for n in ("gcov", "gcon", "gdet", "conn")]
    stream = torch.cuda.current_stream()
    prm = _params(pb, ctypes.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    for call in range(2):
        dn = ctypes.c_double()
        rc = L.hamr_step_noalloc(ctypes.byref(prm), *[ctypes.c_void_p(t.data_ptr()) for t in tabs],
                                 ctypes.c_void_p(p_d.data_ptr()), ctypes.c_void_p(ps_d.data_ptr()), dt,
                                 ctypes.byref(dn))
        assert rc == 0, f"call {call}: rc {rc}"
        torch.cuda.synchronize()
        p_host = p_d.cpu().numpy()
        ps_host = ps_d.cpu().numpy()
        pr, psr = ref_states[call]
        assert _rel(pb.active(p_host), pb.active(pr)) <= TOL, f"call {call}: primitives differ"
        assert _rel(pb.active(ps_host), pb.active(psr)) <= TOL, f"call {call}: face field differs"
        assert abs(dn.value - dn_ctx[call]) <= TOL * dn_ctx[call]


def test_noalloc_rejects_oversized_block_before_device_work():
    L = _lib.load()
    pb = problems.fm_torus(64, 32, 32, rout=40.0)
    assert pb.ksize > _lib.NOALLOC_MAX_CELLS
    prm = _params(pb, None)
    dummy = ctypes.c_void_p(16)   # never dereferenced: the size check comes first
    rc = L.hamr_step_noalloc(ctypes.byref(prm), dummy, dummy, dummy, dummy, dummy, dummy, 0.01, None)
    assert rc == -1
