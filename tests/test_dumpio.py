"""Dump and restart files in the reference's formats (hamr_gamma_wind_b200.dumpio),
on the host: the parameter header's byte layout follows dump_params field by
field, the restart array carries the primitives and the face field times the
face sqrt(-g) over the ghost-inclusive block, the dump the active zones'
rho, u, u^mu, B^i in float32."""
import os
import struct
import tempfile

import numpy as np
import pytest

from hamr_gamma_wind_b200 import dumpio, problems


def _torus():
    return problems.fm_torus(24, 16, 8, rout=40.0)


def test_header_layout_follows_dump_params():
    pb = _torus()
    prm = dumpio.params_for(pb, t=12.5, nstep=40, dt=0.01, spin=0.9375, rin=1.0, rout=40.0, tf=2000.0)
    prm.dump_cnt, prm.rdump_cnt = 3, 7
    buf = dumpio.pack_params(prm)
    # t, n_active, n_active_total, nstep, DTd, DTl, DTr, dump_cnt, rdump_cnt, dt, failed
    assert struct.unpack_from("<diiidddiidi", buf, 0) == (12.5, 1, 1, 40, 0.0, 0.0, 0.0, 3, 7, 0.01, 0)
    off = struct.calcsize("<diiidddiidi")
    # block sizes and counts, then startx[1..3], dx[0][1..3]
    assert struct.unpack_from("<iiiiiii", buf, off) == (24, 16, 8, 1, 1, 1, 1)
    off += 7 * 4
    sx = struct.unpack_from("<dddddd", buf, off)
    assert sx[3:] == tuple(float(x) for x in pb.dx)
    off += 6 * 8
    # tf, a, gam, cour, Rin, Rout, R0, density
    assert struct.unpack_from("<dddddddd", buf, off)[:4] == (2000.0, 0.9375, pb.gam, pb.cour)
    off += 8 * 8
    # lim, stag, dump_cnt_reduced, f1-f3, r1-r3, nl, rd, rt, rb, docyl, dk: 15
    # ints, then one (n_ord, level, node) triple
    assert len(buf) == off + 15 * 4 + 3 * 4
    back = dumpio.unpack_params(buf)
    assert back == prm


def test_restart_round_trip_and_layout():
    pb = _torus()
    with tempfile.TemporaryDirectory() as root:
        prm = dumpio.params_for(pb, t=1.0, nstep=5, dt=0.02)
        d = dumpio.write_restart(root, pb, pb.p, pb.ps, pb.geo, prm)
        raw = np.fromfile(f"{d}/rdump0", np.float64)
        g1, g2, g3 = pb.g
        arr = raw.reshape(g1, g2, g3, dumpio.NPR + dumpio.NDIM)
        pv = pb.view(pb.p)
        np.testing.assert_array_equal(arr[..., :9], np.moveaxis(pv, 0, -1))
        gd1 = pb.geo.gdet[0 * pb.geo.gsize:0 * pb.geo.gsize + g1 * g2].reshape(g1, g2)
        np.testing.assert_array_equal(arr[..., 10], pb.view(pb.ps)[0] * gd1[:, :, None])
        assert open(f"{d}/checkfile", "rb").read() == struct.pack("<i", 0)
        prm2, p, ps = dumpio.read_restart(root, pb, pb.geo, cnt=prm.rdump_cnt)
        assert prm2 == prm
        np.testing.assert_array_equal(p, pb.p)
        # B^d = (B^d sqrt(-g)) / sqrt(-g): within one rounding of each value
        a, b = pb.view(ps), pb.view(pb.ps)
        assert np.all(np.abs(a - b) <= 2.3e-16 * np.abs(b))


def test_dump_variables_and_normalisation():
    pb = _torus()
    with tempfile.TemporaryDirectory() as root:
        prm = dumpio.params_for(pb)
        dumpio.write_dump(root, pb, pb.p, pb.geo, prm)
        prm2, arr = dumpio.read_dump(root, 0, (pb.n1, pb.n2, pb.n3))
    assert prm2 == prm and arr.dtype == np.float32
    act = pb.active(pb.p)
    np.testing.assert_array_equal(arr[..., 0], act[0].astype(np.float32))
    np.testing.assert_array_equal(arr[..., 6:9], np.moveaxis(act[5:8], 0, -1).astype(np.float32))
    # u^mu u_mu = -1 with the centre metric (in double, before the float cast)
    uc = dumpio.ucon_centre(pb, pb.p, pb.geo)
    g1, g2, g3 = pb.g
    gc = lambda s: pb.geo.gcov[(s * 5 + 3) * pb.geo.gsize:(s * 5 + 3) * pb.geo.gsize + g1 * g2].reshape(g1, g2)[:, :, None]
    sym = [[0, 1, 2, 3], [1, 4, 5, 6], [2, 5, 7, 8], [3, 6, 8, 9]]
    norm = sum(gc(sym[a][b]) * uc[a] * uc[b] for a in range(4) for b in range(4))
    ng = pb.ng
    np.testing.assert_allclose(norm[ng:ng + pb.n1, ng:ng + pb.n2, ng:ng + pb.n3], -1.0, atol=1e-12)
    np.testing.assert_array_equal(arr[..., 2:6], np.moveaxis(uc[:, ng:ng + pb.n1, ng:ng + pb.n2, ng:ng + pb.n3],
                                                             0, -1).astype(np.float32))


def _ours(tmp_path, pb, prm):
    ours = tmp_path / "ours"
    ddir = dumpio.write_dump(str(ours), pb, pb.p, pb.geo, prm)
    rdir = dumpio.write_restart(str(ours), pb, pb.p, pb.ps, pb.geo, prm)
    return (open(f"{ddir}/parameters", "rb").read(), open(f"{ddir}/new_dump0", "rb").read(),
            open(f"{rdir}/rdump0", "rb").read())


def _same_files(ref, ours):
    """byte for byte, except the 8 bytes of DTr in the header: dump_params
    writes sizeof(double) bytes from the int DTr (dump.c:216, decs.h:855), so
    its upper four bytes are whatever follows it in memory"""
    a, b = ref[0], ours[0]
    assert len(a) == len(b)
    dtr = struct.calcsize("<diiidd")   # offset of DTr
    assert a[:dtr + 4] == b[:dtr + 4] and a[dtr + 8:] == b[dtr + 8:]
    assert ref[1] == ours[1], "float dump differs"
    assert ref[2] == ours[2], "restart differs"


@pytest.mark.parametrize("variant", ["t3", "t2"])
def test_files_match_the_reference_writers(variant, tmp_path):
    """dumpio's parameter header, dump and restart files against the ones the
    reference's own writers produce (dump_params, dump_block,
    rdump_block_write from dump.c and restart.c, host-built for the block of
    the variant, oracle/ref_dumpio.c) for the same state and metric."""
    from oracle import oracle as O
    from tests.golden.make_golden import dump_case
    if not O.ref_dump_available(variant):
        pytest.skip("reference host build not present")
    pb, prm, prm_d, prm_i = dump_case(variant)
    ref = tmp_path / "ref"
    ref.mkdir()
    paths = [str(ref / f) for f in ("parameters", "new_dump0", "rdump0")]
    O.ref_dump_files(variant, pb.p, pb.ps, pb.ksize, pb.geo, prm_d, prm_i, *paths)
    _same_files([open(pth, "rb").read() for pth in paths], _ours(tmp_path, pb, prm))


def test_files_match_the_reference_golden_files(tmp_path):
    """The same against the committed output of the reference's writers
    (tests/golden/ref_dump_t2.npz), where the reference is absent."""
    from tests.golden.make_golden import digest, dump_case
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_dump_t2.npz"))
    pb, prm, _, _ = dump_case("t2")
    assert str(g["inputs"]) == digest(pb.p, pb.ps, pb.geo.gcov, pb.geo.gcon, pb.geo.gdet)
    _same_files([g[k].tobytes() for k in ("params", "dump", "rdump")], _ours(tmp_path, pb, prm))
