"""Dump and restart files of a single block in the reference's formats, so
that runs of this library can be post-processed and restarted by the
reference's own tools, and the other way round.

* Parameter header: the field sequence of dump_params (dump.c:168-272), each
  field written on its own with the host's int (4 bytes) and double (8 bytes),
  little-endian, then the block list (n_ord, AMR time level, AMR node) per
  block. Written as `dumps<cnt>/parameters` and `rdumps<cnt % 2>/parameter`.
* Dump: dump_block (dump.c:276-...): float32 over the active zones in
  [i][j][z][var] order with NPRDUMP = 9 variables of an ideal-GRMHD build
  without CALC_MDOT: rho, u, u^0..u^3 (ucon_calc at the zone centre), and
  the cell-centred B^1..B^3. File `dumps<cnt>/new_dump0` (rank 0, one block).
* Restart: rdump_block_write (restart.c:54-76): float64 over the ghost-
  inclusive block in [i][j][z][var] order, the NPR primitives then NDIM
  face-field slots (slot 0 the unused component 0, slot d = B^d on the lower
  d-face times that face's sqrt(-g)). Files `rdumps<cnt % 2>/rdump0` and a
  `checkfile` (one int 0), as restart_write writes them.

Arrays in and out are in the library's layout (NPR planes of primitives,
3 planes of face field, plane stride ksize; see include/hamr_b200.h).
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass, field, fields

import numpy as np

NPR = 9
NDIM = 4
NPRDUMP = 9
FACE1, FACE2, CENT, FACE3 = 0, 1, 3, 4


@dataclass
class Params:
    """The dump_params header (dump.c:211-271), in write order. Counts and
    block sizes describe a run of one block."""
    t: float = 0.0
    n_active: int = 1
    n_active_total: int = 1
    nstep: int = 0
    DTd: float = 0.0
    DTl: float = 0.0
    DTr: float = 0.0
    dump_cnt: int = 0
    rdump_cnt: int = 0
    dt: float = 0.0
    failed: int = 0
    BS1: int = 0
    BS2: int = 0
    BS3: int = 0
    NB: int = 1
    NB1: int = 1
    NB2: int = 1
    NB3: int = 1
    startx1: float = 0.0
    startx2: float = 0.0
    startx3: float = 0.0
    dx1: float = 0.0
    dx2: float = 0.0
    dx3: float = 0.0
    tf: float = 0.0
    a: float = 0.0
    gam: float = 0.0
    cour: float = 0.0
    Rin: float = 0.0
    Rout: float = 0.0
    R0: float = 0.0            # mdot in CALC_MDOT builds
    # MASS_DENSITY_SCALE of the torus build (config.h:804, the M87 scaling)
    density: float = 0.001 * 0.00001 * 0.0000000002 * 3.1 * 0.000001 * 0.1 / 30.0
    lim: int = 0
    stag: int = 1              # STAGGERED
    dump_cnt_reduced: int = 0
    f1: int = 2                # REDUCE_FACTOR1-3 (config.h:578-580)
    f2: int = 2
    f3: int = 2
    r1: int = 1
    r2: int = 1
    r3: int = 1
    nl: int = 1
    rd: int = 0
    rt: int = 5000000          # (int) RTRANS
    rb: int = 0                # (int) RB
    docyl: int = 0
    dk: int = 1                # DOKTOT
    blocks: list = field(default_factory=lambda: [(0, 0, 0)])   # (n_ord, AMR time level, AMR node)


_SCALAR_FIELDS = [f for f in fields(Params) if f.name != "blocks"]


def _fmt(f) -> str:
    return "<d" if f.type in (float, "float") else "<i"


def pack_params(prm: Params) -> bytes:
    out = bytearray()
    for f in _SCALAR_FIELDS:
        v = getattr(prm, f.name)
        out += struct.pack(_fmt(f), float(v) if _fmt(f) == "<d" else int(v))
    for n_ord, level, node in prm.blocks:
        out += struct.pack("<iii", int(n_ord), int(level), int(node))
    return bytes(out)


def unpack_params(buf: bytes) -> Params:
    prm = Params(blocks=[])
    off = 0
    for f in _SCALAR_FIELDS:
        fmt = _fmt(f)
        (v,) = struct.unpack_from(fmt, buf, off)
        off += struct.calcsize(fmt)
        setattr(prm, f.name, v)
    while off + 12 <= len(buf):
        prm.blocks.append(struct.unpack_from("<iii", buf, off))
        off += 12
    return prm


def _views(pb_like, p, ps):
    n1, n2, n3, ng = pb_like.n1, pb_like.n2, pb_like.n3, pb_like.ng
    g1, g2 = n1 + 2 * ng, n2 + 2 * ng
    g3 = n3 + 2 * ng if n3 > 1 else 1
    ks = pb_like.ksize
    n = g1 * g2 * g3
    pv = np.asarray(p).reshape(NPR, ks)[:, :n].reshape(NPR, g1, g2, g3)
    sv = np.asarray(ps).reshape(3, ks)[:, :n].reshape(3, g1, g2, g3)
    return pv, sv, (g1, g2, g3)


def _geo_plane(geo, name, comp, loc, g1, g2):
    a = getattr(geo, name)
    k = comp * 5 + loc if name in ("gcov", "gcon") else loc
    return a[k * geo.gsize:k * geo.gsize + g1 * g2].reshape(g1, g2)


def ucon_centre(pb_like, p, geo) -> np.ndarray:
    """u^mu at the zone centres (ucon_calc, GPU_phys_mhd.h:692-716): gamma from
    the relative velocity u~^i and the spatial metric, u^0 = gamma/alpha,
    u^i = u~^i - gamma beta^i/alpha; shape (4, g1, g2, g3)."""
    pv, _, (g1, g2, g3) = _views(pb_like, p, np.zeros(3 * pb_like.ksize))
    gc = lambda s: _geo_plane(geo, "gcov", s, CENT, g1, g2)[:, :, None]
    gn = lambda s: _geo_plane(geo, "gcon", s, CENT, g1, g2)[:, :, None]
    u1, u2, u3 = pv[2], pv[3], pv[4]
    qsq = (gc(4) * u1 * u1 + gc(7) * u2 * u2 + gc(9) * u3 * u3
           + 2. * (gc(5) * u1 * u2 + gc(6) * u1 * u3 + gc(8) * u2 * u3))
    gamma = np.where(qsq < 0., np.where(np.abs(qsq) > 1e-10, 1.0, np.sqrt(1. + 1e-10)), np.sqrt(1. + np.abs(qsq)))
    alpha = 1. / np.sqrt(-gn(0))
    out = np.empty((4, g1, g2, g3))
    out[0] = gamma / alpha
    for j, u in zip((1, 2, 3), (u1, u2, u3)):
        beta = gn(j) * alpha * alpha
        out[j] = u - gamma * beta / alpha
    return out


def dump_array(pb_like, p, geo) -> np.ndarray:
    """The dump_block float array over the active zones, [i][j][z][NPRDUMP]."""
    pv, _, _ = _views(pb_like, p, np.zeros(3 * pb_like.ksize))
    ng = pb_like.ng
    g3 = ng if pb_like.n3 > 1 else 0
    act = (slice(ng, ng + pb_like.n1), slice(ng, ng + pb_like.n2), slice(g3, g3 + pb_like.n3))
    uc = ucon_centre(pb_like, p, geo)
    out = np.empty((pb_like.n1, pb_like.n2, pb_like.n3, NPRDUMP), np.float32)
    out[..., 0] = pv[0][act]
    out[..., 1] = pv[1][act]
    for k in range(4):
        out[..., 2 + k] = uc[k][act]
    for k in range(3):
        out[..., 6 + k] = pv[5 + k][act]
    return out


def restart_array(pb_like, p, ps, geo) -> np.ndarray:
    """The rdump_block_write float64 array over the ghost-inclusive block,
    [i][j][z][NPR + NDIM]."""
    pv, sv, (g1, g2, g3) = _views(pb_like, p, ps)
    out = np.zeros((g1, g2, g3, NPR + NDIM))
    for k in range(NPR):
        out[..., k] = pv[k]
    out[..., NPR] = 0.0   # the face field's unused component 0
    for d, loc in ((1, FACE1), (2, FACE2), (3, FACE3)):
        gd = _geo_plane(geo, "gdet", 0, loc, g1, g2)[:, :, None]
        out[..., NPR + d] = sv[d - 1] * gd
    return out


def restart_state(pb_like, arr, geo):
    """(p, ps) in the library's layout from a restart array (the face slots
    divided by the face sqrt(-g), as the reference's restart read does)."""
    g1, g2, g3 = arr.shape[:3]
    ks = pb_like.ksize
    n = g1 * g2 * g3
    p = np.zeros(NPR * ks)
    ps = np.zeros(3 * ks)
    pv = p.reshape(NPR, ks)[:, :n].reshape(NPR, g1, g2, g3)
    sv = ps.reshape(3, ks)[:, :n].reshape(3, g1, g2, g3)
    for k in range(NPR):
        pv[k] = arr[..., k]
    for d, loc in ((1, FACE1), (2, FACE2), (3, FACE3)):
        gd = _geo_plane(geo, "gdet", 0, loc, g1, g2)[:, :, None]
        with np.errstate(divide="ignore", invalid="ignore"):
            sv[d - 1] = np.where(gd != 0., arr[..., NPR + d] / gd, 0.)
    return p, ps


def params_for(pb_like, t=0.0, nstep=0, dt=0.0, spin=0.0, rin=0.0, rout=0.0, tf=0.0, startx=None, **kw) -> Params:
    sx = startx if startx is not None else getattr(pb_like, "startx", (0.0, 0.0, 0.0, 0.0))
    # REF_d is 0 for a direction of one zone (config.h:373-387)
    kw.setdefault("r1", int(pb_like.n1 > 1))
    kw.setdefault("r2", int(pb_like.n2 > 1))
    kw.setdefault("r3", int(pb_like.n3 > 1))
    return Params(t=t, nstep=nstep, dt=dt, BS1=pb_like.n1, BS2=pb_like.n2, BS3=pb_like.n3,
                  startx1=float(sx[1]), startx2=float(sx[2]), startx3=float(sx[3]),
                  dx1=float(pb_like.dx[0]), dx2=float(pb_like.dx[1]), dx3=float(pb_like.dx[2]),
                  tf=tf, a=spin, gam=float(pb_like.gam), cour=float(pb_like.cour), Rin=rin, Rout=rout, **kw)


def write_dump(root, pb_like, p, geo, prm: Params):
    """dumps<cnt>/parameters and dumps<cnt>/new_dump0."""
    d = os.path.join(root, f"dumps{prm.dump_cnt}")
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "parameters"), "wb") as f:
        f.write(pack_params(prm))
    dump_array(pb_like, p, geo).tofile(os.path.join(d, "new_dump0"))
    return d


def read_dump(root, cnt, shape):
    """(Params, float32 array [n1][n2][n3][NPRDUMP]) of dumps<cnt>."""
    d = os.path.join(root, f"dumps{cnt}")
    prm = unpack_params(open(os.path.join(d, "parameters"), "rb").read())
    arr = np.fromfile(os.path.join(d, "new_dump0"), np.float32).reshape(*shape, NPRDUMP)
    return prm, arr


def write_restart(root, pb_like, p, ps, geo, prm: Params):
    """rdumps<cnt % 2>/{checkfile, parameter, rdump0} as restart_write does."""
    d = os.path.join(root, f"rdumps{prm.rdump_cnt % 2}")
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "checkfile"), "wb") as f:
        f.write(struct.pack("<i", 0))
    with open(os.path.join(d, "parameter"), "wb") as f:
        f.write(pack_params(prm))
    restart_array(pb_like, p, ps, geo).tofile(os.path.join(d, "rdump0"))
    return d


def read_restart(root, pb_like, geo, cnt=0):
    """(Params, p, ps) from rdumps<cnt % 2>."""
    d = os.path.join(root, f"rdumps{cnt % 2}")
    prm = unpack_params(open(os.path.join(d, "parameter"), "rb").read())
    ng = pb_like.ng
    g1, g2 = pb_like.n1 + 2 * ng, pb_like.n2 + 2 * ng
    g3 = pb_like.n3 + 2 * ng if pb_like.n3 > 1 else 1
    arr = np.fromfile(os.path.join(d, "rdump0"), np.float64).reshape(g1, g2, g3, NPR + NDIM)
    p, ps = restart_state(pb_like, arr, geo)
    return prm, p, ps
