"""Test infrastructure (oracle) -- never imported by the product.

ctypes bindings for
  * ``liboracle.so``        the C restatement of the single-block RK2 sub-step
                            (oracle/hamr_oracle.c),
  * ``liboracle_fma.so``    the same sources compiled with fused multiply-add
                            contraction (selected inside ``contracted()``): how
                            far the step moves when its roundings change, the
                            envelope a contracted GPU build is held to, and
  * ``_ref/libref_<v>.so``  host builds of the reference's own kernels for the
                            compile-time variants listed in oracle/Makefile
                            (only present where the reference sources were).

Only tests, ``__graft_entry__.smoke`` and the CPU-baseline leg of ``bench.py``
use this module.
"""
from __future__ import annotations

import contextlib
import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NPR = 9
RHO, UU, U1, U2, U3, B1, B2, B3, KTOT = range(9)
FACE1, FACE2, CORN, CENT, FACE3 = range(5)
BC_PERIODIC, BC_OUTFLOW, BC_POLE_TRANS, BC_POLE_REFL = range(4)

_vp = ctypes.c_void_p
_d = ctypes.c_double
_i = ctypes.c_int


def _ptr(a):
    return a.ctypes.data_as(_vp)


class HoGrid(ctypes.Structure):
    _fields_ = [("n1", _i), ("n2", _i), ("n3", _i), ("ng", _i),
                ("ksize", ctypes.c_long), ("gsize", ctypes.c_long),
                ("dx1", _d), ("dx2", _d), ("dx3", _d), ("gam", _d), ("cour", _d),
                ("pole1", _i), ("pole2", _i), ("bc1", _i), ("bc2", _i), ("bc3", _i),
                ("inversion", _i), ("ct_upwind", _i), ("recon", _i), ("riemann", _i), ("halo", _i),
                ("floors", _i), ("repair", _i)]


class HoGeom(ctypes.Structure):
    _fields_ = [("gcov", _vp), ("gcon", _vp), ("gdet", _vp), ("conn", _vp)]


class HoState(ctypes.Structure):
    _fields_ = [(n, _vp) for n in ("p", "ph", "ps", "psh", "U", "F1", "F2", "F3",
                                   "E_cent", "emf", "pflag", "failimage")]


_libs: dict = {}
_variant = "liboracle.so"


@contextlib.contextmanager
def contracted():
    """Inside the block every oracle call runs the build with fused
    multiply-add contraction (liboracle_fma.so)."""
    global _variant
    old, _variant = _variant, "liboracle_fma.so"
    try:
        yield
    finally:
        _variant = old


def lib():
    """The restatement library (built by ``make -C oracle``)."""
    name = _variant
    if name not in _libs:
        path = os.path.join(HERE, name)
        if not os.path.exists(path):
            raise RuntimeError(f"oracle/{name} missing: run `make -C oracle`")
        L = ctypes.CDLL(path)
        L.ho_stage.argtypes = [ctypes.POINTER(HoGrid), ctypes.POINTER(HoGeom), ctypes.POINTER(HoState),
                               _i, _d, _d, _i, _vp]
        L.ho_bound.argtypes = [ctypes.POINTER(HoGrid), ctypes.POINTER(HoGeom), _vp, _vp]
        L.ho_bound_dim.argtypes = [ctypes.POINTER(HoGrid), ctypes.POINTER(HoGeom), _vp, _vp, _i]
        L.ho_para.argtypes = [_vp, _vp, _vp]
        L.ho_primtoflux.argtypes = [_d, _vp, _vp, _vp, _d, _i, _vp, _vp, _vp]
        for nm in ("ho_utoprim_2d", "ho_utoprim_1dvsq2fix1", "ho_utoprim_1dfix1", "ho_utoprim_nm"):
            f = getattr(L, nm)
            f.argtypes = [_d, _vp, _vp, _vp, _d, _vp]
            f.restype = _i
        L.ho_utoprim_nm_max_index.restype = _i
        L.ho_divb_max.argtypes = [ctypes.POINTER(HoGrid), ctypes.POINTER(HoGeom), _vp]
        L.ho_divb_max.restype = _d
        L.ho_set_mud.argtypes = [_vp, _vp, _i, _vp, _vp]
        L.ho_fixup_cell.argtypes = [_d, _vp, _vp, _vp, _d]
        L.ho_fixup_cell.restype = _i
        L.ho_fixup_utoprim.argtypes = [ctypes.POINTER(HoGrid), _vp, _vp, _vp]
        L.ho_build_geometry.argtypes = [_i, _d, _i, _i, _i, _i, ctypes.c_long, _vp, _vp, _vp, _vp, _vp, _vp]
        L.ho_build_geometry.restype = _i
        L.ho_bl_coord.argtypes = [_i, _d, _vp, _vp]
        L.ho_num_threads.restype = _i
        L.ho_div_rcp_mismatches.argtypes = [_vp, ctypes.c_long, _vp, ctypes.c_long]
        L.ho_div_rcp_mismatches.restype = ctypes.c_long
        L.ho_div_rcp_mismatches_g.argtypes = [_vp, ctypes.c_long, _vp, ctypes.c_long, ctypes.c_int]
        L.ho_div_rcp_mismatches_g.restype = ctypes.c_long
        _libs[name] = L
    return _libs[name]


def ref_available(variant: str) -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", f"libref_{variant}.so"))


_refs: dict = {}


def ref(variant: str):
    """Host build of the reference kernels for one compile-time variant."""
    if variant not in _refs:
        L = ctypes.CDLL(os.path.join(HERE, "_ref", f"libref_{variant}.so"))
        L.ref_dims.argtypes = [_vp, _vp]
        L.ref_stage.argtypes = ([_i, _d, _d, _d, _d, _d, _d, _i, _i] + [_vp] * 19 + [_i, _vp])
        L.ref_geometry.argtypes = [_d, _vp, _vp, _vp, _vp, _vp, _vp]
        L.ref_geometry.restype = _i
        L.ref_bound_pole_trans.argtypes = [_vp, _vp, _vp, _i, _i]
        for nm in ("ref_utoprim_2d", "ref_utoprim_1dvsq2fix1", "ref_utoprim_1dfix1", "ref_utoprim_nm"):
            f = getattr(L, nm)
            f.argtypes = [_vp, _vp, _vp, _d, _vp]
            f.restype = _i
        L.ref_primtoflux.argtypes = [_vp, _vp, _vp, _d, _i, _vp, _vp, _vp]
        L.ref_para.argtypes = [_vp, _vp, _vp]
        L.ref_bl_coord.argtypes = [_vp, _vp]
        L.ref_fixuputoprim.argtypes = [_vp] * 7
        L.ref_fixup_utoprim.argtypes = [_vp, _vp, _vp, ctypes.c_long]
        if hasattr(L, "ref_set_mud"):
            L.ref_set_mud.argtypes = [_vp, _vp]
            L.ref_mud_plane.restype = ctypes.c_long
            L.ref_nsolver.restype = _i
        _refs[variant] = L
    return _refs[variant]


def ref_dims(variant: str):
    L = ref(variant)
    dims = np.zeros(9, np.int64)
    gam = ctypes.c_double()
    L.ref_dims(_ptr(dims), ctypes.byref(gam))
    return dims, gam.value


def pad64(n: int) -> int:
    """Plane stride rule of the reference device buffers (GPU_program1.cu:92)."""
    return n + (64 - n % 64)


@dataclass
class Block:
    """One uniform block in the shared SoA layout."""
    n1: int
    n2: int
    n3: int
    ng: int = 3
    ksize: int = 0
    gsize: int = 0
    arrays: dict = field(default_factory=dict)

    def __post_init__(self):
        self.g1 = self.n1 + 2 * self.ng
        self.g2 = self.n2 + 2 * self.ng
        self.g3 = self.n3 + 2 * self.ng if self.n3 > 1 else 1
        self.ng3 = self.ng if self.n3 > 1 else 0
        if not self.ksize:
            self.ksize = pad64(self.g1 * self.g2 * self.g3)
        if not self.gsize:
            self.gsize = pad64(self.g1 * self.g2)
        ks = self.ksize
        for name, planes in (("p", NPR), ("ph", NPR), ("ps", 3), ("psh", 3), ("U", NPR),
                             ("F1", NPR), ("F2", NPR), ("F3", NPR), ("E_cent", 4), ("emf", 4),
                             ("dq1", NPR), ("dq2", NPR)):
            self.arrays[name] = np.zeros(planes * ks)
        self.arrays["pflag"] = np.zeros(ks, np.int32)
        self.arrays["failimage"] = np.zeros(5 * ks, np.int32)
        self.arrays["radius"] = np.zeros(max(self.g1, ks))

    def __getattr__(self, item):
        arrays = self.__dict__.get("arrays")
        if arrays is not None and item in arrays:
            return arrays[item]
        raise AttributeError(item)

    def view(self, name, planes=None):
        """(planes, g1, g2, g3) view of a cell array."""
        a = self.arrays[name]
        n = self.g1 * self.g2 * self.g3
        k = a.size // self.ksize if planes is None else planes
        return a.reshape(k, self.ksize)[:, :n].reshape(k, self.g1, self.g2, self.g3)

    def active(self, name, planes=None):
        v = self.view(name, planes)
        g, g3 = self.ng, self.ng3
        return v[:, g:g + self.n1, g:g + self.n2, g3:g3 + self.n3]

    def copy(self):
        b = Block(self.n1, self.n2, self.n3, self.ng, self.ksize, self.gsize)
        for k, v in self.arrays.items():
            b.arrays[k] = v.copy()
        return b


@dataclass
class Geometry:
    """Metric tables in the shared device layout."""
    gsize: int
    gcov: np.ndarray
    gcon: np.ndarray
    gdet: np.ndarray
    conn: np.ndarray

    @classmethod
    def empty(cls, gsize):
        return cls(gsize, np.zeros(50 * gsize), np.zeros(50 * gsize), np.zeros(5 * gsize), np.zeros(40 * gsize))

    def c(self):
        return HoGeom(_ptr(self.gcov), _ptr(self.gcon), _ptr(self.gdet), _ptr(self.conn))


def ref_geometry(variant, spin, startx, dx):
    dims, _ = ref_dims(variant)
    geo = Geometry.empty(int(dims[8]))
    sx = np.asarray(startx, float)
    dd = np.asarray(dx, float)
    nfail = ref(variant).ref_geometry(spin, _ptr(sx), _ptr(dd), _ptr(geo.gcov), _ptr(geo.gcon),
                                      _ptr(geo.gdet), _ptr(geo.conn))
    if nfail:
        raise RuntimeError(f"reference geometry reported {nfail} failures")
    return geo


def build_geometry(coords: str, spin: float, n1: int, n2: int, n3: int, startx, dx, ng: int = 3,
                   gsize: int = 0) -> "Geometry":
    """The oracle's own metric tables (hamr_oracle_geom.c), same call and
    layout as the product's hamr_gamma_wind_b200.api.build_geometry: lets a
    problem be set up with no product code loaded."""
    g1 = n1 + 2 * ng if n1 > 1 else 1
    g2 = n2 + 2 * ng if n2 > 1 else 1
    gs = gsize or pad64(g1 * g2)
    geo = Geometry.empty(gs)
    sx = np.ascontiguousarray(startx, float)
    dd = np.ascontiguousarray(dx, float)
    rc = lib().ho_build_geometry({"ks": 0, "cartesian": 1}[coords], spin, n1, n2, n3, ng, gs, _ptr(sx), _ptr(dd),
                                 _ptr(geo.gcov), _ptr(geo.gcon), _ptr(geo.gdet), _ptr(geo.conn))
    if rc:
        raise RuntimeError(f"ho_build_geometry: {rc}")
    return geo


def num_threads() -> int:
    """OpenMP threads the oracle's parallel loops use."""
    return int(lib().ho_num_threads())


@dataclass
class Setup:
    blk: Block
    geo: Geometry
    dx: tuple
    gam: float
    cour: float
    pole1: int
    pole2: int
    bc: tuple  # (bc1, bc2, bc3)
    ct_upwind: int = 1
    inversion: int = 0  # 0: Noble 2D, 1: Newman-Hamlin
    recon: int = 0      # 0: PPM, 1: MC-limited linear
    riemann: int = 0    # 0: HLL, 1: HLLC, 2: HLLD
    halo: int = 0       # sides filled by a neighbour block: bits 0, 1 lower/upper x1; 2, 3 lower/upper x2
    floors: int = 0     # 1: drift-frame floors after the inversion
    repair: int = 0     # failed zones: 1 reset to the floor state, 2 neighbour interpolation

    def grid(self):
        b = self.blk
        return HoGrid(b.n1, b.n2, b.n3, b.ng, b.ksize, b.gsize, self.dx[0], self.dx[1], self.dx[2],
                      self.gam, self.cour, self.pole1, self.pole2, self.bc[0], self.bc[1], self.bc[2],
                      self.inversion, self.ct_upwind, self.recon, self.riemann, self.halo,
                      self.floors, self.repair)


def _state(b: Block):
    a = b.arrays
    return HoState(*[_ptr(a[n]) for n in ("p", "ph", "ps", "psh", "U", "F1", "F2", "F3",
                                           "E_cent", "emf", "pflag", "failimage")])


def oracle_stage(s: Setup, full, Dt, dt, calc_dt=False):
    g = s.grid()
    m = s.geo.c()
    st = _state(s.blk)
    dtdir = np.full(4, 1e9)
    lib().ho_stage(ctypes.byref(g), ctypes.byref(m), ctypes.byref(st), int(full), Dt, dt,
                   int(bool(calc_dt)), _ptr(dtdir))
    return dtdir


def oracle_bound(s: Setup, pname="p", psname="ps"):
    g = s.grid()
    m = s.geo.c()
    lib().ho_bound(ctypes.byref(g), ctypes.byref(m), _ptr(s.blk.arrays[pname]), _ptr(s.blk.arrays[psname]))


def oracle_bound_dim(s: Setup, dim, pname="p", psname="ps"):
    """Ghost fill of one direction on the physical sides (halo sides skipped)."""
    g = s.grid()
    m = s.geo.c()
    lib().ho_bound_dim(ctypes.byref(g), ctypes.byref(m), _ptr(s.blk.arrays[pname]), _ptr(s.blk.arrays[psname]),
                       int(dim))


def set_mud(gcov10, gcon10, d):
    """Orthonormal face frame of direction d (oracle restatement of set_Mud):
    (Mud, Mud_inv) as 4x4 arrays."""
    M = np.zeros(16)
    Mi = np.zeros(16)
    lib().ho_set_mud(_ptr(np.ascontiguousarray(gcov10, float)), _ptr(np.ascontiguousarray(gcon10, float)), int(d),
                     _ptr(M), _ptr(Mi))
    return M.reshape(4, 4), Mi.reshape(4, 4)


_mud_cache: dict = {}


def ref_mud_tables(variant, s: Setup):
    """Frame tables of every (i, j) and face direction in the layout the
    reference's HLLC kernel reads (get_trans, GPU_hllc.h:878-900)."""
    key = (variant, id(s.geo))
    if key in _mud_cache:
        return _mud_cache[key]
    L = ref(variant)
    plane, nsolver = L.ref_mud_plane(), L.ref_nsolver()
    b, gs = s.blk, s.geo.gsize
    mud = np.zeros(16 * nsolver * plane)
    inv = np.zeros(16 * nsolver * plane)
    loc = {1: FACE1, 2: FACE2, 3: FACE3}
    for ii in range(b.g1):
        for jj in range(b.g2):
            gid = ii * b.g2 + jj
            for kk in (1, 2, 3):
                gcov = np.array([s.geo.gcov[(c * 5 + loc[kk]) * gs + gid] for c in range(10)])
                gcon = np.array([s.geo.gcon[(c * 5 + loc[kk]) * gs + gid] for c in range(10)])
                M, Mi = set_mud(gcov, gcon, kk)
                for a in range(4):
                    for c in range(4):
                        idx = (a * 4 + c) * nsolver * plane + kk * plane + gid
                        mud[idx] = M[a, c]
                        inv[idx] = Mi[a, c]
    _mud_cache[key] = (mud, inv)
    return mud, inv


def ref_stage(variant, s: Setup, full, Dt, dt, calc_dt=False):
    b = s.blk
    a = b.arrays
    dtdir = np.full(4, 1e9)
    if s.riemann >= 1:
        mud, inv = ref_mud_tables(variant, s)
        ref(variant).ref_set_mud(_ptr(mud), _ptr(inv))
    ref(variant).ref_stage(int(full), Dt, dt, s.cour, s.dx[0], s.dx[1], s.dx[2], s.pole1, s.pole2,
                           _ptr(a["p"]), _ptr(a["ph"]), _ptr(a["ps"]), _ptr(a["psh"]), _ptr(a["U"]),
                           _ptr(a["F1"]), _ptr(a["F2"]), _ptr(a["F3"]), _ptr(a["dq1"]), _ptr(a["dq2"]),
                           _ptr(a["E_cent"]), _ptr(a["emf"]), _ptr(a["pflag"]), _ptr(a["failimage"]),
                           _ptr(s.geo.gcov), _ptr(s.geo.gcon), _ptr(s.geo.gdet), _ptr(s.geo.conn),
                           _ptr(a["radius"]), int(bool(calc_dt)), _ptr(dtdir))
    return dtdir


def step(stage, bound, s: Setup, dt):
    """One RK2 midpoint step as GPU_step_ch runs it (step_ch.c:916-990):
    half sub-step, ghost fill of (ph, psh), full sub-step, ghost fill of (p, ps).
    Returns the CFL timestep 1/(1/dt1 + 1/dt2 + 1/dt3) of the full sub-step."""
    stage(s, 0, 0.5 * dt, dt, False)
    bound(s, "ph", "psh")
    dtd = stage(s, 1, dt, dt, True)
    bound(s, "p", "ps")
    return 1.0 / (1.0 / dtd[1] + 1.0 / dtd[2] + 1.0 / dtd[3])


def fixup_cell(gam, pf, gcov10, gcon10, gdet):
    """Floors of one zone (oracle restatement of fixup_cell): (flag, prims)."""
    pf = np.array(pf, float)
    rc = lib().ho_fixup_cell(gam, _ptr(pf), _ptr(np.ascontiguousarray(gcov10, float)),
                             _ptr(np.ascontiguousarray(gcon10, float)), gdet)
    return rc, pf


def oracle_fixup_utoprim(s: Setup, pname="p"):
    """Neighbour repair of the failed zones of one state (fixup_utoprim)."""
    g = s.grid()
    a = s.blk.arrays
    lib().ho_fixup_utoprim(ctypes.byref(g), _ptr(a[pname]), _ptr(a["pflag"]), _ptr(a["failimage"]))


def ref_fixup_utoprim(variant, s: Setup, pname="p"):
    """The reference's CPU fixup_utoprim (fixup.c:764) on one state."""
    a = s.blk.arrays
    ref(variant).ref_fixup_utoprim(_ptr(a[pname]), _ptr(a["pflag"]), _ptr(a["failimage"]), s.blk.ksize)


def ref_fixuputoprim(variant, s: Setup, pname="p"):
    """The reference's GPU fixuputoprim kernel (GPU_fixup.h:735), host build."""
    a = s.blk.arrays
    ref(variant).ref_fixuputoprim(_ptr(a[pname]), _ptr(a["radius"]), _ptr(s.geo.gcov), _ptr(s.geo.gcon),
                                  _ptr(s.geo.gdet), _ptr(a["pflag"]), _ptr(a["failimage"]))


def divb_max(s: Setup, psname="ps"):
    g = s.grid()
    m = s.geo.c()
    return lib().ho_divb_max(ctypes.byref(g), ctypes.byref(m), _ptr(s.blk.arrays[psname]))


def para(x):
    l = np.zeros(1)
    r = np.zeros(1)
    lib().ho_para(_ptr(np.ascontiguousarray(x, float)), _ptr(l), _ptr(r))
    return l[0], r[0]


def utoprim(name, gam, U, gcov10, gcon10, gdet, prim):
    U = np.array(U, float)
    prim = np.array(prim, float)
    rc = getattr(lib(), "ho_utoprim_" + name)(gam, _ptr(U), _ptr(np.asarray(gcov10, float)),
                                             _ptr(np.asarray(gcon10, float)), gdet, _ptr(prim))
    return rc, prim


def ref_utoprim(variant, name, U, gcov10, gcon10, gdet, prim):
    U = np.array(U, float)
    prim = np.array(prim, float)
    rc = getattr(ref(variant), "ref_utoprim_" + name)(_ptr(U), _ptr(np.asarray(gcov10, float)),
                                                     _ptr(np.asarray(gcon10, float)), gdet, _ptr(prim))
    return rc, prim


def ref_dump_available(variant: str) -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", f"libref_dump_{variant}.so"))


def ref_dump_files(variant, p, ps, ksize, geo, prm_d, prm_i, param_path, dump_path, rdump_path):
    """The reference's own writers (dump_params, dump_block,
    rdump_block_write; oracle/ref_dumpio.c) on one block of a compile-time
    variant: state (p, ps) and metric tables in the device layout; prm_d = (t,
    dt, DTd, DTl, startx1-3, dx1-3, tf, a, gam, cour, Rin, Rout, R0), prm_i =
    (nstep, dump_cnt, rdump_cnt, failed, lim, dump_cnt_reduced)."""
    L = ctypes.CDLL(os.path.join(HERE, "_ref", f"libref_dump_{variant}.so"))
    L.ref_dump_files.restype = _i
    d = np.ascontiguousarray(prm_d, dtype=np.float64)
    i = np.ascontiguousarray(prm_i, dtype=np.int32)
    rc = L.ref_dump_files(_ptr(np.ascontiguousarray(p)), _ptr(np.ascontiguousarray(ps)), ctypes.c_long(ksize),
                          _ptr(geo.gcov), _ptr(geo.gcon), _ptr(geo.gdet), ctypes.c_long(geo.gsize), _ptr(d), _ptr(i),
                          param_path.encode(), dump_path.encode(), rdump_path.encode())
    if rc:
        raise RuntimeError(f"ref_dump_files: {rc}")
