"""Host-side mirror of the reference's per-block step interface.

The reference drives one block through globals: ``GPU_write`` /
``GPU_write_metric`` upload state and metric (GPU_main.cu:309,139),
``advance_GPU`` runs one RK2 sub-step (step_ch.c:997), ``GPU_step_ch`` a time
step with its dt bookkeeping (step_ch.c:916), ``GPU_read`` copies back
(GPU_main.cu:2646) and ``divb_calc`` checks the field (diag.c:153). ``Block``
offers the same operations on an explicit context of the C ABI.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib

BC = {"periodic": 0, "outflow": 1, "pole_trans": 2, "pole_refl": 3}
PRECISION = {"fp64": 0, "mixed": 1}
INVERSION = {"2d": 0, "nm": 1}
RECON = {"ppm": 0, "mc": 1}
RIEMANN = {"hll": 0, "hllc": 1, "hlld": 2}
REPAIR = {"none": 0, "reset": 1, "neighbours": 2}
RHO, UU, U1, U2, U3, B1, B2, B3, KTOT = range(9)
FACE1, FACE2, CORN, CENT, FACE3 = range(5)
NPR = _lib.NPR


def pad64(n: int) -> int:
    """Plane stride rule of the reference device buffers (GPU_program1.cu:92)."""
    return n + (64 - n % 64)


class Geometry:
    """Metric tables in the device layout (see include/hamr_b200.h)."""

    def __init__(self, gsize: int):
        self.gsize = gsize
        self.gcov = np.zeros(50 * gsize)
        self.gcon = np.zeros(50 * gsize)
        self.gdet = np.zeros(5 * gsize)
        self.conn = np.zeros(40 * gsize)

    def plane(self, name, comp, loc=None):
        a = getattr(self, name)
        k = comp if loc is None else comp * 5 + loc
        return a[k * self.gsize:(k + 1) * self.gsize]


def build_geometry(coords: str, spin: float, n1: int, n2: int, n3: int, startx, dx, ng: int = 3,
                   gsize: int = 0) -> Geometry:
    """Host metric tables: ``coords`` is "ks" (Kerr-Schild in the reference's
    log-r / uniform-theta code coordinates) or "cartesian" (Minkowski)."""
    L = _lib.load()
    g1 = n1 + 2 * ng if n1 > 1 else 1
    g2 = n2 + 2 * ng if n2 > 1 else 1
    gs = gsize or pad64(g1 * g2)
    geo = Geometry(gs)
    sx = np.ascontiguousarray(startx, float)
    dd = np.ascontiguousarray(dx, float)
    p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    rc = L.hamr_build_geometry({"ks": 0, "cartesian": 1}[coords], spin, n1, n2, n3, ng, gs, p(sx), p(dd),
                               p(geo.gcov), p(geo.gcon), p(geo.gdet), p(geo.conn))
    if rc:
        raise _lib.HamrError(f"hamr_build_geometry: {_lib.ERRORS.get(rc, rc)}")
    return geo


def ks_grid(n1, n2, n3, spin, rout):
    """startx/dx of the reference's torus grid: X1 = log r from 0.9 r_H to rout,
    x2 over the full theta range (less one zone either side with transmissive
    poles), x3 = phi over 2 pi (set_gridparam / set_points, coord.c:327-461)."""
    rin = 0.9 * (1.0 + np.sqrt(1.0 - spin * spin))
    frac = 1.0 - 2.0 / n2 if n3 > 1 else 1.0
    startx = [0.0, np.log(rin), -1.0 + (1.0 - frac), 0.0]
    dx = [0.0, (np.log(rout) - np.log(rin)) / n1, 2.0 * frac / n2, 2.0 * np.pi / n3]
    return startx, dx


class Block:
    """One uniform block on the current CUDA device."""

    def __init__(self, n1, n2, n3, dx, gam, cour=0.8, bc=("outflow", "pole_trans", "periodic"),
                 poles=(1, 1), ct_upwind=True, precision="fp64", strict=False, ng=3, stream=None,
                 inversion="2d", recon="ppm", riemann="hll", halo=0, floors=False, repair="none"):
        """floors: the drift-frame floors after the inversion (off in the
        reference's shipped step); repair: what happens to zones whose
        inversion failed -- "none" (the reference's step), "reset" (floor
        state, zero velocity: fixuputoprim) or "neighbours" (average of good
        neighbours: fixup_utoprim)."""
        self.L = _lib.load(strict)
        self.n1, self.n2, self.n3, self.ng = n1, n2, n3, ng
        self.g1 = n1 + 2 * ng
        self.g2 = n2 + 2 * ng
        self.g3 = n3 + 2 * ng if n3 > 1 else 1
        prm = _lib.HamrParams(n1, n2, n3, ng, 0, 0, float(dx[0]), float(dx[1]), float(dx[2]), float(gam),
                              float(cour), int(poles[0]), int(poles[1]), BC[bc[0]], BC[bc[1]], BC[bc[2]],
                              int(bool(ct_upwind)), PRECISION[precision], stream, INVERSION[inversion],
                              RECON[recon], RIEMANN[riemann], int(halo), int(bool(floors)), REPAIR[repair])
        ctx = ctypes.c_void_p()
        rc = self.L.hamr_ctx_create(ctypes.byref(prm), ctypes.byref(ctx))
        if rc:
            raise _lib.HamrError(f"hamr_ctx_create: {_lib.ERRORS.get(rc, rc)}")
        self.ctx = ctx
        ks, gs = ctypes.c_long(), ctypes.c_long()
        self.L.hamr_strides(ctx, ctypes.byref(ks), ctypes.byref(gs))
        self.ksize, self.gsize = ks.value, gs.value

    # -- lifecycle ---------------------------------------------------------
    def close(self):
        if getattr(self, "ctx", None):
            self.L.hamr_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc:
            msg = self.L.hamr_last_error(self.ctx).decode()
            raise _lib.HamrError(f"{what}: {_lib.ERRORS.get(rc, rc)} {msg}")

    # -- host arrays in the device layout -------------------------------------
    def empty_state(self):
        return np.zeros(NPR * self.ksize), np.zeros(3 * self.ksize)

    def view(self, a, planes=None):
        n = self.g1 * self.g2 * self.g3
        k = a.size // self.ksize if planes is None else planes
        return a.reshape(k, self.ksize)[:, :n].reshape(k, self.g1, self.g2, self.g3)

    def active(self, a, planes=None):
        v = self.view(a, planes)
        g = self.ng
        g3 = g if self.n3 > 1 else 0
        return v[:, g:g + self.n1, g:g + self.n2, g3:g3 + self.n3]

    # -- the reference's operations ----------------------------------------
    def set_geometry(self, geo: Geometry):
        """GPU_write_metric (GPU_main.cu:139)."""
        if geo.gsize != self.gsize:
            raise ValueError("geometry plane stride does not match the block")
        p = lambda a: np.ascontiguousarray(a).ctypes.data_as(ctypes.c_void_p)
        self._check(self.L.hamr_set_geometry(self.ctx, p(geo.gcov), p(geo.gcon), p(geo.gdet), p(geo.conn)),
                    "hamr_set_geometry")

    def upload(self, p, ps):
        """GPU_write (GPU_main.cu:309)."""
        p = np.ascontiguousarray(p, float)
        ps = np.ascontiguousarray(ps, float)
        if p.size != NPR * self.ksize or ps.size != 3 * self.ksize:
            raise ValueError("state arrays do not match the block layout")
        self._check(self.L.hamr_upload(self.ctx, p.ctypes.data_as(ctypes.c_void_p),
                                       ps.ctypes.data_as(ctypes.c_void_p)), "hamr_upload")

    def download(self):
        """GPU_read (GPU_main.cu:2646)."""
        p, ps = self.empty_state()
        self._check(self.L.hamr_download(self.ctx, p.ctypes.data_as(ctypes.c_void_p),
                                         ps.ctypes.data_as(ctypes.c_void_p)), "hamr_download")
        return p, ps

    def download_flags(self):
        pflag = np.zeros(self.ksize, np.int32)
        fail = np.zeros(5 * self.ksize, np.int32)
        self._check(self.L.hamr_download_flags(self.ctx, pflag.ctypes.data_as(ctypes.c_void_p),
                                               fail.ctypes.data_as(ctypes.c_void_p)), "hamr_download_flags")
        return pflag, fail

    def bound(self):
        """GPU_boundprim (GPU_main.cu:2113)."""
        self._check(self.L.hamr_bound(self.ctx), "hamr_bound")

    def advance_stage(self, full: int, Dt: float, dt: float):
        """advance_GPU for one block (step_ch.c:997) plus the ghost fill."""
        self._check(self.L.hamr_stage(self.ctx, int(full), float(Dt), float(dt)), "hamr_stage")

    def step(self, dt: float) -> float:
        """One RK2 step; returns the CFL step of its full sub-step."""
        out = ctypes.c_double()
        self._check(self.L.hamr_step(self.ctx, float(dt), ctypes.byref(out)), "hamr_step")
        return out.value

    def step_ch(self, nsteps: int, dt: float, interval: int = 16) -> float:
        """GPU_step_ch-style stepping (step_ch.c:916-990): nsteps steps whose
        size is refreshed from the CFL limit (growth capped at 1.3x) every
        `interval` steps, all on the device from one captured graph."""
        d = ctypes.c_double(dt)
        self._check(self.L.hamr_advance(self.ctx, int(nsteps), int(interval), ctypes.byref(d)), "hamr_advance")
        return d.value

    def divb_max(self) -> float:
        """max |div B| over active zones (divb_calc, diag.c:153)."""
        out = ctypes.c_double()
        self._check(self.L.hamr_divb_max(self.ctx, ctypes.byref(out)), "hamr_divb_max")
        return out.value

    def device_pointers(self):
        ptrs = [ctypes.c_void_p() for _ in range(4)]
        self._check(self.L.hamr_device_state(self.ctx, *[ctypes.byref(x) for x in ptrs]), "hamr_device_state")
        return [x.value for x in ptrs]

    # -- a slab of a domain decomposed along x1 (halo != 0) ---------------------
    def bound_dim(self, full: int, dim: int):
        """Ghost fill of one direction on the physical sides (hamr_bound_dim)."""
        self._check(self.L.hamr_bound_dim(self.ctx, int(full), int(dim)), "hamr_bound_dim")

    def halo_count(self) -> int:
        return int(self.L.hamr_halo_count(self.ctx))

    def halo_pack(self, full: int, side: int, dev_ptr: int):
        """Active layers next to side `side` (0, 1: lower and upper x1; 2, 3:
        lower and upper x2) into a device buffer."""
        self._check(self.L.hamr_halo_pack(self.ctx, int(full), int(side), ctypes.c_void_p(dev_ptr)),
                    "hamr_halo_pack")

    def halo_unpack(self, full: int, side: int, dev_ptr: int):
        """A device buffer into the ghost layers beyond side `side` (0-3)."""
        self._check(self.L.hamr_halo_unpack(self.ctx, int(full), int(side), ctypes.c_void_p(dev_ptr)),
                    "hamr_halo_unpack")

    def cfl_dirs(self):
        """Per-direction CFL minima of the last full sub-step (hamr_cfl_dirs)."""
        out = np.zeros(3)
        self._check(self.L.hamr_cfl_dirs(self.ctx, out.ctypes.data_as(ctypes.c_void_p)), "hamr_cfl_dirs")
        return out


class Batch:
    """An ensemble of Blocks advanced together (hamr_batch_*): one launch per
    sub-step phase for all members, per-member step sizes, an optional
    autotuned launch shape per phase. Members stay owned by the caller and
    must outlive the batch."""

    def __init__(self, blocks, stream=None):
        if not blocks:
            raise ValueError("empty batch")
        self.blocks = list(blocks)
        self.L = self.blocks[0].L
        arr = (ctypes.c_void_p * len(self.blocks))(*[b.ctx.value for b in self.blocks])
        self._arr = arr
        h = ctypes.c_void_p()
        rc = self.L.hamr_batch_create(arr, len(self.blocks), stream, ctypes.byref(h))
        if rc:
            raise _lib.HamrError(f"hamr_batch_create: {_lib.ERRORS.get(rc, rc)}")
        self.h = h

    @property
    def n(self):
        return len(self.blocks)

    def close(self):
        if getattr(self, "h", None):
            self.L.hamr_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc:
            msg = self.L.hamr_batch_last_error(self.h).decode()
            raise _lib.HamrError(f"{what}: {_lib.ERRORS.get(rc, rc)} {msg}")

    def _dts(self, dt):
        return np.ascontiguousarray(np.broadcast_to(np.asarray(dt, float), (self.n,)), dtype=float)

    def step(self, dt):
        """One RK2 step of every member (dt: scalar or one per member);
        returns each member's CFL step."""
        d = self._dts(dt)
        out = np.zeros(self.n)
        self._check(self.L.hamr_batch_step(self.h, d.ctypes.data_as(ctypes.c_void_p),
                                           out.ctypes.data_as(ctypes.c_void_p)), "hamr_batch_step")
        return out

    def advance(self, nsteps, dt, interval=16):
        """nsteps steps with per-member step-size refresh from one captured
        graph; returns each member's step size afterwards."""
        d = self._dts(dt).copy()
        self._check(self.L.hamr_batch_advance(self.h, int(nsteps), int(interval),
                                              d.ctypes.data_as(ctypes.c_void_p)), "hamr_batch_advance")
        return d

    def set_persistent(self, on=True):
        """One persistent cooperative launch per sub-step (True) or one
        launch per phase (False, the default)."""
        self._check(self.L.hamr_batch_set_persistent(self.h, int(bool(on))), "hamr_batch_set_persistent")

    def autotune(self, dt, reps=3):
        d = self._dts(dt)
        self._check(self.L.hamr_batch_autotune(self.h, d.ctypes.data_as(ctypes.c_void_p), int(reps)),
                    "hamr_batch_autotune")
        return self.tuning()

    def tuning(self):
        n = len(_lib.BATCH_PHASES)
        tile, grid, order = (np.zeros(n, np.int32) for _ in range(3))
        ms = np.zeros(n, np.float32)
        p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        self._check(self.L.hamr_batch_tuning(self.h, p(tile), p(grid), p(order), p(ms), n), "hamr_batch_tuning")
        # tile 0: the conserved update's row kernel with bulk-copy staging
        return {ph: dict(tile=int(tile[k]), grid=int(grid[k]), order=("largest-first" if order[k] else "given"),
                         ms=float(ms[k])) for k, ph in enumerate(_lib.BATCH_PHASES)}


class Adjoint:
    """Reverse mode of the FP64 step of a 2-D torus Block (hamr_adjoint_*):
    the accretion-rate objective J = sum_n dt_n Mdot_n through x1 face column
    `mdot_face` and its gradient w.r.t. the initial state and gamma."""

    def __init__(self, block, mdot_face):
        self.block = block
        self.L = block.L
        h = ctypes.c_void_p()
        rc = self.L.hamr_adjoint_create(block.ctx, int(mdot_face), ctypes.byref(h))
        if rc:
            raise _lib.HamrError(f"hamr_adjoint_create: {_lib.ERRORS.get(rc, rc)}")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.hamr_adjoint_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc:
            msg = self.L.hamr_adjoint_last_error(self.h).decode()
            raise _lib.HamrError(f"{what}: {_lib.ERRORS.get(rc, rc)} {msg}")

    def forward(self, dts):
        """Ghost fill and len(dts) steps (the block's state advances); returns J."""
        d = np.ascontiguousarray(dts, dtype=float)
        J = ctypes.c_double()
        self._check(self.L.hamr_mdot_forward(self.h, len(d), d.ctypes.data_as(ctypes.c_void_p), ctypes.byref(J)),
                    "hamr_mdot_forward")
        return J.value

    def gradient(self, dts, every=20):
        """(J, dJ/dp (9 planes), dJ/dps (3 planes), dJ/dgamma); the block's
        state is left at its initial value."""
        d = np.ascontiguousarray(dts, dtype=float)
        gp = np.zeros(9 * self.block.ksize)
        gs = np.zeros(3 * self.block.ksize)
        J, gg = ctypes.c_double(), ctypes.c_double()
        p = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        self._check(self.L.hamr_adjoint_run(self.h, len(d), p(d), int(every), ctypes.byref(J), p(gp), p(gs),
                                            ctypes.byref(gg)), "hamr_adjoint_run")
        return J.value, gp, gs, gg.value

    def step_backward(self, dt, mdot_weight=0.0):
        self._check(self.L.hamr_step_backward(self.h, float(dt), float(mdot_weight)), "hamr_step_backward")

    def cotangent_pointers(self):
        ptrs = [ctypes.c_void_p() for _ in range(3)]
        self._check(self.L.hamr_adjoint_cotangent(self.h, *[ctypes.byref(x) for x in ptrs]), "hamr_adjoint_cotangent")
        return [x.value for x in ptrs]

    def zero(self):
        self._check(self.L.hamr_adjoint_zero(self.h), "hamr_adjoint_zero")
