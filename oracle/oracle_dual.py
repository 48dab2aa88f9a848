"""Test infrastructure (oracle) -- never imported by the product.

ctypes binding of ``liboracle_dual.so``: the oracle restatement compiled with
every double a forward-mode dual number carrying NT tangents
(dual_prelude.hpp, oracle_dual.cpp). Its arrays hold, per entry, the value
followed by NT tangents. ``TangentRun`` advances a block and NT tangent
directions together, with the step sizes held fixed (as the CUDA adjoint
holds them), and accumulates the tangents of the accretion-rate objective
J = sum_n w_n Mdot_n, Mdot = -sum_j F1[RHO](ih, j) dx2 dx3 of the full
sub-step (calc_Mdot, restart.c:864-903). This is the FP64 tangent-linear
reference the adjoint's gradient is checked against: <dJ/dx, v> = dJ(x; v).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
NT = 8   # tangents per pass (HD_NT of the build)
_vp = ctypes.c_void_p
_d = ctypes.c_double
_i = ctypes.c_int


class Dual(ctypes.Structure):
    _fields_ = [("v", _d), ("d", _d * NT)]


def dual(v, tangents=None):
    x = Dual()
    x.v = float(v)
    for q in range(NT):
        x.d[q] = 0.0 if tangents is None else float(tangents[q])
    return x


class HoGridD(ctypes.Structure):
    _fields_ = [("n1", _i), ("n2", _i), ("n3", _i), ("ng", _i),
                ("ksize", ctypes.c_long), ("gsize", ctypes.c_long),
                ("dx1", Dual), ("dx2", Dual), ("dx3", Dual), ("gam", Dual), ("cour", Dual),
                ("pole1", _i), ("pole2", _i), ("bc1", _i), ("bc2", _i), ("bc3", _i),
                ("inversion", _i), ("ct_upwind", _i), ("recon", _i), ("riemann", _i), ("halo", _i),
                ("floors", _i), ("repair", _i)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle_dual.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle_dual.so missing: run `make -C oracle`")
        L = ctypes.CDLL(path)
        L.ho_stage.argtypes = [ctypes.POINTER(HoGridD), ctypes.POINTER(O.HoGeom), ctypes.POINTER(O.HoState),
                               _i, Dual, Dual, _i, _vp]
        L.ho_bound.argtypes = [ctypes.POINTER(HoGridD), ctypes.POINTER(O.HoGeom), _vp, _vp]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(_vp)


class TangentRun:
    """A plain-oracle setup (oracle.Setup) lifted to dual numbers. Tangent
    directions are seeded with ``seed`` before the first ghost fill; the
    adiabatic index may carry tangents too (``gam_tangents``)."""

    ARRAYS = (("p", 9), ("ph", 9), ("ps", 3), ("psh", 3), ("U", 9), ("F1", 9), ("F2", 9), ("F3", 9),
              ("E_cent", 4), ("emf", 4))

    def __init__(self, s: O.Setup, gam_tangents=None):
        self.s = s
        b = s.blk
        self.ks = b.ksize
        self.a = {}
        for name, planes in self.ARRAYS:
            x = np.zeros((planes * self.ks, 1 + NT))
            x[:, 0] = b.arrays[name][:planes * self.ks]
            self.a[name] = x
        self.pflag = np.zeros(self.ks, np.int32)
        self.failimage = np.zeros(5 * self.ks, np.int32)
        self.geo = {}
        for name in ("gcov", "gcon", "gdet", "conn"):
            src = getattr(s.geo, name)
            x = np.zeros((src.size, 1 + NT))
            x[:, 0] = src
            self.geo[name] = x
        g = s.grid()
        self.grid = HoGridD(g.n1, g.n2, g.n3, g.ng, g.ksize, g.gsize, dual(g.dx1), dual(g.dx2), dual(g.dx3),
                            dual(g.gam, gam_tangents), dual(g.cour), g.pole1, g.pole2, g.bc1, g.bc2, g.bc3,
                            g.inversion, g.ct_upwind, g.recon, g.riemann, g.halo, g.floors, g.repair)
        self.gm = O.HoGeom(*[_ptr(self.geo[n]) for n in ("gcov", "gcon", "gdet", "conn")])
        self.st = O.HoState(*[_ptr(self.a[n]) for n in ("p", "ph", "ps", "psh", "U", "F1", "F2", "F3",
                                                         "E_cent", "emf")], _ptr(self.pflag), _ptr(self.failimage))

    def seed(self, name, tangents):
        """tangents: array (NT, planes * ksize) added to the tangents of `name`."""
        self.a[name][:, 1:] += np.asarray(tangents).T

    def bound(self, pname="p", psname="ps"):
        lib().ho_bound(ctypes.byref(self.grid), ctypes.byref(self.gm), _ptr(self.a[pname]), _ptr(self.a[psname]))

    def stage(self, full, Dt, dt):
        dtdir = np.zeros((4, 1 + NT))
        lib().ho_stage(ctypes.byref(self.grid), ctypes.byref(self.gm), ctypes.byref(self.st), int(full),
                       dual(Dt), dual(dt), 0, _ptr(dtdir))

    def step(self, dt):
        self.stage(0, 0.5 * dt, dt)
        self.bound("ph", "psh")
        self.stage(1, dt, dt)
        self.bound("p", "ps")

    def mdot(self, ih):
        """(Mdot, its NT tangents) of the last full sub-step through x1 face column ih."""
        b = self.s.blk
        g3 = b.g3
        cols = [(ih * b.g2 + (b.ng + j)) * g3 for j in range(b.n2)]
        f = self.a["F1"][[RHO_PLANE * self.ks + c for c in cols]]
        w = -self.s.dx[1] * self.s.dx[2]
        return w * f[:, 0].sum(), w * f[:, 1:].sum(axis=0)

    def objective(self, ih, dts):
        """Ghost fill, then the steps dts with J = sum_n dts[n] Mdot_n.
        Returns (J, dJ along each of the NT seeded directions)."""
        self.bound()
        J, dJ = 0.0, np.zeros(NT)
        for dt in dts:
            self.step(dt)
            m, dm = self.mdot(ih)
            J += dt * m
            dJ += dt * dm
        return J, dJ


RHO_PLANE = 0
