"""C ABI checks that need no GPU: every symbol include/hamr_b200.h declares is
exported, argument validation answers before any device work, and the host
geometry builder reproduces the reference's metric tables bit for bit."""
import ctypes
import os
import re

import numpy as np
import pytest

from hamr_gamma_wind_b200 import _lib
from hamr_gamma_wind_b200.api import build_geometry, ks_grid
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "hamr_b200.h")).read()
    return sorted(set(re.findall(r"^(?:int|long|const char \*)\s*(hamr_\w+)\(", text, re.M)))


@pytest.mark.parametrize("strict", [False, True])
def test_library_exports_every_declared_symbol(strict):
    L = _lib.load(strict)
    syms = declared_symbols()
    assert syms, "no declarations parsed"
    for s in syms:
        assert hasattr(L, s), s
    assert sorted(_lib.SYMBOLS) == syms


def test_create_rejects_bad_parameters_without_device_work():
    L = _lib.load()
    ctx = ctypes.c_void_p()
    prm = _lib.HamrParams(16, 8, 8, 2, 0, 0, 0.1, 0.1, 0.1, 13 / 9, 0.8, 1, 1, 1, 2, 0, 1, 0, None)
    assert L.hamr_ctx_create(ctypes.byref(prm), ctypes.byref(ctx)) == -1      # ng 2 only with MC
    prm.recon = 7
    prm.ng = 3
    assert L.hamr_ctx_create(ctypes.byref(prm), ctypes.byref(ctx)) == -1      # no such reconstruction
    prm.recon = 0
    prm.riemann = 3
    assert L.hamr_ctx_create(ctypes.byref(prm), ctypes.byref(ctx)) == -1      # no such Riemann solver
    prm.riemann = 4
    assert L.hamr_ctx_create(ctypes.byref(prm), ctypes.byref(ctx)) == -1      # no such Riemann solver
    prm.riemann = 0
    prm.halo = 4
    assert L.hamr_ctx_create(ctypes.byref(prm), ctypes.byref(ctx)) == -1      # halo sides along x1 only
    prm.halo = 1
    bc1, prm.bc1 = prm.bc1, 0
    assert L.hamr_ctx_create(ctypes.byref(prm), ctypes.byref(ctx)) == -1      # a periodic x1 has no neighbours
    prm.bc1 = bc1
    prm.repair = 2
    assert L.hamr_ctx_create(ctypes.byref(prm), ctypes.byref(ctx)) == -1      # neighbour repair spans the domain
    prm.repair = 0
    prm.halo = 0
    prm.floors = 2
    assert L.hamr_ctx_create(ctypes.byref(prm), ctypes.byref(ctx)) == -1      # floors are on or off
    prm.floors = 0
    prm.repair = 3
    assert L.hamr_ctx_create(ctypes.byref(prm), ctypes.byref(ctx)) == -1      # no such repair
    prm.repair = 0
    prm.ng = 3
    prm.gam = 1.0
    assert L.hamr_ctx_create(ctypes.byref(prm), ctypes.byref(ctx)) == -1      # gamma <= 1
    prm.gam = 13 / 9
    prm.n3 = 7
    assert L.hamr_ctx_create(ctypes.byref(prm), ctypes.byref(ctx)) == -1      # transmissive pole needs even n3
    prm.n3 = 8
    prm.inversion = 2
    assert L.hamr_ctx_create(ctypes.byref(prm), ctypes.byref(ctx)) == -1      # no such primary inversion
    prm.inversion = 0
    prm.precision = 5
    assert L.hamr_ctx_create(ctypes.byref(prm), ctypes.byref(ctx)) == -1      # no such precision
    assert L.hamr_ctx_create(None, ctypes.byref(ctx)) == -1
    assert L.hamr_stage(None, 0, 0.1, 0.1) == -1
    assert L.hamr_step(None, 0.1, None) == -1
    out = ctypes.c_void_p()
    assert L.hamr_batch_create(None, 0, None, ctypes.byref(out)) == -1
    assert L.hamr_batch_step(None, None, None) == -1
    assert L.hamr_batch_advance(None, 1, 1, None) == -1


def _compare_tables(a, b):
    for name in ("gcov", "gcon", "gdet", "conn"):
        x, y = getattr(a, name), getattr(b, name)
        assert x.shape == y.shape, name
        d = np.abs(x - y)
        assert np.array_equal(x, y), f"{name}: {np.count_nonzero(d)} differ, max {d.max():.3e}"


@pytest.mark.parametrize("variant", ["t3", "t2"])
def test_ks_geometry_matches_reference_bitwise(variant):
    if not O.ref_available(variant):
        pytest.skip("reference host build not present")
    dims, _ = O.ref_dims(variant)
    n1, n2, n3 = (int(x) for x in dims[:3])
    spin = 0.9375
    startx, dx = ks_grid(n1, n2, n3, spin, 40.0)
    ours = build_geometry("ks", spin, n1, n2, n3, startx, dx)
    ref = O.ref_geometry(variant, spin, startx, dx)
    _compare_tables(ours, ref)


def test_cartesian_geometry_matches_reference_bitwise():
    if not O.ref_available("ot"):
        pytest.skip("reference host build not present")
    ours = build_geometry("cartesian", 0.0, 32, 32, 1, [0, 0, 0, 0], [0, 1 / 32, 1 / 32, 1.0])
    ref = O.ref_geometry("ot", 0.0, [0, 0, 0, 0], [0, 1 / 32, 1 / 32, 1.0])
    _compare_tables(ours, ref)


def test_bl_coord_matches_reference():
    if not O.ref_available("t3"):
        pytest.skip("reference host build not present")
    L = _lib.load()
    R = O.ref("t3")
    rng = np.random.default_rng(0)
    for _ in range(200):
        X = np.array([0.0, rng.uniform(-0.5, 5), rng.uniform(-1.5, 1.5), rng.uniform(0, 6.3)])
        a = np.zeros(3)
        b = np.zeros(3)
        L.hamr_bl_coord(0, 0.9375, X.ctypes.data_as(ctypes.c_void_p), a.ctypes.data_as(ctypes.c_void_p))
        R.ref_bl_coord(X.ctypes.data_as(ctypes.c_void_p), b.ctypes.data_as(ctypes.c_void_p))
        assert np.array_equal(a, b), (X, a, b)


@pytest.mark.parametrize("variant", ["t3", "t2", "ot"])
def test_oracle_geometry_matches_reference_bitwise(variant):
    """The oracle's own metric tables (used to set up the CPU arm with no
    library code) are the reference's tables bit for bit."""
    if not O.ref_available(variant):
        pytest.skip("reference host build not present")
    dims, _ = O.ref_dims(variant)
    n1, n2, n3 = (int(x) for x in dims[:3])
    if variant == "ot":
        startx, dx, coords, spin = [0, 0, 0, 0], [0, 1 / n1, 1 / n2, 1.0], "cartesian", 0.0
    else:
        spin = 0.9375
        startx, dx = ks_grid(n1, n2, n3, spin, 40.0)
        coords = "ks"
    _compare_tables(O.build_geometry(coords, spin, n1, n2, n3, startx, dx), O.ref_geometry(variant, spin, startx, dx))


@pytest.mark.parametrize("n", [(24, 16, 8), (96, 48, 32), (64, 64, 1)])
def test_oracle_geometry_matches_library_bitwise(n):
    n1, n2, n3 = n
    spin = 0.9375
    startx, dx = ks_grid(n1, n2, n3, spin, 1000.0)
    _compare_tables(O.build_geometry("ks", spin, n1, n2, n3, startx, dx),
                    build_geometry("ks", spin, n1, n2, n3, startx, dx))
