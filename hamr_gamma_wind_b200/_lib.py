"""ctypes binding of the in-tree CUDA library (include/hamr_b200.h).

The library is required: there is no CPU fallback for the step. Importing a
binding whose shared object is missing raises immediately.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
NPR = 9

_vp = ctypes.c_void_p
_d = ctypes.c_double
_i = ctypes.c_int
_l = ctypes.c_long


class HamrParams(ctypes.Structure):
    _fields_ = [("n1", _i), ("n2", _i), ("n3", _i), ("ng", _i), ("ksize", _l), ("gsize", _l),
                ("dx1", _d), ("dx2", _d), ("dx3", _d), ("gam", _d), ("cour", _d),
                ("pole1", _i), ("pole2", _i), ("bc1", _i), ("bc2", _i), ("bc3", _i),
                ("ct_upwind", _i), ("precision", _i), ("stream", _vp), ("inversion", _i), ("recon", _i),
                ("riemann", _i), ("halo", _i), ("floors", _i), ("repair", _i)]


ERRORS = {0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "out of device memory",
          -4: "call out of order", -5: "non-finite or non-positive CFL step"}


class HamrError(RuntimeError):
    pass


_libs: dict = {}


def lib_path(strict: bool = False) -> str:
    return os.path.join(HERE, "libhamr_b200_strict.so" if strict else "libhamr_b200.so")


def load(strict: bool = False):
    """The CUDA library; ``strict`` selects the build without FMA contraction."""
    key = bool(strict)
    if key in _libs:
        return _libs[key]
    path = lib_path(strict)
    if not os.path.exists(path):
        raise HamrError(f"{os.path.basename(path)} is not built (run __graft_entry__.build())")
    L = ctypes.CDLL(path)
    P = ctypes.POINTER
    L.hamr_ctx_create.argtypes = [P(HamrParams), P(_vp)]
    L.hamr_ctx_destroy.argtypes = [_vp]
    L.hamr_last_error.argtypes = [_vp]
    L.hamr_last_error.restype = ctypes.c_char_p
    L.hamr_strides.argtypes = [_vp, P(_l), P(_l)]
    L.hamr_set_geometry.argtypes = [_vp, _vp, _vp, _vp, _vp]
    L.hamr_upload.argtypes = [_vp, _vp, _vp]
    L.hamr_download.argtypes = [_vp, _vp, _vp]
    L.hamr_download_flags.argtypes = [_vp, _vp, _vp]
    L.hamr_bound.argtypes = [_vp]
    L.hamr_stage.argtypes = [_vp, _i, _d, _d]
    L.hamr_step.argtypes = [_vp, _d, _vp]
    L.hamr_advance.argtypes = [_vp, _i, _i, P(_d)]
    L.hamr_device_state.argtypes = [_vp, _vp, _vp, _vp, _vp]
    L.hamr_profile_step.argtypes = [_vp, _d, _i, _vp, _i]
    L.hamr_divb_max.argtypes = [_vp, P(_d)]
    L.hamr_build_geometry.argtypes = [_i, _d, _i, _i, _i, _i, _l, _vp, _vp, _vp, _vp, _vp, _vp]
    L.hamr_bl_coord.argtypes = [_i, _d, _vp, _vp]
    L.hamr_step_noalloc.argtypes = [P(HamrParams), _vp, _vp, _vp, _vp, _vp, _vp, _d, P(_d)]
    L.hamr_batch_create.argtypes = [_vp, _i, _vp, P(_vp)]
    L.hamr_batch_destroy.argtypes = [_vp]
    L.hamr_batch_last_error.argtypes = [_vp]
    L.hamr_batch_last_error.restype = ctypes.c_char_p
    L.hamr_batch_step.argtypes = [_vp, _vp, _vp]
    L.hamr_batch_advance.argtypes = [_vp, _i, _i, _vp]
    L.hamr_batch_autotune.argtypes = [_vp, _vp, _i]
    L.hamr_batch_set_persistent.argtypes = [_vp, _i]
    L.hamr_batch_tuning.argtypes = [_vp, _vp, _vp, _vp, _vp, _i]
    L.hamr_adjoint_create.argtypes = [_vp, _i, P(_vp)]
    L.hamr_adjoint_destroy.argtypes = [_vp]
    L.hamr_adjoint_last_error.argtypes = [_vp]
    L.hamr_adjoint_last_error.restype = ctypes.c_char_p
    L.hamr_adjoint_cotangent.argtypes = [_vp, _vp, _vp, _vp]
    L.hamr_adjoint_zero.argtypes = [_vp]
    L.hamr_step_backward.argtypes = [_vp, _d, _d]
    L.hamr_mdot_forward.argtypes = [_vp, _i, _vp, P(_d)]
    L.hamr_adjoint_run.argtypes = [_vp, _i, _vp, _i, P(_d), _vp, _vp, P(_d)]
    L.hamr_bound_dim.argtypes = [_vp, _i, _i]
    L.hamr_halo_count.argtypes = [_vp]
    L.hamr_halo_count.restype = _l
    L.hamr_halo_pack.argtypes = [_vp, _i, _i, _vp]
    L.hamr_halo_unpack.argtypes = [_vp, _i, _i, _vp]
    L.hamr_cfl_dirs.argtypes = [_vp, _vp]
    _libs[key] = L
    return L


# exported symbols the header declares (checked by the CPU test suite)
SYMBOLS = ["hamr_ctx_create", "hamr_ctx_destroy", "hamr_last_error", "hamr_strides",
           "hamr_set_geometry", "hamr_upload", "hamr_download", "hamr_download_flags",
           "hamr_bound", "hamr_stage", "hamr_step", "hamr_advance", "hamr_device_state", "hamr_profile_step",
           "hamr_divb_max", "hamr_build_geometry", "hamr_bl_coord", "hamr_step_noalloc",
           "hamr_batch_create", "hamr_batch_destroy", "hamr_batch_last_error", "hamr_batch_step",
           "hamr_batch_advance", "hamr_batch_autotune", "hamr_batch_set_persistent", "hamr_batch_tuning",
           "hamr_adjoint_create", "hamr_adjoint_destroy", "hamr_adjoint_last_error", "hamr_adjoint_cotangent",
           "hamr_adjoint_zero", "hamr_step_backward", "hamr_mdot_forward", "hamr_adjoint_run",
           "hamr_bound_dim", "hamr_halo_count", "hamr_halo_pack", "hamr_halo_unpack", "hamr_cfl_dirs"]
NOALLOC_MAX_CELLS = 32768

BATCH_PHASES = ["flux3", "flux2", "flux1", "fix_flux", "emf_centre", "emf_edge", "pole_average",
                "face_update", "update", "invert", "bound_x1", "bound_x3", "bound_x2"]

PROF_SLOTS = ["flux3", "flux2", "flux1", "fix_flux", "emf_centre", "emf_edge", "pole_average",
              "face_update", "update", "invert", "bound"]
