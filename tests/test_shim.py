"""The C shim of the drop-in boundary (hamr_gamma_wind_b200/shim) is compiled
against the reference's own decs.h / config.h by oracle/Makefile (target
shim-check, run by __graft_entry__.build() where the reference sources are
present). Here: the object exists and binds what it should -- the library's
C ABI on one side, the reference's host state and globals on the other."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OBJ = os.path.join(ROOT, "oracle", "_ref", "hamr_step_ch_shim.o")


@pytest.mark.skipif(not os.path.exists(OBJ), reason="reference sources not present (shim not compiled)")
def test_shim_binds_abi_and_reference_state():
    nm = shutil.which("nm")
    assert nm
    out = subprocess.run([nm, "-u", OBJ], capture_output=True, text=True, check=True).stdout
    undef = {line.split()[-1] for line in out.splitlines() if line.strip()}
    for sym in ("hamr_ctx_create", "hamr_set_geometry", "hamr_upload", "hamr_bound", "hamr_advance",
                "hamr_download", "hamr_strides", "hamr_ctx_destroy"):
        assert sym in undef, sym
    # the reference's host state and globals (decs.h)
    for sym in ("p", "ps", "dx", "nl", "block", "gcov_GPU", "gcon_GPU", "gdet_GPU", "conn_GPU", "dt", "t",
                "nstep", "n_active", "n_ord", "index_3D", "N1_GPU_offset"):
        assert sym in undef, sym
    out = subprocess.run([nm, "-g", "--defined-only", OBJ], capture_output=True, text=True, check=True).stdout
    defined = {line.split()[-1] for line in out.splitlines() if line.strip()}
    assert {"hamr_shim_attach", "hamr_shim_step_ch", "hamr_shim_read", "hamr_shim_detach"} <= defined
