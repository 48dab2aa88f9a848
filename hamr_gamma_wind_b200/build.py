"""Builds the in-tree CUDA library for sm_100a.

Two shared objects come out of the same sources:
  libhamr_b200.so         production build (fused multiply-add contraction on)
  libhamr_b200_strict.so  --fmad=false: reproduces the reference's operation
                          order, used by the bit-level parity tests
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
SOURCES = [os.path.join(CSRC, "hamr_kernels.cu"), os.path.join(CSRC, "hamr_geometry.cpp")]
# every source and header the library is compiled from (the .cuh files are
# included into hamr_kernels.cu)
DEPS = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".cpp", ".h"))) + [
    os.path.abspath(__file__), os.path.join(os.path.dirname(HERE), "include", "hamr_b200.h")]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

TARGETS = {
    "libhamr_b200.so": [],
    "libhamr_b200_strict.so": ["--fmad=false"],
}


def _stale(out):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in DEPS)


def build(force=False, verbose=False):
    outs, jobs = [], []
    for name, extra in TARGETS.items():
        out = os.path.join(HERE, name)
        outs.append(out)
        if not force and not _stale(out):
            continue
        # -prec-div/-prec-sqrt=false: single-precision division and square
        # root use the approximate instructions (the mixed-precision step's
        # FP32 reconstruction, flux and EMF arithmetic); double precision is
        # unaffected
        cmd = [NVCC, *ARCH, "-lineinfo", "-O3", "-std=c++17", "--shared", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-ffp-contract=off", "-prec-div=false", "-prec-sqrt=false",
               "-Xptxas", "-v" if verbose else "-O3", *extra, *SOURCES, "-o", out]
        # the builds are independent: compile them side by side
        jobs.append((name, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
    failed = []
    for name, proc in jobs:
        so, se = proc.communicate()
        if proc.returncode != 0:
            sys.stderr.write(so + se)
            failed.append(name)
        elif verbose:
            sys.stderr.write(se)
    if failed:
        raise RuntimeError(f"nvcc failed building {', '.join(failed)}")
    return outs


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
