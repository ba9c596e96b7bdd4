"""Build recipe of the native library and the drop-in executable.

    python -m kirch_datuming_b200.build [--force]

produces, in-tree,
    kirch_datuming_b200/libkcig.so          the C-ABI library (include/kcig.h)
    kirch_datuming_b200/bin/kirchmig2d_cig  the drop-in migration / modelling tool
    kirch_datuming_b200/bin/eikods2d        the drop-in table generator
    kirch_datuming_b200/bin/kirchmig2d      the drop-in plain Kirchhoff migration
    kirch_datuming_b200/bin/layercom_cig    the drop-in ADCIG stitching of depth windows
    kirch_datuming_b200/bin/greensol_auto   the drop-in datum-depth slice of a traveltime table
    kirch_datuming_b200/bin/kirchdat2d_freq the drop-in frequency-domain datuming between depth levels
compiled for sm_100a only (nvcc cross-compiles; no GPU needed to build).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libkcig.so")
CLI = os.path.join(PKG, "bin", "kirchmig2d_cig")
EIK_CLI = os.path.join(PKG, "bin", "eikods2d")
K2D_CLI = os.path.join(PKG, "bin", "kirchmig2d")
STITCH_CLI = os.path.join(PKG, "bin", "layercom_cig")
GREEN_CLI = os.path.join(PKG, "bin", "greensol_auto")
DATUM_CLI = os.path.join(PKG, "bin", "kirchdat2d_freq")

SOURCES = ["kcig_kernels.cu", "kcig_plan.cu", "kcig_eikods.cu", "kcig_mlp.cu", "kcig_params.cpp", "kcig_rsf.cpp", "kcig_cli.cpp",
           "kcig_eikods_cli.cpp", "kcig_stitch.cu", "kcig_stitch_cli.cpp", "kcig_datum.cu", "kcig_datum_cli.cpp"]
HEADERS = ["kcig_common.h", "kcig_tc.h", "kcig_aperture.h", "kcig_par.h", "kcig_rsf.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> None:
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "kcig.h"),
                                                                 os.path.abspath(__file__)]
    env = dict(os.environ)
    env.setdefault("CC", "gcc")
    env["CXX"] = "g++"
    host = ["-ccbin", "g++"]
    if force or _stale(LIB, deps):
        # a variable used before it is set is an error, not a warning
        cmd = [nvcc(), *ARCH, *host, "-O3", "-lineinfo", "-std=c++17", "-Xcudafe", "--diag_error=549",
               "-Xcompiler", "-fPIC,-O3,-Werror=uninitialized,-Werror=maybe-uninitialized",
               "-Xptxas", "-v" if verbose else "-O3", "-shared", "-o", LIB,
               *[os.path.join(CSRC, s) for s in SOURCES], "-lcufft"]
        r = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True, env=env)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + r.stdout[-6000:] + r.stderr[-6000:])
        if verbose or "warning" in r.stderr:
            sys.stderr.write(r.stderr)
    for exe, src in ((CLI, "kirchmig2d_cig_main.cpp"), (EIK_CLI, "eikods2d_main.cpp"),
                     (K2D_CLI, "kirchmig2d_main.cpp"), (STITCH_CLI, "layercom_cig_main.cpp"),
                     (GREEN_CLI, "greensol_auto_main.cpp"), (DATUM_CLI, "kirchdat2d_freq_main.cpp")):
        main = os.path.join(CSRC, src)
        if force or _stale(exe, [LIB, main]):
            os.makedirs(os.path.dirname(exe), exist_ok=True)
            cmd = [nvcc(), *ARCH, *host, "-O2", "-std=c++17", "-o", exe, main, "-L" + PKG, "-lkcig",
                   "-Xlinker", "-rpath=$ORIGIN/.."]
            r = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True, env=env)
            if r.returncode != 0:
                raise RuntimeError("nvcc (%s) failed:\n" % src + r.stdout[-4000:] + r.stderr[-4000:])

if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
