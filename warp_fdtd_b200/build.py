"""Build the in-tree CUDA library warp_fdtd_b200/libwarp_fdtd_b200.so.

Every .cu under csrc/ is compiled for sm_100a only, with --fmad=false so that
float expressions round exactly as written (the arithmetic contract the
parity tests rely on), then linked with the static CUDA runtime into one
shared library exporting the C ABI declared in include/warp_fdtd_b200.h.

    python -m warp_fdtd_b200.build [--force] [-v]
"""

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = ROOT / "_build" / "obj"
LIB = PKG / "libwarp_fdtd_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = [
    "-O3",
    "-lineinfo",
    "--fmad=false",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "-I",
    str(ROOT / "include"),
]


def nvcc():
    found = shutil.which("nvcc")
    if found:
        return found
    cand = Path("/usr/local/cuda/bin/nvcc")
    if cand.exists():
        return str(cand)
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build")


def sources():
    return sorted(CSRC.glob("*.cu"))


def headers():
    return sorted(CSRC.glob("*.cuh")) + sorted((ROOT / "include").glob("*.h"))


def build(force=False, verbose=False, ptxas_info=False):
    OBJ.mkdir(parents=True, exist_ok=True)
    newest_header = max((p.stat().st_mtime for p in headers()), default=0)
    objs = []
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    for src in sources():
        obj = OBJ / (src.stem + ".o")
        objs.append(obj)
        if (
            not force
            and obj.exists()
            and obj.stat().st_mtime >= max(src.stat().st_mtime, newest_header)
        ):
            continue
        cmd = [nvcc(), *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if (
        force
        or not LIB.exists()
        or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs)
        or LIB.stat().st_mtime < CSRC.stat().st_mtime  # a source added or removed
    ):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", *map(str, objs), "-o", str(tmp)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers/spills")
    args = ap.parse_args()
    print(build(args.force, args.verbose, args.ptxas_info))
    sys.exit(0)
