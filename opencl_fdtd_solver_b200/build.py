"""Build ``libfdtd_b200.so`` (the C ABI in ``include/fdtd_b200.h``) with nvcc for sm_100a.

    python -m opencl_fdtd_solver_b200.build [--force]

Every ``csrc/*.cu`` is compiled to an object with ``-gencode
arch=compute_100a,code=sm_100a -lineinfo -O3`` and linked into the package
directory, where ``_capi.py`` loads it.  Files that restate the reference's
per-cell arithmetic (the Yee kernels and the DFT) add ``--fmad=false`` so that
every product and sum is rounded separately, as in the CPU oracle.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
ROOT = PKG.parent
OUT = PKG / "libfdtd_b200.so"
BUILD_DIR = ROOT / "_build" / "csrc"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", str(ROOT / "include")]
# Files whose arithmetic must round like the oracle.
NO_FMA = {"yee_split.cu", "yee_fused.cu", "yee_shell.cu", "yee_face.cu", "dft.cu", "adjoint.cu",
          "adjoint_fused.cu", "materials.cu"}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; set NVCC or put the CUDA toolkit on PATH")


def build(force: bool = False, verbose: bool = False) -> Path:
    sources = sorted(CSRC.glob("*.cu"))
    headers = list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    newest = max(p.stat().st_mtime for p in sources + headers + [Path(__file__)])
    if OUT.exists() and not force and OUT.stat().st_mtime >= newest:
        return OUT
    BUILD_DIR.mkdir(parents=True, exist_ok=True)
    cc = nvcc()
    objs = []
    for src in sources:
        obj = BUILD_DIR / (src.stem + ".o")
        flags = list(COMMON)
        if src.name in NO_FMA:
            flags.append("--fmad=false")
        cmd = [cc, *ARCH, *flags, "-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [cc, *ARCH, "-shared", "-o", str(tmp), *objs, "-lcudart"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    args = ap.parse_args(argv)
    print(build(force=args.force, verbose=args.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
