"""Build libwpsph.so (sm_100a) in-tree with nvcc.

    python -m warpsph_b200.build [--force] [--verbose-ptxas]

The library is plain CUDA C++ with a C ABI (include/wpsph.h); it has no
PyTorch dependency and is loaded by warpsph_b200._lib through ctypes.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libwpsph.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libwpsph.so")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = sources() + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, ptxas_verbose: bool = False) -> Path:
    if not force and not _stale():
        return LIB
    ccbin = "/usr/bin/g++" if Path("/usr/bin/g++").exists() else "g++"
    cmd = [nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "-ccbin", ccbin,
           "-Xcompiler", "-fPIC", "-shared", "-I", str(ROOT / "include"),
           "-o", str(LIB)]
    if ptxas_verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [str(s) for s in sources()]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_verbose=a.verbose_ptxas))
    sys.exit(0)
