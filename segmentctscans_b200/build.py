"""Build recipe for the native library (sm_100a) — compiled in-tree.

``python -m segmentctscans_b200.build`` (or ``build_native()``) compiles
``csrc/potts_b200.cu`` into ``segmentctscans_b200/libpotts_b200.so`` with nvcc
for ``sm_100a`` only.  The CUDA runtime is linked statically, so the library
needs only the NVIDIA driver at run time.  Arithmetic is compiled with
``-fmad=false``: the kernels fuse a multiply and an add only where the source
writes ``fmaf``.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
CSRC = PKG_DIR / "csrc"
INCLUDE = PKG_DIR.parent / "include"
LIB_NAME = "libpotts_b200.so"
LIB_PATH = PKG_DIR / LIB_NAME

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O2",
    "-shared",
]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def up_to_date() -> bool:
    if not LIB_PATH.exists():
        return False
    t = LIB_PATH.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in sources() + headers())


def build_native(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compile the CUDA library into the package directory; returns its path."""
    if not force and up_to_date():
        return LIB_PATH
    cmd = [_nvcc(), *NVCC_FLAGS, "-I", str(INCLUDE)]
    if ptxas_info:
        cmd += ["-Xptxas", "-v"]
    cmd += [str(p) for p in sources()] + ["-o", str(LIB_PATH) + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    if ptxas_info or verbose:
        sys.stderr.write(res.stderr)
    os.replace(str(LIB_PATH) + ".tmp", LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    build_native(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB_PATH)
