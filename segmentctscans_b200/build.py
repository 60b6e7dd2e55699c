"""Build recipe for the native library (sm_100a) — compiled in-tree.

``python -m segmentctscans_b200.build`` (or ``build_native()``) compiles the
``csrc/*.cu`` translation units (in parallel, objects under ``_build/``) and
links them into ``segmentctscans_b200/libpotts_b200.so`` with nvcc for
``sm_100a`` only.  The CUDA runtime is linked statically, so the library
needs only the NVIDIA driver at run time.  Arithmetic is compiled with
``-fmad=false``: the kernels fuse a multiply and an add only where the source
writes ``fmaf``.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
CSRC = PKG_DIR / "csrc"
INCLUDE = PKG_DIR.parent / "include"
LIB_NAME = "libpotts_b200.so"
LIB_PATH = PKG_DIR / LIB_NAME

COMPILE_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O2",
]
LINK_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-shared"]
OBJ_DIR = PKG_DIR / "_build"


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


def _compile(src: Path, ptxas_info: bool) -> tuple[Path, str]:
    obj = OBJ_DIR / (src.stem + ".o")
    cmd = [_nvcc(), *COMPILE_FLAGS, "-I", str(INCLUDE)]
    if ptxas_info:
        cmd += ["-Xptxas", "-v"]
    cmd += ["-c", str(src), "-o", str(obj) + ".tmp"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name} ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    os.replace(str(obj) + ".tmp", obj)
    return obj, res.stderr


def build_native(force: bool = False, verbose: bool = False, ptxas_info: bool = False,
                 jobs: int | None = None) -> Path:
    """Compile the CUDA library into the package directory; returns its path.  Each .cu file is
    one translation unit (the fused kernel variants have several), compiled in parallel and
    linked with the static CUDA runtime."""
    if not force and up_to_date():
        return LIB_PATH
    OBJ_DIR.mkdir(exist_ok=True)
    srcs = sources()
    newest_header = max((p.stat().st_mtime for p in headers()), default=0.0)

    def stale(src: Path) -> bool:
        obj = OBJ_DIR / (src.stem + ".o")
        return force or ptxas_info or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime,
                                                                                     newest_header)

    todo = [p for p in srcs if stale(p)]
    workers = max(1, min(len(todo) or 1, jobs or os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as pool:
        for obj, err in pool.map(lambda p: _compile(p, ptxas_info), todo):
            if ptxas_info or verbose:
                sys.stderr.write(err)
    objs = [OBJ_DIR / (p.stem + ".o") for p in srcs]
    cmd = [_nvcc(), *LINK_FLAGS, *map(str, objs), "-o", str(LIB_PATH) + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    os.replace(str(LIB_PATH) + ".tmp", LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    build_native(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB_PATH)
