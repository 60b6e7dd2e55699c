"""Build recipe for the CPU oracle (test infrastructure only).

Compiles ``potts_oracle.c`` twice (REAL=double -> ``*_f64`` symbols, REAL=float
-> ``*_f32`` symbols) plus ``cylinder_oracle.c``, ``label_oracle.c`` and
``fieldio_oracle.c`` into
``oracle/_build/libpotts_oracle.so`` with gcc, OpenMP and ``-ffp-contract=off``
(no multiply-add is fused unless the source calls fma/fmaf).
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT_DIR = HERE / "_build"
LIB_PATH = OUT_DIR / "libpotts_oracle.so"
CFLAGS = ["-O2", "-fPIC", "-fopenmp", "-ffp-contract=off", "-fno-math-errno", "-std=c11", "-Wall", "-Wno-unused-variable"]
SOURCES = [HERE / "potts_oracle.c", HERE / "cylinder_oracle.c", HERE / "label_oracle.c", HERE / "fieldio_oracle.c"]


def up_to_date() -> bool:
    if not LIB_PATH.exists():
        return False
    t = LIB_PATH.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in SOURCES + [Path(__file__)])


def _run(cmd):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed: {' '.join(map(str, cmd))}\n{res.stdout}\n{res.stderr}")


def build_oracle(force: bool = False) -> Path:
    if not force and up_to_date():
        return LIB_PATH
    OUT_DIR.mkdir(exist_ok=True)
    cc = os.environ.get("ORACLE_CC") or ("/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc")
    objs = []
    for real, sfx, extra in (("double", "f64", []), ("float", "f32", ["-DORACLE_REAL_IS_FLOAT"])):
        obj = OUT_DIR / f"potts_oracle_{sfx}.o"
        _run([cc, *CFLAGS, f"-DREAL={real}", f"-DSFX={sfx}", *extra, "-c", str(SOURCES[0]), "-o", str(obj)])
        objs.append(obj)
    for src in SOURCES[1:]:
        obj = OUT_DIR / (src.stem + ".o")
        _run([cc, *CFLAGS, "-c", str(src), "-o", str(obj)])
        objs.append(obj)
    tmp = str(LIB_PATH) + ".tmp"
    _run([cc, "-shared", "-fopenmp", *map(str, objs), "-o", tmp, "-lm"])
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
