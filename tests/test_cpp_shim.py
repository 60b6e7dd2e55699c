"""The header-only C++ layer (include/potts_min_partition.hpp) compiles against the C ABI and
links with libpotts_b200.so; without a GPU it reports the missing device as the reference does
(an exception), with one it runs a small solve."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_cpp_shim_builds_and_runs(native_lib, tmp_path):
    import torch

    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    lib_dir = ROOT / "segmentctscans_b200"
    exe = tmp_path / "shim_check"
    cmd = [gxx, "-std=c++17", "-O1", "-I", str(ROOT / "include"), str(ROOT / "tests" / "cpp" / "shim_check.cpp"),
           "-L", str(lib_dir), "-lpotts_b200", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    if torch.cuda.is_available():
        assert r.returncode == 0 and "solved" in r.stdout, r.stdout + r.stderr
    else:
        assert r.returncode == 2 and "no CUDA device" in r.stdout, r.stdout + r.stderr
