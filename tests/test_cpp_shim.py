"""The header-only C++ layer (include/potts_min_partition.hpp, include/field_io.hpp) compiles against
the C ABI and links with libpotts_b200.so.  Without a GPU it reports the missing device as the
reference does (an exception); on a GPU it runs a small solve, then saves and loads the result as
a field archive (marked gpu, so the GPU suite runs the C++ layer)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _build_shim(tmp_path) -> Path:
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    lib_dir = ROOT / "segmentctscans_b200"
    exe = tmp_path / "shim_check"
    cmd = [gxx, "-std=c++17", "-O1", "-I", str(ROOT / "include"), str(ROOT / "tests" / "cpp" / "shim_check.cpp"),
           "-L", str(lib_dir), "-lpotts_b200", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def test_cpp_shim_reports_a_missing_device(native_lib, tmp_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present (test_cpp_shim_solves_on_the_gpu covers it)")
    r = subprocess.run([str(_build_shim(tmp_path))], capture_output=True, text=True)
    assert r.returncode == 2 and "no CUDA device" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_cpp_shim_solves_on_the_gpu(native_lib, cuda_device, tmp_path):
    r = subprocess.run([str(_build_shim(tmp_path))], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "solved" in r.stdout, r.stdout + r.stderr
