"""The histogram kernels' bin decision (hist_bin_r, segmentctscans_b200/csrc/kernels_hist.cuh) restated
in C (tests/cpp/bin_rounding_check.c) gives the reference's bin for every value tested: random values,
the values next to both ends of each range and the 129 floats around every rounding boundary, over
ranges from a few ulps wide to subnormal and up to 65535 bins.  The GPU histograms are compared with
the oracle bit for bit in tests/test_gpu_labels.py; this covers the argument behind the reciprocal and
its division fallback on far more values than those tests can hold."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_bin_decision_matches_the_division(tmp_path):
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no gcc")
    exe = tmp_path / "bin_rounding_check"
    subprocess.run([gcc, "-O2", "-std=c11", "-ffp-contract=off", str(ROOT / "tests" / "cpp" / "bin_rounding_check.c"),
                    "-o", str(exe), "-lm"], check=True, capture_output=True)
    r = subprocess.run([str(exe), "500000"], capture_output=True, text=True, timeout=300)
    lines = [ln.split() for ln in r.stdout.splitlines() if ln.strip()]
    assert r.returncode == 0 and len(lines) == 11, r.stdout + r.stderr
    for start, end, nb, values, fallbacks, mismatches in lines:
        assert int(mismatches) == 0, (start, end, nb)
        assert int(values) > 500000
