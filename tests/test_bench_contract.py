"""bench.py's CPU sides: the phantom that the CPU baseline and the reference arm time is built
without loading the GPU library (only the oracle), and it has the config-1 cross-section."""
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]

PROBE = r"""
import sys
sys.argv = ["bench.py"]
sys.path.insert(0, %r)
import bench
ph = bench.cpu_sample_phantom()
maps = open("/proc/self/maps").read()
print(ph.mapping.data_size, ph.mapping.n_lines, "libpotts_b200" in maps, "libpotts_oracle" in maps)
"""


def test_reference_arm_phantom_does_not_load_the_product(oracle_mod):
    r = subprocess.run([sys.executable, "-c", PROBE % str(ROOT)], capture_output=True, text=True, cwd=ROOT,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    size, lines, product, oracle_loaded = r.stdout.split()
    assert (int(size), int(lines)) == (430112 * 16, 430112)
    assert product == "False" and oracle_loaded == "True"
