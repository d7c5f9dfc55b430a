"""bench.py's reference arm: the CPU restatement of the reference's algorithm on the workload's
whole volume, printed as the bench line, in a process that never loads this package's CUDA
library (the arm must not run any of this repository's product code)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = """
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--config", "tubes128", "--steps", "2", "--warmup", "1"]
runpy.run_path("bench.py", run_name="__main__")
maps = open("/proc/self/maps").read()
print("LOADED" if "libbrook_b200" in maps else "NOT LOADED")
"""


def test_reference_arm_prints_its_line_without_the_cuda_library():
    out = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    assert lines[-1] == "NOT LOADED"
    line = json.loads(lines[-2])
    assert line["impl"] == "reference" and line["unit"] == "voxels/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "voxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["config"]["voxels_per_gpu"] == 128 ** 3
