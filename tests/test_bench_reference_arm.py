"""bench.py --impl reference (the reference arm, the FP32 restatement of the
reference loop on the host): one JSON line with the keys the driver reads,
and nothing of the CUDA product imported or loaded."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import runpy, sys
sys.argv = ["bench.py", "--impl", "reference", "--steps", "1", "--warmup", "0"]
try:
    runpy.run_path("bench.py", run_name="__main__")
except SystemExit:
    pass
maps = open("/proc/self/maps").read()
print("PRODUCT", "wavesim_b200._lib" in sys.modules, "libwavesim_b200" in maps)
"""


def test_reference_arm_line():
    out = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "higher_is_better", "config", "cpu_baseline",
              "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["higher_is_better"] is False and d["steps"] == 1
    assert d["e2e"]["value"] == d["value"] and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["cpu_baseline"]["value"] == d["value"]
    assert "PRODUCT False False" in out.stdout
