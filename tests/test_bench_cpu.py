"""The bench's reference arm (the reference's CPU path: the oracle port of ParticlesPhysics.py,
FP64, all host threads) runs without a GPU; its JSON line carries the keys the measurement
contract asks for."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    res = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "2",
                          "--warmup", "1", "--n", "4096"], cwd=ROOT, capture_output=True,
                         text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
    line = json.loads(res.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "dtype", "data", "config", "cpu_baseline",
                "e2e"):
        assert key in line, key
    assert line["value"] > 0 and line["unit"] == "Gpairs/s" and line["steps"] == 2
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["e2e"]["value"] == line["value"]
