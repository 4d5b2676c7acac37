"""bench.py's reference arm on the CPU: it times the oracle (the CPU
restatement of the reference's step) on the bench's own workload, with the
requested warm-up, and prints the one JSON line the contract asks for, with
the same metric, unit and configuration as the GPU arm and no host-device
traffic in its e2e figure."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--nx", "256",
                        "--ny", "128", "--steps", "4", "--warmup", "3"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "MLUPS" and d["higher_is_better"] is True
    assert d["warmup"] == 3 and 1 <= d["steps"] <= 4 and d["value"] > 0
    assert d["config"]["nx"] == 256 and d["config"]["ny"] == 128
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
