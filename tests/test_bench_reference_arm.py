"""The reference arm of bench.py (`--impl reference`) on the host: the C++
restatement of the reference's OpenMP path times a bounded sample and prints
one JSON line with the contract's keys; ranks other than 0 print nothing."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CMD = [sys.executable, "bench.py", "--impl", "reference", "--workload", "turb_inflow_q27_256x128x128",
       "--steps", "1", "--warmup", "0"]


def run(env_extra):
    env = dict(os.environ, **env_extra)
    r = subprocess.run(CMD, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return [ln for ln in r.stdout.splitlines() if ln.startswith("{")]


def test_reference_arm_prints_the_contract_line():
    lines = run({"RANK": "0"})
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "MLUPS" and d["value"] > 0
    assert d["higher_is_better"] is True and d["steps"] == 1 and d["warmup"] == 0
    assert d["config"]["workload"] == "turb_inflow_q27_256x128x128"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_do_no_work():
    assert run({"RANK": "1"}) == []
