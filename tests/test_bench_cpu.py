"""bench.py's reference arm on the CPU: the JSON line it prints and its ranks.

`bench.py --impl reference` times the CPU restatement of the stage path on the
host cores (no GPU). Here it runs on the small Orszag-Tang workload: the line
must carry the contract's keys, the requested warm-up and timed step counts,
and zero host-device bytes; under a launcher every rank but 0 exits at once
without output.
"""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench(*args, env=None):
    e = dict(os.environ)
    e.update(env or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], cwd=ROOT,
                          env=e, capture_output=True, text=True, timeout=600)


def test_reference_arm_line():
    r = _bench("--impl", "reference", "--workload", "ot", "--steps", "3", "--warmup", "4")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "impl", "cpu_baseline", "e2e"):
        assert key in d, key
    assert d["impl"] == "reference"
    assert d["metric"] == d["unit"] == "zone-cycles/s" and d["higher_is_better"] is True
    assert d["steps"] == 3 and d["warmup"] == 4
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["config"]["workload"].startswith("orszag_tang_2d_256x256")
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["kind"] in ("port", "reference") and cb["cores"] >= 1
    assert cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_exit_quietly():
    r = _bench("--impl", "reference", "--workload", "ot", "--steps", "2", "--warmup", "3",
               env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
