"""bench.py's reference arm and the CPU sampler behind it, without a GPU.

The reference is single-threaded; the c4 ensemble's members are independent simulations, so the
reference arm runs one member per usable host core side by side (oracle/ref_runner.py run_parallel)
and reports the sum of their step rates.  These tests check the core assignment with a stand-in for
the reference binary, and the JSON line of `bench.py --impl reference` when the reference is built.
"""
import json
import os
import subprocess
import sys
import threading
import time

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_parallel_runs_never_share_a_core(monkeypatch):
    from oracle import ref_runner
    monkeypatch.setattr(ref_runner, "usable_cpus", lambda: [3, 5, 7])
    lock = threading.Lock()
    spans = []

    def fake_run(wl, tag, steps, warmup, timeout, cpu, keep_cache):
        t0 = time.monotonic()
        time.sleep(0.02 + 0.01 * (int(tag) % 3))
        with lock:
            spans.append((cpu, t0, time.monotonic()))
        return {"tag": tag, "cpu": cpu}

    monkeypatch.setattr(ref_runner, "run", fake_run)
    jobs = [(None, str(i)) for i in range(10)]
    out = ref_runner.run_parallel(jobs, steps=1, warmup=0)
    assert [r["tag"] for r in out] == [str(i) for i in range(10)]  # job order
    assert {r["cpu"] for r in out} <= {3, 5, 7}
    for i, (c1, a1, b1) in enumerate(spans):
        for c2, a2, b2 in spans[i + 1:]:
            if c1 == c2:
                assert b1 <= a2 or b2 <= a1  # one run per core at a time


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "ref_driver")),
                    reason="the reference is not built (oracle/Makefile)")
def test_reference_arm_json_line():
    p = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", "1", "--warmup", "1"],
                       cwd=ROOT, capture_output=True, text=True, timeout=900)
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads([l for l in p.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference"
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "dtype", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["config"]["workload"] == "c4" and line["config"]["members"] == 64
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == line["value"]
    from oracle import ref_runner
    assert cb["cores"] == min(len(ref_runner.usable_cpus()), 37)  # one member per core (37 have n <= 256)
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
