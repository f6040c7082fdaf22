"""bench.py's reference arm (the reference algorithm on the host cores, no GPU)
prints the one JSON line of the bench contract: the same metric and unit as the
GPU arm, impl "reference", its cpu_baseline and an e2e block without copies,
warm-up raised to at least 3; under a launcher, ranks other than 0 exit 0
without output."""
import json
import os
import subprocess
import sys

import bench

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_bench(args, env_extra=None):
    env = dict(os.environ)
    env.update(env_extra or {})
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args],
                          capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)


def test_reference_arm_line():
    r = run_bench(["--impl", "reference", "--steps", "2", "--warmup", "0", "--ref-n", "16"])
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["impl"] == "reference" and d["steps"] == 2 and d["warmup"] == 3
    assert d["value"] > 0 and d["ms_per_step"] > 0
    assert d["higher_is_better"] is True and d["dtype"] == "f64" and d["data"] == "synthetic"
    assert d["vs_baseline"] is None and d["scaling"] in ("weak", "strong")
    assert "workload" in d["config"]
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"] and cb["kind"] == "port"
    assert cb["cores"] >= 1 and cb["sample"]
    e = d["e2e"]
    assert e["value"] == d["value"] and e["unit"] == d["unit"]
    assert e["h2d_bytes_per_step"] == 0 and e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_are_silent():
    r = run_bench(["--impl", "reference", "--steps", "1", "--ref-n", "16"],
                  {"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_timeline_summary():
    """The e2e timeline summary: copy spans, busy times, the gaps between
    consecutive downloads and the compute's stage-1 ends, from per-slab rows."""
    import numpy as np
    # three slabs: upload start/end, stage 0, stage 1 end, conversion, download start/end
    tl = np.array([[0.0, 1.0, 1.1, 2.0, 2.1, 2.1, 3.0],
                   [1.0, 2.0, 2.1, 3.0, 3.1, 3.1, 4.0],
                   [2.0, 3.0, 3.1, 5.0, 5.1, 5.5, 6.5]])
    s = bench.io_timeline_summary(tl)
    assert s["slabs"] == 3 and s["ms_end"] == 6.5
    assert s["upload_start_end_ms"] == [0.0, 3.0] and s["upload_busy_ms"] == 3.0
    assert s["download_start_end_ms"] == [2.1, 6.5]
    assert abs(s["download_busy_ms"] - 2.8) < 1e-12
    assert abs(s["download_idle_ms"] - 1.6) < 1e-12  # 3.0 -> 3.1 and 4.0 -> 5.5
    assert s["download_longest_gaps_ms"][0] == 1.5
    assert s["stage1_first_last_end_ms"] == [2.0, 5.0] and s["conversion_last_end_ms"] == 5.1


def test_host_plan_uses_the_schedule_counts(monkeypatch):
    """The adjoint's host level is chosen from the checkpoint schedule's own
    recompute counts within the host memory cap: none when the host holds too
    little, and then a stride whose segments recompute fewer steps than the
    device pool alone."""
    from boxzyhydro_b200.adjoint import plan
    set_bytes = 5.5e9
    monkeypatch.setattr(bench, "host_mem_available", lambda: int(20e9))
    assert bench.auto_host_plan(400, 20, set_bytes) == (0, None)
    monkeypatch.setattr(bench, "host_mem_available", lambda: int(196e9))
    L, snaps = bench.auto_host_plan(400, 20, set_bytes)
    assert L >= 2 and snaps == 16
    assert ((400 - 1) // L) * set_bytes <= 0.45 * 196e9
    host = sum(plan(min(L, 400 - a), snaps - 2)["recomputed_again"]
               for a in range(0, 400, L) if min(L, 400 - a) > 1)
    assert host < plan(400, 16)["recomputed_first"]
