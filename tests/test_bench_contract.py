"""bench.py on the CPU: the reference arm prints one JSON line with the
contract's keys on rank 0 and nothing (exit 0) on the other ranks of a
multi-rank launch; the served form's rate bisection against a fake server."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
KEYS = ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
        "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e")


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--workload", "small",
                           "--steps", "2", "--warmup", "1"], cwd=ROOT, env=env, timeout=600,
                          stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)


def test_reference_arm_line():
    r = _run({"RANK": "0", "WORLD_SIZE": "1", "LOCAL_RANK": "0"})
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in KEYS:
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "GB/s"
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["config"]["bytes_per_spmv"] == 4 * (65536 + 1) + 4 * d["config"]["nnz"] + 8 * 65536


def test_reference_arm_other_ranks_idle():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]


def test_highest_passing_rate():
    """The served form's rate search against a fake server whose p99 grows
    with the rate (2 ms at 2,000 requests/s) and which serves every rate in
    full: the sweep stops after two failing rates in a row and the bisection
    closes in on 2,000 from below; a lone failing rate (a stall) does not end
    the sweep."""
    sys.path.insert(0, ROOT)
    import bench
    calls = []

    def serve_at(rate):
        calls.append(rate)
        return {"p99_ms": rate / 1000.0, "spmv_per_s": rate}

    best, runs = bench.highest_passing_rate(serve_at, [500.0, 1000.0, 4000.0, 8000.0, 9000.0], 6)
    assert calls[:4] == [500.0, 1000.0, 4000.0, 8000.0] and len(calls) == 4 + 6
    assert 2000.0 - 3000.0 / 64 <= best["spmv_per_s"] < 2000.0
    assert len(runs) == len(calls)
    # a stall at 1,000 only: the sweep goes on to 1,500
    stall = lambda r: {"p99_ms": 5.0 if r == 1000.0 else r / 1000.0, "spmv_per_s": r}
    best, runs = bench.highest_passing_rate(stall, [500.0, 1000.0, 1500.0, 2500.0, 3000.0], 0)
    assert best["spmv_per_s"] == 1500.0
    # nothing passes: no best run, and no bisection
    best, runs = bench.highest_passing_rate(lambda r: {"p99_ms": 5.0, "spmv_per_s": r}, [100.0, 200.0, 300.0], 4)
    assert best is None and len(runs) == 2
    # everything passes: the highest rate, no bisection
    best, runs = bench.highest_passing_rate(lambda r: {"p99_ms": 0.1, "spmv_per_s": r}, [1.0, 2.0, 3.0], 4)
    assert best["spmv_per_s"] == 3.0 and len(runs) == 3
