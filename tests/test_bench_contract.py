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


def test_refine_rate_bisection():
    """The served form's rate search: a fake server whose p99 grows with the
    rate (2 ms at 2,000 requests/s) and which serves every rate in full."""
    sys.path.insert(0, ROOT)
    import bench
    calls = []

    def p99_at(rate):
        calls.append(rate)
        return rate / 1000.0, rate

    rate, tput = bench.refine_rate(p99_at, (1000.0, 1000.0), 4000.0, 6)
    assert len(calls) == 6
    assert 2000.0 - 3000.0 / 64 <= rate < 2000.0 and tput == rate
    # nothing passes above the start: the start is kept
    rate, tput = bench.refine_rate(lambda r: (5.0, r), (1000.0, 900.0), 4000.0, 3)
    assert (rate, tput) == (1000.0, 900.0)
