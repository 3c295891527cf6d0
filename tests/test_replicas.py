"""The multi-GPU path of the bench is N independent replicas; these tests run
its process-group plumbing as two gloo ranks on the CPU: every rank gets the
slowest rank's time, and the reference arm works on rank 0 alone."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from taichi_b200 import replicas
    r, w, lr = replicas.init("gloo", timeout_s=60)
    replicas.barrier(w)
    got = replicas.max_over_ranks(1.5 + r, w)        # rank 1 is the slow one
    replicas.barrier(w)
    replicas.finish(w)
    with open(os.path.join(out, "rank%d.json" % r), "w") as f:
        json.dump({"rank": r, "world": w, "local_rank": lr, "max": got}, f)


def test_max_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        with open(tmp_path / ("rank%d.json" % r)) as f:
            d = json.load(f)
        assert d == {"rank": r, "world": 2, "local_rank": r, "max": 2.5}


def test_single_rank_needs_no_group():
    sys.path.insert(0, ROOT)
    from taichi_b200 import replicas
    assert replicas.max_over_ranks(3.25, 1) == 3.25
    replicas.barrier(1)
    replicas.finish(1)


@pytest.mark.parametrize("rank", [1])
def test_reference_arm_other_ranks_exit_quietly(rank):
    """Under torchrun only rank 0 runs and prints the reference arm; the other
    ranks exit 0 without work."""
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "1"],
                       env=env, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
