"""Served form (resident matrices, HBM admission, continuous batching) and
the autotuner.  Every served result must equal the same matrix's solo
multiply bit for bit, alone and in the mix."""
import numpy as np
import pytest

import oracle
from tests.golden import cases

pytestmark = pytest.mark.gpu

NAMES = ["band_holes", "two_segments", "multi_shape", "cfg1_small", "wide_band", "rmat16_selfloops"]


def make_plans(tc):
    plans, mats = [], []
    for nm in NAMES:
        case = next(c for c in cases.MATRIX_CASES if c["name"] == nm)
        M, N, rp, col = cases.matrix(case)
        plans.append(tc.Plan.from_csr(M, N, rp, col))
        mats.append((M, N, rp, col))
    return plans, mats


def solo(plan, x, M, dev):
    import torch
    y = torch.empty(M, device=dev)
    plan.spmv(torch.from_numpy(x).to(dev), y)
    torch.cuda.synchronize()
    return y.cpu().numpy()


@pytest.mark.parametrize("mode,solo_bytes", [(0, 0), (1, 0), (2, 0), (3, 0), (0, 1), (2, 1)],
                         ids=["batched", "plain", "batched_dev", "plain_dev", "batched_solo", "batched_dev_solo"])
def test_served_results_identical_to_solo(tc, dev, mode, solo_bytes):
    """solo_bytes = 1: every matrix counts as large, so each request runs its own
    multiply launch inside its batch (the path of large matrices)."""
    import torch
    plans, mats = make_plans(tc)
    srv = tc.Server(contexts=3, max_batch=32, arena_bytes=64 << 20, solo_bytes=solo_bytes)
    ids = [srv.admit(p) for p in plans]
    rng = np.random.default_rng(3 + mode)
    n = 300
    matrix = rng.integers(0, len(plans), n)
    # a burst: the requests arrive within half a millisecond, so batches mix matrices
    arrival = np.sort(rng.uniform(0, 0.0005, n))
    xs, ys, want = [], [], []
    for r in range(n):
        M, N, rp, col = mats[matrix[r]]
        x = torch.from_numpy(rng.uniform(-1, 1, N).astype(np.float32)).pin_memory()
        want.append(solo(plans[matrix[r]], x.numpy(), M, dev))
        if mode & tc.SERVE_DEVICE_VECTORS:
            xs.append(x.to(dev))
            ys.append(torch.full((M,), float("nan"), device=dev))
        else:
            xs.append(x)
            ys.append(torch.full((M,), float("nan")).pin_memory())
    stats, lat = srv.run(arrival, [ids[m] for m in matrix], xs, ys, mode=mode)
    torch.cuda.synchronize()
    xs = [x.cpu() for x in xs]
    ys = [y.cpu() for y in ys]
    for r in range(n):
        np.testing.assert_array_equal(ys[r].numpy(), want[r], err_msg="request %d" % r)
    assert stats["requests"] == n and (lat > 0).all()
    if mode & 1 == 0:
        assert stats["mean_batch"] > 1.0          # requests were batched together
    print("mode %d: %.0f SpMV/s, p50 %.3f ms, p99 %.3f ms, mean batch %.1f" % (
        mode, stats["spmv_per_s"], stats["p50_ms"], stats["p99_ms"], stats["mean_batch"]))
    # and against the FP64 oracle within the stated tolerance
    for r in range(0, n, 37):
        M, N, rp, col = mats[matrix[r]]
        y64 = oracle.spmv_csr_f64(M, rp, col, xs[r].numpy().astype(np.float64))
        assert np.linalg.norm(ys[r].numpy() - y64) <= 1e-5 * np.linalg.norm(y64)
    srv.close()


def test_admission_by_footprint(tc, dev):
    plans, _ = make_plans(tc)
    arena = 16 << 20
    budget = 3 * arena + sum(p.info()["device_bytes"] for p in plans[:3]) + 1024
    srv = tc.Server(contexts=3, arena_bytes=arena, hbm_budget=budget)
    ids = [srv.admit(p) for p in plans[:3]]
    with pytest.raises(tc.TcError) as e:
        srv.admit(plans[3])
    assert e.value.status == 6          # TC_ERR_CAPACITY
    used = srv.hbm_used()
    srv.evict(ids[0])
    assert srv.hbm_used() == used - plans[0].info()["device_bytes"]
    if plans[3].info()["device_bytes"] <= plans[0].info()["device_bytes"] + 1024:
        srv.admit(plans[3])
    srv.close()


def test_tuner(tc, dev):
    import torch
    case = next(c for c in cases.MATRIX_CASES if c["name"] == "overlap")
    M, N, rp, col = cases.matrix(case)
    tc.lib().tc_tune_cache_clear()
    r = tc.tune(M, N, rp, col, max_trials=10)
    assert 1 <= r.trials <= 10 and r.cached == 0 and r.spmv_us > 0
    assert r.spmv_us <= r.default_us * 1.0001
    again = tc.tune(M, N, rp, col, max_trials=10)
    assert again.cached == 1 and again.trials == 0 and again.fingerprint == r.fingerprint
    # the tuned plan computes the same product
    plan = tc.Plan.from_csr(M, N, rp, col, prm=r.params)
    x = np.random.default_rng(0).integers(-8, 9, N).astype(np.float32)
    y = solo(plan, x, M, dev)
    np.testing.assert_array_equal(y.astype(np.float64),
                                  oracle.spmv_csr_f64(M, rp, col, x.astype(np.float64)))
    print("tuned: density %.2f tile_rows %d max_lanes %d ctas/SM %d: %.2f us (default %.2f us)" % (
        r.params.density, r.params.tile_rows, r.params.max_lanes, r.params.ctas_per_sm, r.spmv_us,
        r.default_us))


def test_online_submit_poll_wait(tc, dev):
    """The online interface: requests submitted from two threads while the
    dispatcher batches them, completed through poll and wait; every y equals
    the matrix's solo multiply bit for bit.  Then the host-vector form."""
    import threading
    import torch
    plans, mats = make_plans(tc)
    srv = tc.Server(contexts=3, max_batch=32, max_inflight=2, arena_bytes=64 << 20)
    ids = [srv.admit(p) for p in plans]
    rng = np.random.default_rng(21)
    n = 400
    matrix = rng.integers(0, len(plans), n)
    xs = [torch.from_numpy(rng.uniform(-1, 1, mats[m][1]).astype(np.float32)) for m in matrix]
    want = [solo(plans[m], x.numpy(), mats[m][0], dev) for m, x in zip(matrix, xs)]
    for device_vectors in (True, False):
        if device_vectors:
            X = [x.to(dev) for x in xs]
            Y = [torch.full((mats[m][0],), float("nan"), device=dev) for m in matrix]
        else:
            X = [x.pin_memory() for x in xs]
            Y = [torch.full((mats[m][0],), float("nan")).pin_memory() for m in matrix]
        srv.start(device_vectors=device_vectors)
        tickets = [None] * n

        def feed(lo):
            for r in range(lo, n, 2):
                tickets[r] = srv.submit(ids[matrix[r]], X[r], Y[r])

        th = [threading.Thread(target=feed, args=(k,)) for k in (0, 1)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        import time
        pending, t0 = set(range(n)), time.time()
        while pending:                       # poll until all are done
            pending = {r for r in pending if not srv.poll(tickets[r])}
            assert time.time() - t0 < 60, "%d requests not done after 60 s" % len(pending)
        srv.wait(tickets[-1], 10.0)
        st = srv.stats()
        srv.stop()
        assert st["requests"] == n and st["batches"] >= 1
        for r in range(n):
            np.testing.assert_array_equal(Y[r].cpu().numpy(), want[r], err_msg="request %d" % r)
        print("online %s: %d batches, mean batch %.1f, p99 %.3f ms" % (
            "device" if device_vectors else "host", st["batches"], st["mean_batch"], st["p99_ms"]))
    with pytest.raises(tc.TcError):
        srv.submit(ids[0], X[0], Y[0])          # stopped
    srv.close()


def test_served_pool_48(tc, dev):
    """The served workload's own pool (48 resident matrices: R-MAT scales
    14-22 and banded matrices of 1e4-4e6 rows), 1,500 requests with Zipf(1.1)
    matrix choice arriving as a Poisson stream: each y bit-identical to the
    matrix's solo multiply of the same x (alone vs in the mix), and within
    1e-5 of the FP64 oracle normwise on every request of a strided sample."""
    import torch
    from taichi_b200 import workloads
    mats = workloads.pool_matrices("serve", 48, 11)
    srv = tc.Server(contexts=4, max_batch=64, max_inflight=2, arena_bytes=256 << 20)
    plans, ids = [], []
    for name, M, rp, col in mats:
        p = tc.Plan.from_csr(M, M, rp, col)
        plans.append(p)
        ids.append(srv.admit(p))
    rng = np.random.default_rng(31)
    pz = np.arange(1, 49, dtype=np.float64) ** -1.1
    pz /= pz.sum()
    n = 1500
    matrix = rng.choice(48, size=n, p=pz)
    xs = [torch.empty(m[1], device=dev).uniform_(-1, 1) for m in mats]      # one x per matrix
    solo_y = []
    for p, x, m in zip(plans, xs, mats):
        y = torch.empty(m[1], device=dev)
        p.spmv(x, y)
        solo_y.append(y)
    ys = [torch.full((mats[m][1],), float("nan"), device=dev) for m in matrix]
    arrival = np.cumsum(rng.exponential(1.0 / 50000, n))
    stats, lat = srv.run(arrival, [ids[m] for m in matrix], [xs[m] for m in matrix], ys,
                         mode=tc.SERVE_DEVICE_VECTORS)
    torch.cuda.synchronize()
    assert stats["requests"] == n
    for r in range(n):
        assert torch.equal(ys[r], solo_y[matrix[r]]), "request %d (matrix %d)" % (r, matrix[r])
    worst = 0.0
    for r in range(0, n, 61):
        name, M, rp, col = mats[matrix[r]]
        y64 = oracle.spmv_csr_f64(M, rp, col, xs[matrix[r]].cpu().numpy().astype(np.float64))
        rel = np.linalg.norm(ys[r].cpu().numpy() - y64) / np.linalg.norm(y64)
        worst = max(worst, rel)
        assert rel <= 1e-5, (r, name, rel)
    print("pool48: %.0f SpMV/s, p50 %.3f ms, p99 %.3f ms, mean batch %.1f, worst rel err %.2e" % (
        stats["spmv_per_s"], stats["p50_ms"], stats["p99_ms"], stats["mean_batch"], worst))
    srv.close()
    for p in plans:
        p.close()
