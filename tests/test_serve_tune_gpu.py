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


@pytest.mark.parametrize("mode", [0, 1, 2, 3], ids=["batched", "plain", "batched_dev", "plain_dev"])
def test_served_results_identical_to_solo(tc, dev, mode):
    import torch
    plans, mats = make_plans(tc)
    srv = tc.Server(contexts=3, max_batch=32, arena_bytes=64 << 20)
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
