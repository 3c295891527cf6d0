"""SpMM (1..64 right-hand sides) and the batched launch over many plans,
against the FP64 oracle and against the single-plan multiply
(bit-identical, including plans of wide direct tiles, which the batch runs as
quarter-tile work items)."""
import numpy as np
import pytest

import oracle
from tests.golden import cases

pytestmark = pytest.mark.gpu


def dev_t(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


@pytest.mark.parametrize("k", [1, 2, 7, 32, 33, 64])
@pytest.mark.parametrize("name", ["band_holes", "multi_shape", "cfg1_small"])
def test_spmm(tc, dev, k, name):
    import torch
    case = next(c for c in cases.MATRIX_CASES if c["name"] == name)
    M, N, rp, col = cases.matrix(case)
    fmt, _ = oracle.partition(M, N, rp, col)
    plan = tc.Plan.from_format(M, N, fmt)
    rng = np.random.default_rng(k)
    X = rng.integers(-8, 9, (N, k)).astype(np.float32)
    Y = torch.full((M, k), float("nan"), device=dev)
    plan.spmm(dev_t(X, dev), Y)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(Y.cpu().numpy().astype(np.float64),
                                  oracle.spmm_csr_f64(M, rp, col, X.astype(np.float64)))
    # column j of SpMM == SpMV of column j for integer X (exact either way)
    Xf = rng.uniform(-1, 1, (N, k)).astype(np.float32)
    plan.spmm(dev_t(Xf, dev), Y)
    torch.cuda.synchronize()
    Y64 = oracle.spmm_csr_f64(M, rp, col, Xf.astype(np.float64))
    rel = np.linalg.norm(Y.cpu().numpy() - Y64) / np.linalg.norm(Y64)
    print("spmm %s k=%d rel err %.2e" % (name, k, rel))
    assert rel <= 1e-5


def test_spmm_strided(tc, dev):
    import torch
    case = cases.MATRIX_CASES[2]
    M, N, rp, col = cases.matrix(case)
    fmt, _ = oracle.partition(M, N, rp, col)
    plan = tc.Plan.from_format(M, N, fmt)
    X = np.random.default_rng(0).integers(-8, 9, (N, 40)).astype(np.float32)
    Y = torch.zeros((M, 48), device=dev)
    plan.spmm(dev_t(X, dev), Y, k=20, ldx=40, ldy=48)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(Y.cpu().numpy()[:, :20].astype(np.float64),
                                  oracle.spmm_csr_f64(M, rp, col, X[:, :20].astype(np.float64)))
    assert not Y.cpu().numpy()[:, 20:].any()


def test_batch_identical_to_solo(tc, dev):
    import ctypes as C
    import torch
    names = ["band_holes", "two_segments", "multi_shape", "cfg1_small", "wide_band", "overlap",
             "rmat16_selfloops", "plain:rmat16_selfloops", "plain:sparse"]
    plans, xs, ys, solo = [], [], [], []
    rng = np.random.default_rng(5)
    for nm in names:
        if nm == "plain:sparse":             # rows of <= 1 entry on average: wide direct tiles
            M = N = 9000
            rp = np.zeros(M + 1, np.int32)
            np.cumsum(rng.integers(0, 2, M), out=rp[1:])
            col = rng.integers(0, N, int(rp[-1])).astype(np.int32)
            p = tc.Plan.from_csr(M, N, rp, col, partition=False)
        else:
            case = next(c for c in cases.MATRIX_CASES if c["name"] == nm.split(":")[-1])
            M, N, rp, col = cases.matrix(case)
            if nm.startswith("plain:"):
                p = tc.Plan.from_csr(M, N, rp, col, partition=False)
            else:
                fmt, _ = oracle.partition(M, N, rp, col)
                p = tc.Plan.from_format(M, N, fmt)
        x = torch.from_numpy(rng.uniform(-1, 1, N).astype(np.float32)).to(dev)
        y = torch.empty(M, device=dev)
        p.spmv(x, y)
        torch.cuda.synchronize()
        solo.append(y.clone())
        y.fill_(float("nan"))
        plans.append(p); xs.append(x); ys.append(y)
    n = len(plans)
    H = (C.c_void_p * n)(*[p.handle.value for p in plans])
    X = (C.c_void_p * n)(*[x.data_ptr() for x in xs])
    Yp = (C.c_void_p * n)(*[y.data_ptr() for y in ys])
    b = C.c_void_p()
    tc.check(tc.lib().tc_batch_create(n, H, X, Yp, C.byref(b)))
    tc.check(tc.lib().tc_batch_run(b, None))
    torch.cuda.synchronize()
    for y, s in zip(ys, solo):
        assert torch.equal(y, s)
    for y in ys:
        y.fill_(float("nan"))
    for _ in range(3):
        tc.check(tc.lib().tc_batch_graph_launch(b, None))
    torch.cuda.synchronize()
    for y, s in zip(ys, solo):
        assert torch.equal(y, s)
    tc.check(tc.lib().tc_batch_destroy(b))


def test_spmm_rmat22_k64_full_size(tc, dev):
    """The batched-RHS workload at its configured size: R-MAT scale 22
    (a = 0.499, b = c = 0.001, edge factor 16) times a 4,194,304 x 64 FP32
    X, checked on a strided sample of rows (every 61st, 68,760 rows) against
    the FP64 product: integer X in [-8, 8] exact; FP32 X uniform in [-1, 1]
    within 1e-5 normwise and per row (against the row's sum of |terms|)."""
    import torch
    import scipy.sparse as sp
    M, rp, col = tc.gen_rmat(22, 16, 0.499, 0.001, 0.001, seed=1)
    N, k = M, 64
    plan = tc.Plan.from_csr(M, N, rp, col)
    A = sp.csr_matrix((np.ones(len(col)), col, rp), shape=(M, N))
    rows = np.arange(0, M, 61)
    As = A[rows]
    used = np.unique(As.indices)
    As = sp.csr_matrix((As.data, np.searchsorted(used, As.indices), As.indptr), shape=(len(rows), len(used)))
    Y = torch.empty((M, k), device=dev)
    g = torch.Generator(device=dev).manual_seed(3)
    Xi = torch.randint(-8, 9, (N, k), device=dev, generator=g).float()
    plan.spmm(Xi, Y)
    torch.cuda.synchronize()
    want = As @ Xi[torch.from_numpy(used).to(dev)].double().cpu().numpy()
    np.testing.assert_array_equal(Y[torch.from_numpy(rows).to(dev)].double().cpu().numpy(), want)
    Xf = torch.empty((N, k), device=dev).uniform_(-1, 1, generator=g)
    plan.spmm(Xf, Y)
    torch.cuda.synchronize()
    Xu = Xf[torch.from_numpy(used).to(dev)].double().cpu().numpy()
    y64 = As @ Xu
    bound = abs(As) @ np.abs(Xu)
    got = Y[torch.from_numpy(rows).to(dev)].double().cpu().numpy()
    rel = np.linalg.norm(got - y64) / np.linalg.norm(y64)
    roww = np.max(np.abs(got - y64) / np.maximum(bound, 1e-30))
    print("spmm rmat22 k=64: normwise rel err %.2e, max row-wise err %.2e (%d sampled rows)" % (
        rel, roww, len(rows)))
    assert rel <= 1e-5 and roww <= 1e-5
    plan.close()


def test_batch_256_against_oracle(tc, dev):
    """The batched workload at its configured size: 256 matrices of uneven
    size (n log-uniform in [1e3, 2e5], half R-MAT, half banded), one batch
    launch: every matrix's y against the FP64 oracle -- exact for integer x,
    within 1e-5 normwise for FP32 x -- and equal to its solo multiply."""
    import ctypes as C
    import torch
    from taichi_b200 import workloads
    mats = workloads.pool_matrices("batch", 256, 7)
    plans = [tc.Plan.from_csr(M, M, rp, col) for _, M, rp, col in mats]
    rng = np.random.default_rng(19)
    for integer in (True, False):
        xh = [(rng.integers(-8, 9, M) if integer else rng.uniform(-1, 1, M)).astype(np.float32)
              for _, M, _, _ in mats]
        xs = [torch.from_numpy(x).to(dev) for x in xh]
        ys = [torch.full((m[1],), float("nan"), device=dev) for m in mats]
        n = len(plans)
        H = (C.c_void_p * n)(*[p.handle.value for p in plans])
        X = (C.c_void_p * n)(*[x.data_ptr() for x in xs])
        Yp = (C.c_void_p * n)(*[y.data_ptr() for y in ys])
        b = C.c_void_p()
        tc.check(tc.lib().tc_batch_create(n, H, X, Yp, C.byref(b)))
        tc.check(tc.lib().tc_batch_graph_launch(b, None))
        torch.cuda.synchronize()
        worst = 0.0
        for i, (name, M, rp, col) in enumerate(mats):
            y = ys[i].cpu().numpy().astype(np.float64)
            y64 = oracle.spmv_csr_f64(M, rp, col, xh[i].astype(np.float64))
            if integer:
                np.testing.assert_array_equal(y, y64, err_msg=name)
            else:
                rel = np.linalg.norm(y - y64) / max(np.linalg.norm(y64), 1e-300)
                worst = max(worst, rel)
                assert rel <= 1e-5, (name, rel)
            solo = torch.empty(M, device=dev)
            plans[i].spmv(xs[i], solo)
            assert torch.equal(solo, ys[i]), name
        tc.check(tc.lib().tc_batch_destroy(b))
        if not integer:
            print("batch of 256: worst normwise rel err %.2e" % worst)
    for p in plans:
        p.close()
