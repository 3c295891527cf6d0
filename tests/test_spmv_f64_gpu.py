"""Parity of the double-precision multiply (tc_spmv_f64) with the oracle's
FP64 CSR loop, through the C ABI, on the same plans as the FP32 tests.

Bar: bit-exact y for integer-valued x (every partial sum is an exact double);
for x uniform in [-1, 1], normwise relative error <= 1e-12 against the
oracle (the two sum a row's terms in different orders)."""
import numpy as np
import pytest

import oracle
from tests.golden import cases
from taichi_b200 import matgen

pytestmark = pytest.mark.gpu
TOL64 = 1e-12


def run_f64(plan, x, M, dev):
    import torch
    xd = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).to(dev)
    y = torch.full((M,), float("nan"), dtype=torch.float64, device=dev)
    plan.spmv_f64(xd, y)
    torch.cuda.synchronize()
    return y.cpu().numpy()


def check_f64(plan, M, N, rp, col, dev, label):
    rng = np.random.default_rng(17)
    xi = rng.integers(-8, 9, N).astype(np.float64)
    np.testing.assert_array_equal(run_f64(plan, xi, M, dev), oracle.spmv_csr_f64(M, rp, col, xi),
                                  err_msg=label + " integer x")
    xf = rng.uniform(-1, 1, N)
    y = run_f64(plan, xf, M, dev)
    want = oracle.spmv_csr_f64(M, rp, col, xf)
    nrm = np.linalg.norm(want)
    rel = np.linalg.norm(y - want) / nrm if nrm > 0 else np.linalg.norm(y)
    print("%s: FP64 normwise rel err %.2e" % (label, rel))
    assert rel <= TOL64, (label, rel)


F64_CASES = [c for c in cases.MATRIX_CASES
             if c["name"] in ("band_holes", "multi_shape", "many_shapes", "overlap", "rect_cols",
                              "cfg1_small", "rmat16_selfloops", "tiny_no_thumb")]


@pytest.mark.parametrize("mode", [0, 1, 2], ids=["merge", "lanes", "stream"])
@pytest.mark.parametrize("case", F64_CASES, ids=[c["name"] for c in F64_CASES])
def test_spmv_f64_oracle(tc, dev, case, mode):
    """Hybrid plans (dense diagonals + signed CSR) and their plain CSR twins,
    in every tile mode."""
    M, N, rp, col = cases.matrix(case)
    for partition in (True, False):
        plan = tc.Plan.from_csr(M, N, rp, col, prm=tc.params(tile_mode=mode), partition=partition)
        check_f64(plan, M, N, rp, col, dev, "%s/mode%d/%s" % (case["name"], mode, "hybrid" if partition else "plain"))
        plan.close()


def test_spmv_f64_long_and_lane_rows(tc, dev):
    """Rows long enough for a whole CTA, rows for a warp, empty rows."""
    rng = np.random.default_rng(5)
    lengths = np.concatenate([np.zeros(100, int), rng.integers(0, 3, 2000), [9000, 0, 20000],
                              rng.integers(30, 200, 60), rng.integers(0, 12, 3000)])
    M, N = len(lengths), 7000
    rp = np.zeros(M + 1, np.int64)
    np.cumsum(lengths, out=rp[1:])
    rp = rp.astype(np.int32)
    col = rng.integers(0, N, int(rp[-1])).astype(np.int32)
    for mode in (0, 1, 2):
        plan = tc.Plan.from_csr(M, N, rp, col, prm=tc.params(tile_mode=mode, tile_nnz=2048), partition=False)
        check_f64(plan, M, N, rp, col, dev, "long/mode%d" % mode)
        plan.close()


def test_spmv_f64_wide_and_mesh(tc, dev):
    """A wide-direct R-MAT plan and a stream-tile mesh plan, both hybrid."""
    for name, (M, N, rp, col) in (("rmat16_selfloops", matgen.rmat(16, 16, 0.499, 0.001, 0.001, seed=3,
                                                                    self_loops=True)),
                                  ("mesh256", matgen.mesh9(grid=256, permute_frac=0.02, seed=5))):
        plan = tc.Plan.from_csr(M, N, rp, col)
        check_f64(plan, M, N, rp, col, dev, name)
        plan.close()


def test_spmv_f64_matches_f32_on_integers(tc, dev):
    """FP32 and FP64 multiplies of one plan agree exactly where both are exact."""
    import torch
    M, N, rp, col = matgen.mesh9(grid=128, permute_frac=0.02, seed=8)
    plan = tc.Plan.from_csr(M, N, rp, col)
    x = np.random.default_rng(2).integers(-8, 9, N)
    y32 = torch.empty(M, dtype=torch.float32, device=dev)
    plan.spmv(torch.from_numpy(x.astype(np.float32)).to(dev), y32)
    y64 = run_f64(plan, x.astype(np.float64), M, dev)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(y32.cpu().numpy().astype(np.float64), y64)
    plan.close()
