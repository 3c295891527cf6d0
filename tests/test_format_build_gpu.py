"""The format build on the GPU (tc_read_mtx_device): the host parse plus a
device radix sort by row must give readMtx's CSR byte for byte -- the same
row pointers, the same file order within each row (a symmetric file's
mirrors where readMtx puts them) and the same values -- on every golden file
(pinned to the reference's own readMtx) and on large shuffled files against
the host build (tc_read_mtx, itself pinned to the reference)."""
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
pytestmark = pytest.mark.gpu


def test_device_build_matches_reference(tc, dev, golden):
    for name, rec in golden["mtx"].items():
        path = os.path.join(GOLD, "mtx", name)
        if rec["rc"] != 0:
            with pytest.raises(tc.TcError) as e:
                tc.read_mtx_device(path)
            assert "reference code %d" % rec["rc"] in str(e.value), name
            continue
        (M, N, rp, col, val), _ = tc.read_mtx_device(path)
        assert (M, N) == (rec["M"], rec["N"]), name
        assert rp.cpu().tolist() == rec["rowptr"] and col.cpu().tolist() == rec["col"], name
        np.testing.assert_array_equal(val.cpu().numpy(), np.array(rec["val"], np.float32), err_msg=name)


def write_shuffled(path, M, N, rows, cols, vals, symmetric, seed):
    """A coordinate file whose entries are in random order (so the row order
    of the CSR is decided by the file order alone)."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(len(rows))
    with open(path, "w") as f:
        f.write("%%%%MatrixMarket matrix coordinate real %s\n" % ("symmetric" if symmetric else "general"))
        f.write("%d %d %d\n" % (M, N, len(rows)))
        np.savetxt(f, np.stack([rows[perm] + 1, cols[perm] + 1, vals[perm]], 1), fmt="%d %d %.9g")


@pytest.mark.parametrize("symmetric", [False, True])
def test_device_build_large_shuffled(tc, dev, tmp_path, symmetric):
    rng = np.random.default_rng(4 + symmetric)
    M = N = 300000
    n = 2_500_000
    rows = rng.integers(0, M, n)
    cols = np.clip(rows + rng.integers(-50, 51, n), 0, N - 1)
    cols[::7] = rng.integers(0, N, len(cols[::7]))          # some far columns
    if symmetric:                                           # lower triangle, diagonal included
        rows, cols = np.maximum(rows, cols), np.minimum(rows, cols)
    vals = rng.uniform(-10, 10, n)
    path = str(tmp_path / "big.mtx")
    write_shuffled(path, M, N, rows, cols, vals, symmetric, seed=9)
    M1, N1, rp, col, val = tc.read_mtx(path)                # host build
    (M2, N2, rp2, col2, val2), (parse_ms, build_ms) = tc.read_mtx_device(path)
    assert (M1, N1) == (M2, N2)
    np.testing.assert_array_equal(rp2.cpu().numpy(), rp)
    np.testing.assert_array_equal(col2.cpu().numpy(), col)
    np.testing.assert_array_equal(val2.cpu().numpy(), val)
    if symmetric:
        assert rp[-1] > n                                   # mirrors were added
    print("%s: %d entries -> %d; host parse %.1f ms, device build %.1f ms" % (
        "symmetric" if symmetric else "general", n, rp[-1], parse_ms, build_ms))


def test_device_build_feeds_plan(tc, dev, tmp_path):
    """The device CSR goes straight into a plan (on_device = 1): the GPU
    partition then multiplies correctly (x = 1 gives the row lengths)."""
    import torch
    from taichi_b200 import matgen
    M, N, rp, col = matgen.segments(60000, [(0, 60000, 0, 2, 0.97)], noise=3000, seed=6)
    path = str(tmp_path / "band.mtx")
    matgen.to_mtx(path, M, N, rp, col)
    (M2, N2, drp, dcol, dval), _ = tc.read_mtx_device(path)
    plan = tc.Plan.from_csr(M2, N2, drp, dcol, val=dval, on_device=True)
    assert plan.info()["dia_shapes"] >= 1
    y = torch.empty(M, device=dev)
    plan.spmv(torch.ones(N, device=dev), y)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(y.cpu().numpy(), np.diff(rp).astype(np.float32))
    plan.close()
