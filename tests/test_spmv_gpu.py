"""Parity of the CUDA multiply with the oracle (FP64 CPU), through the C ABI.

Bar: bit-exact y for integer-valued x in [-8, 8]; for FP32 x uniform in
[-1, 1], normwise relative error <= 1e-5 against FP64 and, per row,
|y - y64| <= 1e-5 * (sum of |terms| the row adds, holes counted twice)."""
import numpy as np
import pytest

import oracle
from tests.golden import cases
from taichi_b200 import matgen

pytestmark = pytest.mark.gpu
TOL = 1e-5


def to_dev(a, dev):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def run_spmv(plan, x, M, dev):
    import torch
    xd = to_dev(x.astype(np.float32), dev)
    y = torch.full((M,), float("nan"), dtype=torch.float32, device=dev)
    plan.spmv(xd, y)
    torch.cuda.synchronize()
    plan.check()
    return y.cpu().numpy()


def abs_terms(fmt, M, N, rp, col, x):
    """Sum of |terms| a row of the format adds: the pattern plus the holes
    twice (once on the dense diagonal, once subtracted)."""
    a = oracle.spmv_csr_f64(M, rp, col, np.abs(x))
    if fmt["dense_nnz"] > 0 and len(fmt["csrCol"]):
        cc = fmt["csrCol"]
        holes = (cc & 1) == 0
        rows = np.repeat(np.arange(M), np.diff(fmt["csrRow"]))
        a += 2 * np.bincount(rows[holes], weights=np.abs(x[cc[holes] >> 1]), minlength=M)
    return a


def check_plan(plan, fmt, M, N, rp, col, dev, label):
    rng = np.random.default_rng(7)
    # integer x: every partial sum is an exact float
    xi = rng.integers(-8, 9, N).astype(np.float64)
    yi = run_spmv(plan, xi, M, dev)
    want = oracle.spmv_csr_f64(M, rp, col, xi)
    np.testing.assert_array_equal(yi.astype(np.float64), want, err_msg=label + " integer x")
    # x == 1 (the reference's own check, main.cu:53-86): y = row lengths
    y1 = run_spmv(plan, np.ones(N), M, dev)
    np.testing.assert_array_equal(y1, np.diff(rp).astype(np.float32), err_msg=label + " x=1")
    # random FP32 x
    xf = rng.uniform(-1, 1, N).astype(np.float32)
    yf = run_spmv(plan, xf, M, dev).astype(np.float64)
    y64 = oracle.spmv_csr_f64(M, rp, col, xf.astype(np.float64))
    nrm = np.linalg.norm(y64)
    rel = np.linalg.norm(yf - y64) / nrm if nrm > 0 else np.linalg.norm(yf)
    bound = abs_terms(fmt, M, N, rp, col, xf.astype(np.float64))
    roww = np.max(np.abs(yf - y64) / np.maximum(bound, 1e-30)) if M else 0.0
    print("%s: normwise rel err %.2e, max row-wise err %.2e" % (label, rel, roww))
    assert rel <= TOL and roww <= TOL, (label, rel, roww)


PARTITION_CASES = [c for c in cases.MATRIX_CASES if c["name"] not in ("mesh2048",)]


@pytest.mark.parametrize("case", PARTITION_CASES, ids=[c["name"] for c in PARTITION_CASES])
def test_spmv_oracle_format(tc, dev, case):
    """Plans built from the oracle's partition (pinned to the reference)."""
    M, N, rp, col = cases.matrix(case)
    fmt, _ = oracle.partition(M, N, rp, col)
    plan = tc.Plan.from_format(M, N, fmt)
    check_plan(plan, fmt, M, N, rp, col, dev, case["name"])
    plan.close()


@pytest.mark.parametrize("case", PARTITION_CASES[:8], ids=[c["name"] for c in PARTITION_CASES[:8]])
def test_spmv_plain_csr(tc, dev, case):
    M, N, rp, col = cases.matrix(case)
    plan = tc.Plan.from_csr(M, N, rp, col, partition=False)
    fmt = dict(dense_nnz=0, csrRow=rp, csrCol=col)
    check_plan(plan, fmt, M, N, rp, col, dev, case["name"] + "/plain")
    plan.close()


def csr_from_lengths(lengths, N, seed):
    rng = np.random.default_rng(seed)
    rp = np.zeros(len(lengths) + 1, np.int64)
    np.cumsum(lengths, out=rp[1:])
    col = rng.integers(0, N, int(rp[-1])).astype(np.int32)
    return rp.astype(np.int32), col


@pytest.mark.parametrize("tile", [(1024, 4096), (1, 1), (3, 7), (2040, 8192), (64, 100)])
def test_tile_kinds_and_edges(tc, dev, tile):
    """Empty rows, long rows (CTA per row), medium rows (warp per row),
    duplicates, and extreme tile limits."""
    rng = np.random.default_rng(11)
    lengths = np.concatenate([np.zeros(300, int), rng.integers(0, 3, 2000), [5000, 0, 9000],
                              rng.integers(30, 200, 50), [1], np.zeros(5, int), [70000],
                              rng.integers(0, 12, 3000)])
    M, N = len(lengths), 7000
    rp, col = csr_from_lengths(lengths, N, 3)
    prm = tc.params(tile_rows=tile[0], tile_nnz=tile[1])
    plan = tc.Plan.from_csr(M, N, rp, col, prm=prm, partition=False)
    info = plan.info()
    assert info["ntiles_long"] >= 1 if tile[1] < 9000 else True
    check_plan(plan, dict(dense_nnz=0), M, N, rp, col, dev, "edges%s" % (tile,))


MODE_CASES = [c for c in PARTITION_CASES if c["name"] in
              ("band_holes", "multi_shape", "many_shapes", "rmat16_selfloops", "overlap")]


@pytest.mark.parametrize("mode", [0, 1, 2], ids=["merge", "lanes", "stream"])
@pytest.mark.parametrize("case", MODE_CASES, ids=[c["name"] for c in MODE_CASES])
def test_tile_modes(tc, dev, case, mode):
    """Every tile mode against the oracle, hybrid and plain plans."""
    M, N, rp, col = cases.matrix(case)
    fmt, _ = oracle.partition(M, N, rp, col)
    plan = tc.Plan.from_format(M, N, fmt, prm=tc.params(tile_mode=mode))
    check_plan(plan, fmt, M, N, rp, col, dev, "%s/mode%d" % (case["name"], mode))
    plan.close()
    plan = tc.Plan.from_csr(M, N, rp, col, prm=tc.params(tile_mode=mode), partition=False)
    check_plan(plan, dict(dense_nnz=0), M, N, rp, col, dev, "%s/plain/mode%d" % (case["name"], mode))
    plan.close()


@pytest.mark.parametrize("tile", [(1024, 4096), (1, 1), (3, 7), (2040, 8192), (64, 100), (1024, 2048)])
def test_stream_tiles_edges(tc, dev, tile):
    """Stream tiles next to lane and long tiles, unaligned tile starts, empty
    rows, and the tile caps at their extremes."""
    rng = np.random.default_rng(12)
    lengths = np.concatenate([np.zeros(301, int), rng.integers(0, 3, 2003), [5000, 0, 9000],
                              rng.integers(30, 200, 50), [1], np.zeros(5, int), [127, 128, 129],
                              rng.integers(0, 12, 3001), [70000], rng.integers(0, 2, 5000)])
    M, N = len(lengths), 7001
    rp, col = csr_from_lengths(lengths, N, 5)
    prm = tc.params(tile_rows=tile[0], tile_nnz=tile[1], tile_mode=2)
    plan = tc.Plan.from_csr(M, N, rp, col, prm=prm, partition=False)
    check_plan(plan, dict(dense_nnz=0), M, N, rp, col, dev, "stream%s" % (tile,))
    plan.close()


def test_stream_matches_sequential_rows(tc, dev):
    """Stream and direct tiles add a row's terms in the order of one-lane
    tiles, so all give bit-identical FP32 y when every row is short."""
    for name in ("band_holes", "rmat16_selfloops"):
        case = next(c for c in cases.MATRIX_CASES if c["name"] == name)
        M, N, rp, col = cases.matrix(case)
        assert np.diff(rp).max() <= 128
        fmt, _ = oracle.partition(M, N, rp, col)
        x = np.random.default_rng(9).uniform(-1, 1, N).astype(np.float32)
        ys = []
        for mode, flags in ((1, 0), (2, 0), (2, tc.TC_FLAG_NO_WIDE), (2, tc.TC_FLAG_NO_DIRECT),
                            (2, tc.TC_FLAG_ROWS_STRIDED)):
            plan = tc.Plan.from_format(M, N, fmt, prm=tc.params(tile_mode=mode, max_lanes=1, flags=flags))
            ys.append(run_spmv(plan, x, M, dev))
            plan.close()
        for k in range(1, len(ys)):
            np.testing.assert_array_equal(ys[0], ys[k], err_msg="%s variant %d" % (name, k))


@pytest.mark.parametrize("M", [4096, 10001, 3 * 4096 + 4])
def test_wide_direct_tiles(tc, dev, M):
    """A matrix whose rows all average at most one entry runs as wide direct
    tiles (one 1024-thread CTA per 4096 rows): partial last tile and last run,
    against the oracle; and the same y as 256-thread direct tiles."""
    import torch
    rng = np.random.default_rng(M)
    lengths = rng.integers(0, 2, M)
    lengths[rng.integers(0, M, 20)] = rng.integers(2, 60, 20)      # a few longer rows
    N = M + 7
    rp, col = csr_from_lengths(lengths, N, 9)
    assert rp[-1] <= M
    plan = tc.Plan.from_csr(M, N, rp, col, prm=tc.params(flags=tc.TC_FLAG_WIDE_FIXED), partition=False)
    assert plan.info()["ntiles"] == (M + 4095) // 4096              # wide tiles
    check_plan(plan, dict(dense_nnz=0), M, N, rp, col, dev, "wide/M%d" % M)
    x = rng.uniform(-1, 1, N).astype(np.float32)
    y_wide = run_spmv(plan, x, M, dev)
    plan.close()
    plan = tc.Plan.from_csr(M, N, rp, col, prm=tc.params(flags=tc.TC_FLAG_NO_WIDE), partition=False)
    np.testing.assert_array_equal(run_spmv(plan, x, M, dev), y_wide)
    plan.close()


def test_direct_tiles(tc, dev):
    """Direct tiles (rows averaging at most one entry) next to stream, lane
    and long tiles, with an unaligned tail, against the oracle, with and
    without direct tiles."""
    rng = np.random.default_rng(21)
    lengths = np.concatenate([rng.integers(0, 2, 5003), rng.integers(0, 12, 2000), [300, 0, 7],
                              rng.integers(0, 3, 4097), rng.integers(5, 9, 900), rng.integers(0, 2, 2051)])
    M, N = len(lengths), 9000
    rp, col = csr_from_lengths(lengths, N, 8)
    for rows, flags in ((1024, 0), (2048, 0), (1024, tc.TC_FLAG_NO_DIRECT)):
        prm = tc.params(tile_mode=2, tile_rows=rows, flags=flags)
        plan = tc.Plan.from_csr(M, N, rp, col, prm=prm, partition=False)
        check_plan(plan, dict(dense_nnz=0), M, N, rp, col, dev, "direct/rows%d/flags%d" % (rows, flags))
        plan.close()


def test_empty_and_tiny(tc, dev):
    import torch
    # no non-zeros at all
    M, N = 1000, 500
    rp = np.zeros(M + 1, np.int32)
    plan = tc.Plan.from_csr(M, N, rp, np.zeros(0, np.int32), partition=False)
    assert not run_spmv(plan, np.ones(N), M, dev).any()
    # one row, one column
    plan = tc.Plan.from_csr(1, 1, np.array([0, 1], np.int32), np.array([0], np.int32),
                            partition=False)
    assert run_spmv(plan, np.array([3.0]), 1, dev)[0] == 3.0
    # M == 0
    plan = tc.Plan.from_csr(0, 5, np.zeros(1, np.int32), np.zeros(0, np.int32), partition=False)
    plan.spmv(torch.ones(5, device=dev), torch.empty(0, device=dev))
    # N == 0: no terms, y = 0, and x is never read
    plan = tc.Plan.from_csr(10, 0, np.zeros(11, np.int32), np.zeros(0, np.int32), partition=False)
    y = torch.full((10,), float("nan"), device=dev)
    plan.spmv(torch.empty(0, device=dev), y)
    torch.cuda.synchronize()
    assert not y.cpu().numpy().any()


def test_hybrid_without_csr_remainder(tc, dev):
    """All non-zeros on hole-free dense diagonals, so the CSR remainder is
    empty: the reference leaves csrRow unallocated and its kernel reads an
    invalid pointer (TaiChi.cu:579, 1362); here y is the diagonal sums."""
    case = next(c for c in cases.MATRIX_CASES if c["name"] == "multi_shape")
    M, N, rp, col = cases.matrix(case)
    fmt, _ = oracle.partition(M, N, rp, col)
    assert fmt["dia_shapes"] == 3
    diag_only = dict(fmt, zero_elements=0, sparse_nnz=0, csrRow=np.zeros(M + 1, np.int32),
                     csrCol=np.zeros(0, np.int32))
    plan = tc.Plan.from_format(M, N, diag_only)
    x = np.random.default_rng(4).integers(-8, 9, N).astype(np.float64)
    y = run_spmv(plan, x, M, dev)
    want = oracle.spmv_format_f64(diag_only, M, N, x)
    assert np.abs(want).sum() > 0
    np.testing.assert_array_equal(y.astype(np.float64), want)


def test_spmv_host_e2e(tc, dev):
    M, N, rp, col = cases.matrix(cases.MATRIX_CASES[1])
    fmt, _ = oracle.partition(M, N, rp, col)
    plan = tc.Plan.from_format(M, N, fmt)
    x = np.random.default_rng(2).integers(-8, 9, N).astype(np.float32)
    y = np.zeros(M, np.float32)
    plan.spmv_host(x, y)
    np.testing.assert_array_equal(y.astype(np.float64), oracle.spmv_csr_f64(M, rp, col, x.astype(np.float64)))


@pytest.mark.parametrize("slots", [2, 4])
def test_spmv_host_async_slots(tc, dev, slots):
    """Pipelined host multiplies: twelve requests rotate over 2 or 4 staging
    slots on as many streams; each y equals the oracle's (integer x:
    exact).  A slot outside [0, 4) is refused."""
    import torch
    M, N, rp, col = cases.matrix(cases.MATRIX_CASES[1])
    plan = tc.Plan.from_csr(M, N, rp, col)
    rng = np.random.default_rng(5)
    n = 12
    xs = [torch.from_numpy(rng.integers(-8, 9, N).astype(np.float32)).pin_memory() for _ in range(n)]
    ys = [torch.full((M,), float("nan")).pin_memory() for _ in range(n)]
    streams = [torch.cuda.Stream(dev) for _ in range(slots)]
    for i in range(n):
        plan.spmv_host_async(xs[i], ys[i], i % slots, streams[i % slots])
    for s in streams:
        s.synchronize()
    plan.check()
    for i in range(n):
        want = oracle.spmv_csr_f64(M, rp, col, xs[i].numpy().astype(np.float64))
        np.testing.assert_array_equal(ys[i].numpy().astype(np.float64), want, err_msg="request %d" % i)
    with pytest.raises(tc.TcError):
        plan.spmv_host_async(xs[0], ys[0], 4, streams[0])
    with pytest.raises(tc.TcError):
        plan.spmv_host_async(xs[0], ys[0], -1, streams[0])
    plan.close()


MAPPED_CASES = [("rmat20", {}), ("cfg1_small", {}), ("cfg1_small", {"flags": 0x80}),
                ("band_holes", {"tile_mode": 0}), ("band_holes", {"tile_mode": 1}),
                ("multi_shape", {}), ("rect_cols", {}), ("rmat16_selfloops", {})]


@pytest.mark.parametrize("name,over", MAPPED_CASES,
                         ids=["%s-%s" % (n, "-".join("%s%s" % kv for kv in o.items()) or "default")
                              for n, o in MAPPED_CASES])
def test_spmv_host_mapped_y(tc, dev, name, over):
    """TC_FLAG_HOST_Y_MAPPED: the multiply stores y straight into a pinned
    host buffer.  For each kernel kind, y is bit-identical to the device
    multiply of the same plan and, for integer x, to the oracle -- through
    tc_spmv_host and tc_spmv_host_async on two slots, into an aligned pinned
    buffer, a pinned buffer one float off 16-byte alignment, and pageable
    memory (which takes the copy)."""
    import torch
    case = next(c for c in cases.MATRIX_CASES if c["name"] == name)
    M, N, rp, col = cases.matrix(case)
    over = dict(over)
    over["flags"] = over.get("flags", 0) | tc.TC_FLAG_HOST_Y_MAPPED
    plan = tc.Plan.from_csr(M, N, rp, col, prm=tc.params(**over))
    rng = np.random.default_rng(11)
    xi = rng.integers(-8, 9, N).astype(np.float32)
    xf = rng.uniform(-1, 1, N).astype(np.float32)
    want_i = oracle.spmv_csr_f64(M, rp, col, xi.astype(np.float64))
    dev_f = run_spmv(plan, xf, M, dev)
    # the device multiply into a y one float off 16-byte alignment: the
    # kernel path an unaligned host y takes
    yoff = torch.full((M + 1,), float("nan"), device=dev)
    plan.spmv(to_dev(xf, dev), yoff[1:])
    torch.cuda.synchronize()
    dev_f_off = yoff[1:].cpu().numpy()
    for x, want, label in ((xi, want_i, "integer x"), (xf, None, "fp32 x")):
        hx = torch.from_numpy(x).pin_memory()
        pinned = torch.full((M + 1,), float("nan")).pin_memory()
        targets = {"pinned": torch.full((M,), float("nan")).pin_memory(), "pinned+1": pinned[1:],
                   "pageable": np.full(M, np.nan, np.float32)}
        for tname, hy in targets.items():
            plan.spmv_host(hx, hy)
            got = hy.numpy() if hasattr(hy, "numpy") else hy
            if want is not None:
                np.testing.assert_array_equal(got.astype(np.float64), want, err_msg="%s %s %s" % (name, label, tname))
            else:
                np.testing.assert_array_equal(got, dev_f_off if tname == "pinned+1" else dev_f,
                                              err_msg="%s %s %s" % (name, label, tname))
        ys = [torch.full((M,), float("nan")).pin_memory() for _ in range(4)]
        streams = [torch.cuda.Stream(dev) for _ in range(2)]
        for i in range(4):
            plan.spmv_host_async(hx, ys[i], i % 2, streams[i % 2])
        for s in streams:
            s.synchronize()
        plan.check()
        for i in range(4):
            if want is not None:
                np.testing.assert_array_equal(ys[i].numpy().astype(np.float64), want, err_msg="%s async %d" % (name, i))
            else:
                np.testing.assert_array_equal(ys[i].numpy(), dev_f, err_msg="%s async %d" % (name, i))
    plan.close()


def test_spmv_host_mapped_y_no_columns(tc, dev):
    """A plan with rows but no columns keeps the copy under
    TC_FLAG_HOST_Y_MAPPED: y = 0 in a pinned buffer."""
    import torch
    rp = np.zeros(9, np.int32)
    plan = tc.Plan.from_csr(8, 0, rp, np.zeros(0, np.int32),
                            prm=tc.params(flags=tc.TC_FLAG_HOST_Y_MAPPED), partition=False)
    hy = torch.full((8,), float("nan")).pin_memory()
    plan.spmv_host(np.zeros(1, np.float32), hy)
    np.testing.assert_array_equal(hy.numpy(), np.zeros(8, np.float32))
    plan.close()


def test_format_rejected(tc):
    M, N = 10, 10
    rp = np.array([0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10], np.int32)
    bad = dict(dia_shapes=0, num_negs=0, dense_nnz=0, zero_elements=0, sparse_nnz=10,
               row_start=0, row_stop=0, csrRow=rp, csrCol=np.full(10, 12, np.int32))
    with pytest.raises(tc.TcError):
        tc.Plan.from_format(M, N, bad)


@pytest.mark.parametrize("name,mode", [("rmat16", 2), ("rmat16", 0), ("rmat16", 1), ("rmat20", 2),
                                       ("rmat16_selfloops", 2), ("mesh128", 2), ("mesh128", 1),
                                       ("mesh512", 2)])
def test_chained_multiplies(tc, dev, name, mode):
    """Six multiplies back to back on one stream, each reading the vector the
    one before wrote (v <- A v, as a power iteration does): the launches
    overlap under programmatic dependent launch, and every gather must still
    see its producer's writes.  Integer x keeps every value exact."""
    import torch
    if name.startswith("rmat"):
        M, N, rp, col = matgen.rmat(int(name[4:6]), 16, 0.499, 0.001, 0.001, seed=3,
                                    self_loops=name.endswith("selfloops"))
    else:
        M, N, rp, col = matgen.mesh9(grid=int(name[4:]), permute_frac=0.02, seed=5)
    assert M == N
    plan = tc.Plan.from_csr(M, N, rp, col, prm=tc.params(tile_mode=mode))
    v0 = np.random.default_rng(11).integers(-2, 3, N).astype(np.float64)
    bufs = [to_dev(v0.astype(np.float32), dev), torch.empty(N, dtype=torch.float32, device=dev)]
    want = v0
    for k in range(6):
        plan.spmv(bufs[k & 1], bufs[(k + 1) & 1])
        want = oracle.spmv_csr_f64(M, rp, col, want)
    assert np.abs(want).max() < 2 ** 24
    torch.cuda.synchronize()
    plan.check()
    np.testing.assert_array_equal(bufs[0].cpu().numpy().astype(np.float64), want)
    plan.close()


def test_stream_kernel_many_tiles(tc, dev):
    """Plans of stream tiles only, with more tiles than one wave at six CTAs
    per SM, run the 8-CTA stream kernel: the hybrid plan (signed words) and
    the plain CSR plan of the same mesh, both against the oracle (the rows
    kernel, the default for such short rows, turned off)."""
    import torch
    M, N, rp, col = matgen.mesh9(grid=512, permute_frac=0.02, seed=9)
    no_window = tc.params(flags=tc.TC_FLAG_NO_WINDOW | tc.TC_FLAG_NO_ROWS)
    plan = tc.Plan.from_csr(M, N, rp, col, prm=no_window)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    assert plan.info()["ntiles"] > 6 * sms and plan.info()["nwtiles"] == 0
    assert tc.KERNEL_NAMES[plan.info()["kernel"]] == "stream"
    check_plan(plan, plan.export(), M, N, rp, col, dev, "stream/many")
    x = np.random.default_rng(3).uniform(-1, 1, N).astype(np.float32)
    y_many = run_spmv(plan, x, M, dev)
    plan.close()
    plan = tc.Plan.from_csr(M, N, rp, col, prm=no_window, partition=False)
    assert tc.KERNEL_NAMES[plan.info()["kernel"]] == "stream"
    y_plain = run_spmv(plan, x, M, dev)
    plan.close()
    y64 = oracle.spmv_csr_f64(M, rp, col, x.astype(np.float64))
    assert np.linalg.norm(y_many - y64) <= TOL * np.linalg.norm(y64)
    assert np.linalg.norm(y_plain - y64) <= TOL * np.linalg.norm(y64)


def test_spmv_mesh2048_full_size(tc, dev):
    """The 9-point stencil on a 2048 x 2048 grid with 2% of its rows permuted
    (37.7 M non-zeros, the one plain configuration larger than L2), formatted
    by the GPU partitioner (whose format equals the reference's for this
    matrix, see test_partition_gpu): integer x exact, x = 1, FP32 x within
    1e-5 of FP64 normwise and per row.  The window plan of the same format
    gives the same y bit for bit."""
    case = next(c for c in cases.MATRIX_CASES if c["name"] == "mesh2048")
    M, N, rp, col = cases.matrix(case)
    plan = tc.Plan.from_csr(M, N, rp, col)
    info = plan.info()
    assert info["dia_shapes"] == 1 and info["nwtiles"] == 0, info
    assert tc.KERNEL_NAMES[info["kernel"]] == "rows", info        # short rows: the rows kernel
    fmt = plan.export()
    check_plan(plan, fmt, M, N, rp, col, dev, "mesh2048/default")
    x = np.random.default_rng(17).uniform(-1, 1, N).astype(np.float32)
    y_stream = run_spmv(plan, x, M, dev)
    plan.close()
    plan = tc.Plan.from_format(M, N, fmt, prm=tc.params(flags=tc.TC_FLAG_WINDOW))
    assert plan.info()["nwtiles"] > 0
    check_plan(plan, fmt, M, N, rp, col, dev, "mesh2048/window")
    np.testing.assert_array_equal(run_spmv(plan, x, M, dev), y_stream)
    plan.close()
    for flags, kernel in ((tc.TC_FLAG_ROWS, "rows"), (tc.TC_FLAG_ROWS | tc.TC_FLAG_NO_PREFETCH, "rows"),
                          (tc.TC_FLAG_NO_ROWS, "stream")):
        plan = tc.Plan.from_format(M, N, fmt, prm=tc.params(flags=flags))
        assert tc.KERNEL_NAMES[plan.info()["kernel"]] == kernel
        check_plan(plan, fmt, M, N, rp, col, dev, "mesh2048/%s/%#x" % (kernel, flags))
        np.testing.assert_array_equal(run_spmv(plan, x, M, dev), y_stream)
        plan.close()


@pytest.mark.parametrize("w", [4, 6, 8])
@pytest.mark.parametrize("case", PARTITION_CASES, ids=[c["name"] for c in PARTITION_CASES])
def test_rows_kernel(tc, dev, case, w):
    """The rows kernel (one row per thread, words straight from global
    memory) on every matrix whose rows all fit a stream tile -- no shape,
    one shape of one or several offsets, several shapes (the per-row shape
    search), plain and hybrid words: against the oracle, and bit-identical to
    the stream-tile kernel on the same format (same terms, same order)."""
    M, N, rp, col = cases.matrix(case)
    fmt, _ = oracle.partition(M, N, rp, col)
    if np.diff(fmt["csrRow"]).max(initial=0) > 128:
        pytest.skip("rows longer than a stream tile takes")
    base = tc.TC_FLAG_NO_DIRECT | tc.TC_FLAG_NO_WIDE | tc.TC_FLAG_ROWS_STRIDED | tc.TC_FLAG_NO_WINDOW
    plan = tc.Plan.from_format(M, N, fmt, prm=tc.params(flags=base | tc.TC_FLAG_ROWS, rows_w=w))
    assert tc.KERNEL_NAMES[plan.info()["kernel"]] == "rows", plan.info()
    label = "%s/rows_w%d" % (case["name"], w)
    check_plan(plan, fmt, M, N, rp, col, dev, label)
    x = np.random.default_rng(6).uniform(-1, 1, N).astype(np.float32)
    y_rows = run_spmv(plan, x, M, dev)
    plan.close()
    plan = tc.Plan.from_format(M, N, fmt, prm=tc.params(flags=base | tc.TC_FLAG_NO_ROWS))
    assert tc.KERNEL_NAMES[plan.info()["kernel"]] == "stream", plan.info()
    np.testing.assert_array_equal(run_spmv(plan, x, M, dev), y_rows, err_msg=label)
    plan.close()


def test_rows_kernel_unaligned_and_chained(tc, dev):
    """x and y at odd addresses, and chained multiplies v <- A v under
    programmatic dependent launch (x of each multiply is the y of the one
    before): the rows kernel reads x only after the wait."""
    import torch
    M, N, rp, col = matgen.mesh9(grid=512, permute_frac=0.02, seed=9)
    plan = tc.Plan.from_csr(M, N, rp, col, prm=tc.params(flags=tc.TC_FLAG_ROWS))
    assert tc.KERNEL_NAMES[plan.info()["kernel"]] == "rows"
    x = np.random.default_rng(8).integers(-8, 9, N).astype(np.float32)
    xb = torch.zeros(N + 1, dtype=torch.float32, device=dev)
    xb[1:] = to_dev(x, dev)
    yb = torch.full((M + 1,), float("nan"), dtype=torch.float32, device=dev)
    plan.spmv(xb[1:].data_ptr(), yb[1:].data_ptr())
    torch.cuda.synchronize()
    want = oracle.spmv_csr_f64(M, rp, col, x.astype(np.float64))
    np.testing.assert_array_equal(yb[1:].cpu().numpy().astype(np.float64), want)
    # chained: integers stay exact for 3 steps (|v| grows at most 9x a step)
    v = [to_dev(np.sign(x), dev)] + [torch.empty(M, device=dev) for _ in range(3)]
    for k in range(3):
        plan.spmv(v[k], v[k + 1])
    torch.cuda.synchronize()
    w = np.sign(x).astype(np.float64)
    for k in range(3):
        w = oracle.spmv_csr_f64(M, rp, col, w)
        np.testing.assert_array_equal(v[k + 1].cpu().numpy().astype(np.float64), w, err_msg="step %d" % k)
    plan.close()


WINDOW_CASES = [c for c in PARTITION_CASES if c["name"] in
                ("band_holes", "two_segments", "offdiag_blocks", "wide_band", "overlap", "rect_cols",
                 "multi_shape", "many_shapes", "cfg1_small", "rmat16_selfloops")]


@pytest.mark.parametrize("rows", [1024, 100, 7])
@pytest.mark.parametrize("case", WINDOW_CASES, ids=[c["name"] for c in WINDOW_CASES])
def test_window_plans(tc, dev, case, rows):
    """Window plans forced on every kind of matrix (one and many shapes,
    shapes off the main diagonal, rectangular, random columns, short and
    odd tile heights): against the oracle, and bit-identical to the
    stream-tile plan of the same format when every row is short enough for
    one-row-per-thread tiles (the same terms in the same order)."""
    M, N, rp, col = cases.matrix(case)
    fmt, _ = oracle.partition(M, N, rp, col)
    plan = tc.Plan.from_format(M, N, fmt, prm=tc.params(tile_rows=rows, flags=tc.TC_FLAG_WINDOW))
    assert plan.info()["nwtiles"] >= (M + rows - 1) // rows
    label = "%s/window%d" % (case["name"], rows)
    check_plan(plan, fmt, M, N, rp, col, dev, label)
    x = np.random.default_rng(5).uniform(-1, 1, N).astype(np.float32)
    y_win = run_spmv(plan, x, M, dev)
    plan.close()
    if np.diff(fmt["csrRow"]).max(initial=0) <= 128:
        plan = tc.Plan.from_format(M, N, fmt, prm=tc.params(flags=tc.TC_FLAG_NO_WINDOW))
        np.testing.assert_array_equal(run_spmv(plan, x, M, dev), y_win, err_msg=label)
        plan.close()


def test_window_unaligned_vectors(tc, dev):
    """x and y that are not 16-byte aligned: the window kernel then reads
    every term from global memory (no window copies), same y."""
    import torch
    M, N, rp, col = matgen.mesh9(grid=384, permute_frac=0.02, seed=4)
    plan = tc.Plan.from_csr(M, N, rp, col, prm=tc.params(flags=tc.TC_FLAG_WINDOW))
    assert plan.info()["nwtiles"] > 0
    x = np.random.default_rng(8).integers(-8, 9, N).astype(np.float32)
    xb = torch.zeros(N + 1, dtype=torch.float32, device=dev)
    xb[1:] = to_dev(x, dev)
    yb = torch.full((M + 1,), float("nan"), dtype=torch.float32, device=dev)
    plan.spmv(xb[1:].data_ptr(), yb[1:].data_ptr())
    torch.cuda.synchronize()
    plan.check()
    want = oracle.spmv_csr_f64(M, rp, col, x.astype(np.float64))
    np.testing.assert_array_equal(yb[1:].cpu().numpy().astype(np.float64), want)
    plan.close()


def test_window_plan_selection(tc, dev):
    """Window plans are built on request only (TC_FLAG_WINDOW; the tuner
    tries them): a mesh gets the window covering its stencil columns, a
    banded matrix a narrow one; without the flag, or with TC_FLAG_NO_WINDOW
    as well, no window plan."""
    W = tc.params(flags=tc.TC_FLAG_WINDOW)
    M, N, rp, col = matgen.mesh9(grid=512, permute_frac=0.02, seed=1)     # stencil columns r +- 511..513
    plan = tc.Plan.from_csr(M, N, rp, col, prm=W)
    i = plan.info()
    assert i["nwtiles"] > 0 and -1024 < i["window_lo"] <= -513 and 513 <= i["window_hi"] < 1024, i
    plan.close()
    plan = tc.Plan.from_csr(M, N, rp, col)
    assert plan.info()["nwtiles"] == 0
    plan.close()
    rp, col = tc.gen_banded(300000, 4, 3, seed=2)
    plan = tc.Plan.from_csr(300000, 300000, rp, col, prm=tc.params(flags=tc.TC_FLAG_WINDOW))
    i = plan.info()
    assert i["nwtiles"] > 0 and i["window_lo"] >= -64 and i["window_hi"] <= 64, i
    plan.close()
    plan = tc.Plan.from_csr(300000, 300000, rp, col,
                            prm=tc.params(flags=tc.TC_FLAG_WINDOW | tc.TC_FLAG_NO_WINDOW))
    assert plan.info()["nwtiles"] == 0
    plan.close()


def test_wide_bounds_kernel(tc, dev):
    """Whole wide tiles taking their word ranges from the launch parameters
    and staging their words in shared memory (TC_FLAG_WIDE_BOUNDS): the same
    y, bit for bit, as the kernel that reads them through the row pointers, on
    an R-MAT graph and on a matrix whose first tile holds more words than
    the shared-memory stage (the rest come from global memory); both against
    the oracle."""
    M, rp, col = tc.gen_rmat(16, 16, 0.499, 0.001, 0.001, seed=4)
    cases_ = [("rmat16", M, rp, col)]
    M2 = 16384
    lengths = np.zeros(M2, np.int64)
    lengths[:4096] = 3                      # 12,288 words in tile 0 (stage: 8,192)
    rp2, col2 = csr_from_lengths(lengths, M2, 12)
    cases_.append(("overfull", M2, rp2, col2))
    x = np.random.default_rng(6).uniform(-1, 1, M2 * 4).astype(np.float32)
    for name, M, rp, col in cases_:
        fixed = tc.TC_FLAG_WIDE_FIXED
        plan = tc.Plan.from_csr(M, M, rp, col, prm=tc.params(flags=tc.TC_FLAG_WIDE_BOUNDS | fixed), partition=False)
        assert plan.info()["ntiles"] == M // 4096
        check_plan(plan, dict(dense_nnz=0), M, M, rp, col, dev, "bounds/" + name)
        y1 = run_spmv(plan, x[:M], M, dev)
        plan.close()
        plan = tc.Plan.from_csr(M, M, rp, col, prm=tc.params(flags=fixed), partition=False)
        np.testing.assert_array_equal(run_spmv(plan, x[:M], M, dev), y1, err_msg=name)
        plan.close()


@pytest.mark.parametrize("name", ["rmat16_selfloops", "rmat20", "rmat20_selfloops"])
def test_wide_word_prefetch_forms(tc, dev, name):
    """Wide plans prefetch each tile's CSR words into L2, the range taken
    from the launch parameters (the default for at most 511 tiles), from the
    tile record (TC_FLAG_NO_PARAM_STARTS), or not at all
    (TC_FLAG_NO_PREFETCH): the same y bit for bit, exact for integer x
    against the oracle; hybrid plans of one diagonal included."""
    case = next(c for c in cases.MATRIX_CASES if c["name"] == name)
    M, N, rp, col = cases.matrix(case)
    x = np.random.default_rng(12).uniform(-1, 1, N).astype(np.float32)
    ys = []
    for flags in (0, tc.TC_FLAG_NO_PARAM_STARTS, tc.TC_FLAG_NO_PREFETCH):
        plan = tc.Plan.from_csr(M, N, rp, col, prm=tc.params(flags=flags))
        assert tc.KERNEL_NAMES[plan.info()["kernel"]] == "wide", plan.info()
        xi = np.random.default_rng(2).integers(-8, 9, N).astype(np.float64)
        np.testing.assert_array_equal(run_spmv(plan, xi, M, dev).astype(np.float64),
                                      oracle.spmv_csr_f64(M, rp, col, xi), err_msg="%s %#x" % (name, flags))
        ys.append(run_spmv(plan, x, M, dev))
        plan.close()
    for y in ys[1:]:
        np.testing.assert_array_equal(y, ys[0])


@pytest.mark.parametrize("M", [1 << 18, 300004, 10001])
def test_wide_balanced_tiles(tc, dev, M):
    """Wide tiles sized for two per SM (the default): a whole number of
    tiles, a short last tile (M a multiple of 4) and an M that is not a
    multiple of 4 -- against the oracle and bit-identical to 4096-row tiles
    (TC_FLAG_WIDE_FIXED)."""
    rng = np.random.default_rng(M)
    lengths = rng.integers(0, 2, M)
    lengths[rng.integers(0, M, 30)] = rng.integers(2, 60, 30)
    rp, col = csr_from_lengths(lengths, M, 10)
    assert rp[-1] <= M
    plan = tc.Plan.from_csr(M, M, rp, col, partition=False)
    check_plan(plan, dict(dense_nnz=0), M, M, rp, col, dev, "balanced/M%d" % M)
    x = rng.uniform(-1, 1, M).astype(np.float32)
    y_bal = run_spmv(plan, x, M, dev)
    plan.close()
    plan = tc.Plan.from_csr(M, M, rp, col, prm=tc.params(flags=tc.TC_FLAG_WIDE_FIXED), partition=False)
    np.testing.assert_array_equal(run_spmv(plan, x, M, dev), y_bal)
    plan.close()


@pytest.mark.parametrize("off,keep", [(0, 1.0), (6, 0.98), (-3, 1.0)])
def test_single_diagonal_wide_plans(tc, dev, off, keep):
    """Plans whose dense part is one diagonal (one shape, one offset; holes
    when keep < 1) and whose CSR remainder averages under one entry per row
    run the wide tiles with the diagonal's rows taken from the launch
    parameters: against the oracle (format from the reference-pinned oracle
    partition) and bit-identical to the plan without wide tiles."""
    M, N, rp, col = matgen.segments(300000, [(0, 300000, off, 0, keep)], noise=60000, seed=5)
    fmt, _ = oracle.partition(M, N, rp, col)
    assert fmt["dia_shapes"] == 1 and fmt["num_negs"] == 1, (fmt["dia_shapes"], fmt["num_negs"])
    plan = tc.Plan.from_format(M, N, fmt)
    check_plan(plan, fmt, M, N, rp, col, dev, "diag1/off%d" % off)
    x = np.random.default_rng(2).uniform(-1, 1, N).astype(np.float32)
    y_wide = run_spmv(plan, x, M, dev)
    plan.close()
    plan = tc.Plan.from_format(M, N, fmt, prm=tc.params(flags=tc.TC_FLAG_NO_WIDE))
    np.testing.assert_array_equal(run_spmv(plan, x, M, dev), y_wide)
    plan.close()


@pytest.mark.parametrize("k,r", [(12, 7), (11, 9), (15, 8)])
def test_stream_rows_multiple_of_8(tc, dev, k, r):
    """Banded rows of 32 entries (2k + 1 + r = 32; the plan's stream tiles
    then use skewed shared-memory slots) and of 39 entries (plain slots):
    against the oracle and bit-identical to one-lane tiles (TILE_L1, the
    same terms in the same order)."""
    n = 60000
    rp, col = tc.gen_banded(n, k, r, seed=3)
    plan = tc.Plan.from_csr(n, n, rp, col, partition=False)
    check_plan(plan, dict(dense_nnz=0), n, n, rp, col, dev, "band k%d r%d" % (k, r))
    x = np.random.default_rng(1).uniform(-1, 1, n).astype(np.float32)
    y = run_spmv(plan, x, n, dev)
    plan.close()
    plan = tc.Plan.from_csr(n, n, rp, col, prm=tc.params(tile_mode=1, max_lanes=1), partition=False)
    np.testing.assert_array_equal(run_spmv(plan, x, n, dev), y)
    plan.close()


@pytest.mark.parametrize("n,off,keep", [(300000, 0, 1.0), (300001, 6, 0.98), (299998, -3, 1.0)])
def test_single_diagonal_edge_path(tc, dev, n, off, keep):
    """One-diagonal wide plans on the wide kernel's edge path: x and y one
    float off 16-byte alignment, and row counts that are not a multiple of
    4.  Each y equals the oracle's for integer x and is bit-identical to the
    aligned multiply for FP32 x (the diagonal terms come from the tile
    classes there, from the launch parameters on the aligned path)."""
    import torch
    M, N, rp, col = matgen.segments(n, [(0, n, off, 0, keep)], noise=n // 5, seed=6)
    fmt, _ = oracle.partition(M, N, rp, col)
    assert fmt["dia_shapes"] == 1 and fmt["num_negs"] == 1, (fmt["dia_shapes"], fmt["num_negs"])
    plan = tc.Plan.from_format(M, N, fmt)
    rng = np.random.default_rng(3)
    xi = rng.integers(-8, 9, N).astype(np.float32)
    xf = rng.uniform(-1, 1, N).astype(np.float32)
    want = oracle.spmv_csr_f64(M, rp, col, xi.astype(np.float64))
    y_aligned = run_spmv(plan, xf, M, dev)
    for xshift, yshift in ((0, 1), (1, 0), (1, 1)):
        for x, label in ((xi, "integer"), (xf, "fp32")):
            xb = torch.zeros(N + 1, device=dev)
            xb[xshift:xshift + N] = torch.from_numpy(x).to(dev)
            yb = torch.full((M + 1,), float("nan"), device=dev)
            plan.spmv(xb[xshift:xshift + N], yb[yshift:yshift + M])
            torch.cuda.synchronize()
            plan.check()
            got = yb[yshift:yshift + M].cpu().numpy()
            msg = "n=%d off=%d x+%d y+%d %s" % (n, off, xshift, yshift, label)
            if label == "integer":
                np.testing.assert_array_equal(got.astype(np.float64), want, err_msg=msg)
            else:
                np.testing.assert_array_equal(got, y_aligned, err_msg=msg)
    plan.close()
