"""The GPU partitioner against the reference: thumbnail stages, contours,
shape corners and the whole TaiChi_new format (golden fixtures recorded from
cv2 4.13.0 and from the reference's own partition_shapes), plus the
reference-signature C++ entry points of the library."""
import ctypes as C
import hashlib

import numpy as np
import pytest

import oracle
from tests.golden import cases

pytestmark = pytest.mark.gpu
FLT_MAX = np.float32(np.finfo(np.float32).max)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("idx", range(len(cases.IMAGE_CASES)))
def test_contours_match_cv2(tc, golden, idx):
    rec = golden["images"][idx]
    img = cases.image(**rec["case"])
    H, W = img.shape
    cap = 1 << 20
    lens = np.zeros(cap, np.int32)
    ends = np.zeros((cap, 4), np.int32)
    n = C.c_int()
    tc.check(tc.lib().tc_trace_contours(img.ctypes.data, H, W, lens.ctypes.data, ends.ctypes.data,
                                        cap, C.byref(n)))
    g = rec["contours"]
    assert n.value == g["count"], rec["case"]
    assert sha(lens[:n.value]) == g["lens_sha"], rec["case"]
    assert sha(ends[:n.value]) == g["ends_sha"], rec["case"]


def gpu_plan(tc, case):
    M, N, rp, col = cases.matrix(case)
    plan = tc.Plan.from_csr(M, N, rp, col, keep_host=True)
    return M, N, rp, col, plan


@pytest.mark.parametrize("case", cases.MATRIX_CASES, ids=[c["name"] for c in cases.MATRIX_CASES])
def test_gpu_partition_matches_reference(tc, golden, dev, case):
    rec = next(r for r in golden["partitions"] if r["name"] == case["name"])
    M, N, rp, col, plan = gpu_plan(tc, case)
    corners, stages = plan.thumbnail()
    assert corners.tolist() == rec["corners"], case["name"]
    if rec["stages"] is not None:
        assert [sha(s) for s in stages] == rec["stages"], case["name"]
    got = plan.export()
    for k in oracle.FORMAT_KEYS:
        assert got[k] == rec[k], (case["name"], k, got[k], rec[k])
    for k in ("xStart", "yStart", "xStop", "nDiasPtr", "neg_offsets"):
        assert got[k].tolist() == rec[k], (case["name"], k)
    if rec["dense_nnz"] > 0:
        assert sha(got["csrRow"]) == rec["csrRow_sha"], case["name"]
        assert sha(got["csrCol"]) == rec["csrCol_sha"], case["name"]
    else:   # the format is the input CSR (the reference aliases it)
        np.testing.assert_array_equal(got["csrRow"], rp)
        np.testing.assert_array_equal(got["csrCol"], col)
    print("%s: partition %.2f ms on the GPU" % (case["name"], plan.info()["partition_ms"]))
    plan.close()


def test_device_input_and_getsdf(tc, dev, golden):
    import torch
    case = next(c for c in cases.MATRIX_CASES if c["name"] == "multi_shape")
    rec = next(r for r in golden["partitions"] if r["name"] == "multi_shape")
    M, N, rp, col = cases.matrix(case)
    drp = torch.from_numpy(rp).to(dev)
    dcol = torch.from_numpy(col).to(dev)
    plan = tc.Plan.from_csr(M, N, drp, dcol, on_device=True)
    got = plan.export()
    assert got["neg_offsets"].tolist() == rec["neg_offsets"]
    assert sha(got["csrCol"]) == rec["csrCol_sha"]
    mF, W, nc = C.c_int(), C.c_int(), C.c_int()
    corners = np.zeros((64, 4), np.int32)
    st = np.zeros((5, 512, rec["W"]), np.uint8)
    tc.check(tc.lib().tc_getsdf(M, N, drp.data_ptr(), dcol.data_ptr(), None, C.byref(mF), C.byref(W),
                                corners.ctypes.data, 64, C.byref(nc), st.ctypes.data, None))
    assert (mF.value, W.value) == (rec["mF"], rec["W"])
    assert corners[:nc.value].tolist() == rec["corners"]
    assert [sha(s) for s in st] == rec["stages"]


def test_claimed_values_and_duplicates(tc, dev):
    """Entries whose value is already FLT_MAX count as claimed (TaiChi.cu:730);
    duplicate entries follow the reference's row walk (TaiChi.cu:809-827)."""
    from taichi_b200 import matgen
    M, N, rp, col = matgen.segments(30000, [(0, 30000, 0, 2, 0.9)], noise=300, seed=12)
    rng = np.random.default_rng(1)
    val = np.ones(rp[M], np.float32)
    val[rng.random(rp[M]) < 0.01] = FLT_MAX
    # duplicate a few entries in place (same row, same column, adjacent)
    rows = np.repeat(np.arange(M), np.diff(rp))
    dup_at = np.sort(rng.choice(rp[M], 500, replace=False))
    col2 = np.insert(col, dup_at, col[dup_at])
    val2 = np.insert(val, dup_at, 1.0)
    rows2 = np.insert(rows, dup_at, rows[dup_at])
    rp2 = np.zeros(M + 1, np.int32)
    np.cumsum(np.bincount(rows2, minlength=M), out=rp2[1:])
    want, wval = oracle.partition(M, N, rp2, col2, val=val2)
    plan = tc.Plan.from_csr(M, N, rp2, col2, val=val2, keep_host=True)
    got = plan.export()
    for k in oracle.FORMAT_KEYS:
        assert got[k] == want[k], k
    for k in ("xStart", "yStart", "xStop", "nDiasPtr", "neg_offsets", "csrRow", "csrCol"):
        assert np.array_equal(got[k], want[k]), k


# ------------------------------------------------- reference C++ entry points
class TaiChiNew(C.Structure):
    _fields_ = oracle.TaiChiNew._fields_


def _cpp(tc, name):
    return getattr(tc.lib(), name)


def test_compat_readmtx_partition_spmv(tc, dev, golden, tmp_path, monkeypatch):
    """readMtx -> partition_shapes -> taichi_SpMV through the reference's own
    C++ signatures, as main.cu calls them (main.cu:37-72)."""
    from taichi_b200 import matgen
    case = next(c for c in cases.MATRIX_CASES if c["name"] == "band_holes")
    rec = next(r for r in golden["partitions"] if r["name"] == "band_holes")
    M, N, rp, col = cases.matrix(case)
    path = str(tmp_path / "band_holes.mtx")
    matgen.to_mtx(path, M, N, rp, col)
    monkeypatch.setenv("TAICHI_B200_NUM_RUN", "3")
    monkeypatch.setenv("TAICHI_B200_NUM_TRANSFER", "2")
    L = tc.lib()
    readMtx = _cpp(tc, "_Z7readMtxPcRiS0_RmRPiS3_RPf")
    m, n, z = C.c_int(), C.c_int(), C.c_ulong()
    prp, pcol, pval = C.POINTER(C.c_int)(), C.POINTER(C.c_int)(), C.POINTER(C.c_float)()
    assert readMtx(C.c_char_p(path.encode()), C.byref(m), C.byref(n), C.byref(z), C.byref(prp),
                   C.byref(pcol), C.byref(pval)) == 0
    assert (m.value, n.value, z.value) == (M, N, rp[M])
    part = _cpp(tc, "_Z16partition_shapesPciiiRPiS1_RPfP10TaiChi_new")
    libc = C.CDLL("libc.so.6")
    libc.malloc.restype = C.c_void_p
    libc.calloc.restype = C.c_void_p
    t = C.cast(libc.calloc(1, C.sizeof(TaiChiNew)), C.POINTER(TaiChiNew))
    part(C.c_char_p(path.encode()), M, N, int(rp[M]), C.byref(prp), C.byref(pcol), C.byref(pval), t)
    f = t.contents
    for k in oracle.FORMAT_KEYS:
        assert getattr(f, k) == rec[k], k
    vals = np.ctypeslib.as_array(pval, shape=(int(rp[M]),))
    claimed = (vals == FLT_MAX).astype(np.uint8)
    assert sha(claimed) == rec["claimed_sha"]
    rows = np.ctypeslib.as_array(f.csrRow, shape=(M + 1,))
    assert sha(rows) == rec["csrRow_sha"]
    assert sha(np.ctypeslib.as_array(f.csrCol, shape=(int(rows[M]),))) == rec["csrCol_sha"]
    spmv = _cpp(tc, "_Z11taichi_SpMViiP10TaiChi_newPfS1_")
    x = np.ones(N, np.float32)
    y = np.zeros(M, np.float32)
    spmv(M, N, t, x.ctypes.data_as(C.POINTER(C.c_float)), y.ctypes.data_as(C.POINTER(C.c_float)))
    np.testing.assert_array_equal(y, np.diff(rp).astype(np.float32))   # main.cu:61-86 check
    # beyond the reference's own x = 1 check: integer x (exact) and FP32 x
    # (normwise within 1e-5 of the FP64 oracle)
    rng = np.random.default_rng(13)
    xi = rng.integers(-8, 9, N).astype(np.float32)
    spmv(M, N, t, xi.ctypes.data_as(C.POINTER(C.c_float)), y.ctypes.data_as(C.POINTER(C.c_float)))
    np.testing.assert_array_equal(y.astype(np.float64), oracle.spmv_csr_f64(M, rp, col, xi.astype(np.float64)))
    xf = rng.uniform(-1, 1, N).astype(np.float32)
    spmv(M, N, t, xf.ctypes.data_as(C.POINTER(C.c_float)), y.ctypes.data_as(C.POINTER(C.c_float)))
    y64 = oracle.spmv_csr_f64(M, rp, col, xf.astype(np.float64))
    rel = np.linalg.norm(y.astype(np.float64) - y64) / np.linalg.norm(y64)
    print("taichi_SpMV FP32 x: normwise rel err %.2e" % rel)
    assert rel <= 1e-5
    _cpp(tc, "_Z15free_taichi_newP10TaiChi_new")(t)
    for p in (prp, pcol, pval):
        libc.free(C.cast(p, C.c_void_p))


class Shape(C.Structure):
    _fields_ = [("id", C.c_int), ("category", C.c_char * 1024)] + \
        [(k, C.c_int) for k in ("x1", "y1", "a1", "b1", "area1", "x", "y", "a", "b", "width")]


class TaiChi(C.Structure):
    _fields_ = [("shape", C.c_char)] + [(k, C.c_int) for k in (
        "M_sub", "N_sub", "xStart", "yStart", "width", "neg", "maxNumZero")] + \
        [("neg_offsets", C.POINTER(C.c_int)), ("numZeroNeg", C.POINTER(C.c_int)),
         ("rowZeroNeg", C.POINTER(C.POINTER(C.c_int))), ("start", C.POINTER(C.c_int)),
         ("end", C.POINTER(C.c_int)), ("cStart", C.POINTER(C.c_int)), ("nnz", C.c_int),
         ("csrRow", C.POINTER(C.c_int)), ("csrCol", C.POINTER(C.c_int))]


def test_compat_partition_dia_shape(tc, dev, golden):
    """One shape through partition_dia_shape (TaiChi.cu:677-879): offsets,
    hole rows and the FLT_MAX marks equal the oracle's."""
    case = next(c for c in cases.MATRIX_CASES if c["name"] == "wide_band")
    rec = next(r for r in golden["partitions"] if r["name"] == "wide_band")
    M, N, rp, col = cases.matrix(case)
    x, y = rec["xStart"][0], rec["yStart"][0]
    b = rec["xStop"][0] - x
    sh = Shape(x=x, y=y, a=b, b=b)
    t = TaiChi()
    rpc = rp.copy(); colc = col.copy(); val = np.ones(rp[M], np.float32)
    prp = rpc.ctypes.data_as(C.POINTER(C.c_int))
    pcol = colc.ctypes.data_as(C.POINTER(C.c_int))
    pval = val.ctypes.data_as(C.POINTER(C.c_float))
    f = _cpp(tc, "_Z19partition_dia_shapeiiiRPiS0_RPffR5shapeR6TaiChi")
    f(M, N, int(rp[M]), C.byref(prp), C.byref(pcol), C.byref(pval), C.c_float(1.0), C.byref(sh),
      C.byref(t))
    assert [t.neg_offsets[i] for i in range(t.neg)] == rec["neg_offsets"]
    assert t.M_sub == b and t.xStart == x and t.yStart == y
    want, wval = oracle.partition(M, N, rp, col)
    np.testing.assert_array_equal(val == FLT_MAX, wval == FLT_MAX)
    assert sum(t.numZeroNeg[i] for i in range(t.neg)) == rec["zero_elements"]


def test_invalid_input_rejected(tc, dev):
    rp = np.array([0, 1, 2], np.int32)
    with pytest.raises(tc.TcError):
        tc.Plan.from_csr(2, 5, rp, np.array([0, 7], np.int32))        # column >= N
    with pytest.raises(tc.TcError):
        tc.Plan.from_csr(2, 5, np.array([0, 2, 1], np.int32), np.array([0, 1], np.int32))
