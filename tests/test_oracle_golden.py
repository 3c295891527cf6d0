"""The oracle (CPU restatement) against the golden fixtures recorded from
cv2 4.13.0 and from the reference's own code (tests/golden/make_golden.py)."""
import hashlib
import os

import numpy as np
import pytest

import oracle
from tests.golden import cases

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def contour_summary(cs):
    lens = np.array([len(c) for c in cs], np.int32)
    ends = np.array([[c[0][0], c[0][1], c[len(c) // 2][0], c[len(c) // 2][1]] for c in cs],
                    np.int32).reshape(-1, 4)
    allp = np.concatenate(cs) if cs else np.zeros((0, 2), np.int32)
    return dict(count=len(cs), lens_sha=sha(lens), ends_sha=sha(ends),
                points_sha=sha(allp.astype(np.int32)))


def test_images_morphology_and_contours(golden):
    for rec in golden["images"]:
        img = cases.image(**rec["case"])
        assert sha(oracle.imfill(img)) == rec["imfill"], rec["case"]
        assert sha(oracle.open_rect(img, 30, 1)) == rec["open_30x1"], rec["case"]
        assert sha(oracle.open_rect(img, 1, 30)) == rec["open_1x30"], rec["case"]
        assert sha(oracle.open_eye(img, 5)) == rec["open_eye5"], rec["case"]
        got = contour_summary(oracle.find_contours(img))
        for k in ("count", "lens_sha", "ends_sha", "points_sha"):
            assert got[k] == rec["contours"][k], (rec["case"], k)


def test_read_mtx(golden):
    for name, rec in golden["mtx"].items():
        rc, res = oracle.read_mtx(os.path.join(GOLD, "mtx", name))
        assert rc == rec["rc"], name
        if rc == 0:
            M, N, rp, col, val = res
            assert (M, N) == (rec["M"], rec["N"])
            assert rp.tolist() == rec["rowptr"] and col.tolist() == rec["col"], name
            np.testing.assert_array_equal(val, np.array(rec["val"], np.float32))


@pytest.mark.parametrize("name", [c["name"] for c in cases.MATRIX_CASES])
def test_partition(golden, name):
    rec = next(r for r in golden["partitions"] if r["name"] == name)
    case = next(c for c in cases.MATRIX_CASES if c["name"] == name)
    M, N, rp, col = cases.matrix(case)
    assert (M, N, int(rp[M])) == (rec["M"], rec["N"], rec["nnz"])
    # getSdf restatement == cv2 pipeline
    mF, W, corners, stages = oracle.getsdf(M, N, rp, col, stages=True)
    assert (mF, W) == (rec["mF"], rec["W"])
    assert corners.tolist() == rec["corners"]
    if rec["stages"] is not None:
        assert [sha(s) for s in stages] == rec["stages"]
    # partition restatement == the reference's partition_shapes
    fmt, val = oracle.partition(M, N, rp, col)
    for k in oracle.FORMAT_KEYS:
        assert fmt[k] == rec[k], k
    for k in ("xStart", "yStart", "xStop", "nDiasPtr", "neg_offsets"):
        assert fmt[k].tolist() == rec[k], k
    if not rec["csr_null"]:
        assert int(fmt["csrRow"][M]) == rec["nnz_csr"]
        assert sha(fmt["csrRow"]) == rec["csrRow_sha"]
        assert sha(fmt["csrCol"]) == rec["csrCol_sha"]
    claimed = (val == np.float32(np.finfo(np.float32).max)).astype(np.uint8)
    assert int(claimed.sum()) == rec["claimed_count"] and sha(claimed) == rec["claimed_sha"]
    # the format represents the same matrix: exact for integer x
    rng = np.random.default_rng(0)
    x = rng.integers(-8, 9, N).astype(np.float64)
    np.testing.assert_array_equal(oracle.spmv_format_f64(fmt, M, N, x),
                                  oracle.spmv_csr_f64(M, rp, col, x))


def test_cal_start_end_and_width():
    # square blocks: the valid local rows of an offset are exactly the rows r
    # with 0 <= r + off < size (TaiChi.cu:881-916)
    for size in (5, 17, 1000):
        for w in (1, 2, 4):
            for n in range(2 * w - 1):
                off = n - w + 1
                s, e = oracle.C.c_int(), oracle.C.c_int()
                oracle.lib().or_cal_start_end(size, size, w, off, n, oracle.C.byref(s),
                                              oracle.C.byref(e))
                rows = [r for r in range(size) if 0 <= r + off < size]
                assert (s.value, e.value) == (rows[0], rows[-1] + 1)
    L = oracle.lib()
    assert [L.or_band_width(v) for v in (1000, 9999, 10000, 99999, 100000, 999999, 1000000,
                                         9999999, 10000000)] == \
        [100, 999, 100, 999, 100, 999, 10, 99, 10]
