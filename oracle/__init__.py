"""ctypes view of the oracle -- the CPU checker for taichi_b200.

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline leg; never by the taichi_b200 package.

Two libraries live here:

* ``liboracle.so`` -- taichi_oracle.c, a C restatement of the reference path
  (MM reader, thumbnail, morphology, contours, partition, SpMV).
* ``_ref/libtaichi_ref.so`` -- the reference's own TaiChi.cu + mmio.cpp built
  from source with shim headers (oracle/build.py); used to pin the
  restatement.  Present only where it was built.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_IP = C.POINTER(C.c_int)
_FP = C.POINTER(C.c_float)


class Params(C.Structure):
    _fields_ = [("thumb_height", C.c_int), ("open_len", C.c_int), ("eye_size", C.c_int),
                ("min_contour", C.c_int), ("min_shape_side", C.c_int), ("density", C.c_double)]


class Format(C.Structure):
    _fields_ = [("dia_shapes", C.c_int), ("num_negs", C.c_int), ("dense_nnz", C.c_int),
                ("zero_elements", C.c_int), ("sparse_nnz", C.c_int), ("row_start", C.c_int),
                ("row_stop", C.c_int), ("xStart", _IP), ("yStart", _IP), ("xStop", _IP),
                ("nDiasPtr", _IP), ("neg_offsets", _IP), ("csrRow", _IP), ("csrCol", _IP),
                ("csr_aliases_input", C.c_int)]


class TaiChiNew(C.Structure):
    """Byte layout of the reference's TaiChi_new (TaiChi.h:45-60)."""
    _fields_ = [("dia_shapes", C.c_int), ("num_negs", C.c_int), ("dense_nnz", C.c_int),
                ("zero_elements", C.c_int), ("sparse_nnz", C.c_int), ("row_start", C.c_int),
                ("row_stop", C.c_int), ("xStart", _IP), ("yStart", _IP), ("xStop", _IP),
                ("nDiasPtr", _IP), ("neg_offsets", _IP), ("csrRow", _IP), ("csrCol", _IP)]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            from . import build as _b  # noqa: F401  (only where gcc exists)
            _b.build_oracle()
        L = C.CDLL(path)
        L.or_params_default.argtypes = [C.POINTER(Params)]
        L.or_read_mtx.argtypes = [C.c_char_p, _IP, _IP, C.POINTER(C.c_ulong),
                                  C.POINTER(_IP), C.POINTER(_IP), C.POINTER(_FP)]
        L.or_free.argtypes = [C.c_void_p]
        L.or_thumb_dims.argtypes = [C.c_int, C.c_int, C.c_int, _IP, _IP, _IP]
        L.or_raster.argtypes = [C.c_int, _i32p, _i32p, C.c_int, C.c_int, C.c_int, C.c_int, _u8p]
        L.or_imfill.argtypes = [_u8p, C.c_int, C.c_int, _u8p]
        L.or_open_rect.argtypes = [_u8p, C.c_int, C.c_int, C.c_int, C.c_int, _u8p]
        L.or_open_eye.argtypes = [_u8p, C.c_int, C.c_int, C.c_int, _u8p]
        L.or_find_contours.argtypes = [_u8p, C.c_int, C.c_int, C.POINTER(_IP), C.POINTER(_IP),
                                       C.POINTER(C.c_long)]
        L.or_getsdf.argtypes = [C.c_int, C.c_int, _i32p, _i32p, C.POINTER(Params), _IP, _IP,
                                C.POINTER(_IP), C.c_void_p]
        L.or_cal_shape_size.argtypes = [C.c_int] * 7 + [_IP] * 4 + [C.POINTER(C.c_float)]
        L.or_cal_start_end.argtypes = [C.c_int] * 5 + [_IP, _IP]
        L.or_band_width.argtypes = [C.c_int]
        L.or_partition.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f32p,
                                   C.POINTER(Params), C.c_void_p, C.c_int, C.c_int,
                                   C.POINTER(Format)]
        L.or_format_free.argtypes = [C.POINTER(Format)]
        L.or_spmv_csr_f64.argtypes = [C.c_int, _i32p, _i32p, _f64p, _f64p]
        L.or_spmv_csr_f32_serial.argtypes = [C.c_int, _i32p, _i32p, _f32p, _f32p]
        L.or_spmv_csr_f32_omp.argtypes = [C.c_int, _i32p, _i32p, _f32p, _f32p, C.c_int]
        L.or_spmm_csr_f64.argtypes = [C.c_int, _i32p, _i32p, C.c_int, _f64p, _f64p]
        L.or_spmv_format_f64.argtypes = [C.POINTER(Format), C.c_int, C.c_int, _f64p, _f64p]
        _LIB = L
    return _LIB


def default_params(**over):
    p = Params()
    lib().or_params_default(C.byref(p))
    for k, v in over.items():
        setattr(p, k, v)
    return p


def _take(ptr, n, dtype=np.int32):
    if n <= 0 or not ptr:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


# --------------------------------------------------------------------- reader
def read_mtx(path):
    L = lib()
    m, n, z = C.c_int(), C.c_int(), C.c_ulong()
    rp, ci, va = _IP(), _IP(), _FP()
    rc = L.or_read_mtx(path.encode(), C.byref(m), C.byref(n), C.byref(z),
                       C.byref(rp), C.byref(ci), C.byref(va))
    if rc != 0:
        return rc, None
    M, nnz = m.value, z.value
    out = (M, n.value, _take(rp, M + 1), _take(ci, nnz),
           np.ctypeslib.as_array(va, shape=(max(nnz, 1),))[:nnz].copy())
    for p in (rp, ci, va):
        L.or_free(C.cast(p, C.c_void_p))
    return 0, out


# ---------------------------------------------------------------- morphology
def thumb_dims(M, N, height=512):
    W, pM, pN = C.c_int(), C.c_int(), C.c_int()
    ok = lib().or_thumb_dims(M, N, height, C.byref(W), C.byref(pM), C.byref(pN))
    return ok, W.value, pM.value, pN.value


def raster(M, N, rowptr, col, height=512):
    ok, W, pM, pN = thumb_dims(M, N, height)
    if ok <= 0:
        return None
    img = np.empty((height, W), np.uint8)
    lib().or_raster(M, rowptr, col, height, W, pM, pN, img)
    return img


def imfill(img):
    img = np.ascontiguousarray(img, np.uint8)
    out = np.empty_like(img)
    lib().or_imfill(img, img.shape[0], img.shape[1], out)
    return out


def open_rect(img, kw, kh):
    img = np.ascontiguousarray(img, np.uint8)
    out = np.empty_like(img)
    lib().or_open_rect(img, img.shape[0], img.shape[1], kw, kh, out)
    return out


def open_eye(img, k=5):
    img = np.ascontiguousarray(img, np.uint8)
    out = np.empty_like(img)
    lib().or_open_eye(img, img.shape[0], img.shape[1], k, out)
    return out


def find_contours(img):
    """List of (n, 2) int32 arrays of (x, y) points, in OpenCV's order."""
    img = np.ascontiguousarray(img, np.uint8)
    L = lib()
    pts, lens, tot = _IP(), _IP(), C.c_long()
    n = L.or_find_contours(img, img.shape[0], img.shape[1], C.byref(pts), C.byref(lens),
                           C.byref(tot))
    P = _take(pts, 2 * tot.value).reshape(-1, 2)
    ln = _take(lens, n)
    L.or_free(C.cast(pts, C.c_void_p))
    L.or_free(C.cast(lens, C.c_void_p))
    out, o = [], 0
    for k in ln:
        out.append(P[o:o + k])
        o += k
    return out


def getsdf(M, N, rowptr, col, params=None, stages=False):
    """Returns (mF, W, corners[n,4], stages[5,H,W] or None)."""
    p = params or default_params()
    L = lib()
    mF, W, cs = C.c_int(), C.c_int(), _IP()
    st = None
    stp = None
    ok, Wd, _, _ = thumb_dims(M, N, p.thumb_height)
    if stages and ok > 0:
        st = np.zeros((5, p.thumb_height, Wd), np.uint8)
        stp = st.ctypes.data_as(C.c_void_p)
    n = L.or_getsdf(M, N, np.ascontiguousarray(rowptr, np.int32),
                    np.ascontiguousarray(col, np.int32), C.byref(p), C.byref(mF), C.byref(W),
                    C.byref(cs), stp)
    corners = _take(cs, 4 * max(n, 0)).reshape(-1, 4)
    if cs:
        L.or_free(C.cast(cs, C.c_void_p))
    return mF.value, W.value, corners, st


# ----------------------------------------------------------------- partition
FORMAT_KEYS = ("dia_shapes", "num_negs", "dense_nnz", "zero_elements", "sparse_nnz",
               "row_start", "row_stop")


def _format_dict(f, M):
    d = {k: getattr(f, k) for k in FORMAT_KEYS}
    s = f.dia_shapes
    d["xStart"] = _take(f.xStart, s)
    d["yStart"] = _take(f.yStart, s)
    d["xStop"] = _take(f.xStop, s)
    d["nDiasPtr"] = _take(f.nDiasPtr, s + 1) if s > 0 else np.zeros(0, np.int32)
    d["neg_offsets"] = _take(f.neg_offsets, f.num_negs)
    if f.csrRow:
        d["csrRow"] = _take(f.csrRow, M + 1)
        d["csrCol"] = _take(f.csrCol, int(d["csrRow"][M]))
    else:
        d["csrRow"] = np.zeros(M + 1, np.int32)
        d["csrCol"] = np.zeros(0, np.int32)
    return d


def partition(M, N, rowptr, col, val=None, params=None, corners=None, mF=512):
    """Sequential restatement of partition_shapes.  Returns (format dict,
    mutated val).  `corners` (n x 4) replaces getSdf's shape list."""
    p = params or default_params()
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    nnz = int(rowptr[M])
    v = np.ones(max(nnz, 1), np.float32) if val is None else np.array(val, np.float32, copy=True)
    f = Format()
    cptr, ncs = None, 0
    if corners is not None:
        cs = np.ascontiguousarray(np.asarray(corners, np.int32).reshape(-1, 4))
        cptr, ncs = cs.ctypes.data_as(C.c_void_p), cs.shape[0]
    rc = lib().or_partition(M, N, nnz, rowptr, col, v, C.byref(p), cptr, ncs, mF, C.byref(f))
    if rc != 0:
        raise ValueError("oracle partition failed: %d" % rc)
    d = _format_dict(f, M)
    d["csr_aliases_input"] = bool(f.csr_aliases_input)
    lib().or_format_free(C.byref(f))
    return d, v[:nnz]


def format_struct(d):
    """Builds an oracle Format struct (and keeps its arrays alive)."""
    keep = {}
    f = Format()
    for k in FORMAT_KEYS:
        setattr(f, k, int(d[k]))
    for k in ("xStart", "yStart", "xStop", "nDiasPtr", "neg_offsets", "csrRow", "csrCol"):
        a = np.ascontiguousarray(d[k], np.int32)
        if a.size == 0:
            a = np.zeros(1, np.int32)
        keep[k] = a
        setattr(f, k, a.ctypes.data_as(_IP))
    f.csr_aliases_input = int(d.get("csr_aliases_input", d["dense_nnz"] == 0))
    return f, keep


# ---------------------------------------------------------------------- SpMV
def spmv_csr_f64(M, rowptr, col, x):
    y = np.empty(M, np.float64)
    lib().or_spmv_csr_f64(M, np.ascontiguousarray(rowptr, np.int32),
                          np.ascontiguousarray(col, np.int32),
                          np.ascontiguousarray(x, np.float64), y)
    return y


def spmv_csr_f32_serial(M, rowptr, col, x):
    y = np.empty(M, np.float32)
    lib().or_spmv_csr_f32_serial(M, np.ascontiguousarray(rowptr, np.int32),
                                 np.ascontiguousarray(col, np.int32),
                                 np.ascontiguousarray(x, np.float32), y)
    return y


def spmv_csr_f32_omp(M, rowptr, col, x, threads, y=None):
    if y is None:
        y = np.empty(M, np.float32)
    lib().or_spmv_csr_f32_omp(M, rowptr, col, x, y, threads)
    return y


def spmm_csr_f64(M, rowptr, col, X):
    X = np.ascontiguousarray(X, np.float64)
    k = X.shape[1]
    Y = np.empty((M, k), np.float64)
    lib().or_spmm_csr_f64(M, np.ascontiguousarray(rowptr, np.int32),
                          np.ascontiguousarray(col, np.int32), k, X, Y)
    return Y


def spmv_format_f64(d, M, N, x):
    f, keep = format_struct(d)
    y = np.empty(M, np.float64)
    lib().or_spmv_format_f64(C.byref(f), M, N, np.ascontiguousarray(x, np.float64), y)
    del keep
    return y


# ------------------------------------------------------- the reference itself
def ref_lib():
    """The reference's own code (oracle/_ref), or None where it was not built."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libtaichi_ref.so")
        if not os.path.exists(path):
            return None
        R = C.CDLL(path)
        R.ref_set_shapes.argtypes = [C.c_int, C.c_int, C.c_int, _i32p]
        R.ref_clear_shapes.argtypes = []
        R.ref_read_mtx.argtypes = [C.c_char_p, _IP, _IP, C.POINTER(C.c_ulong),
                                   C.POINTER(_IP), C.POINTER(_IP), C.POINTER(_FP)]
        R.ref_partition.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f32p]
        R.ref_partition.restype = C.POINTER(TaiChiNew)
        R.ref_free_taichi_new.argtypes = [C.POINTER(TaiChiNew)]
        R.ref_free.argtypes = [C.c_void_p]
        R.ref_taichi_spmv.argtypes = [C.c_int, C.c_int, C.POINTER(TaiChiNew), _f32p, _f32p]
        _REF = R
    return _REF


def ref_read_mtx(path):
    R = ref_lib()
    m, n, z = C.c_int(), C.c_int(), C.c_ulong()
    rp, ci, va = _IP(), _IP(), _FP()
    rc = R.ref_read_mtx(path.encode(), C.byref(m), C.byref(n), C.byref(z),
                        C.byref(rp), C.byref(ci), C.byref(va))
    if rc != 0:
        return rc, None
    M, nnz = m.value, z.value
    out = (M, n.value, _take(rp, M + 1), _take(ci, nnz),
           np.ctypeslib.as_array(va, shape=(max(nnz, 1),))[:nnz].copy())
    for p in (rp, ci, va):
        R.ref_free(C.cast(p, C.c_void_p))
    return 0, out


def ref_partition(M, N, rowptr, col, val=None, corners=None, mF=512, W=512, workdir=None):
    """Runs the reference's own partition_shapes.  The shape corners come
    from `corners` (n x 4, e.g. computed by cv2); the reference appends a line
    to ./nnz_density.txt, so it runs inside `workdir` when given."""
    R = ref_lib()
    rowptr = np.array(rowptr, np.int32, copy=True)
    col = np.array(col, np.int32, copy=True)
    nnz = int(rowptr[M])
    v = np.ones(max(nnz, 1), np.float32) if val is None else np.array(val, np.float32, copy=True)
    if corners is None:
        R.ref_clear_shapes()
    else:
        cs = np.ascontiguousarray(np.asarray(corners, np.int32).reshape(-1, 4))
        R.ref_set_shapes(mF, W, cs.shape[0], cs.reshape(-1) if cs.size else np.zeros(1, np.int32))
    cwd = os.getcwd()
    try:
        if workdir:
            os.chdir(workdir)
        t = R.ref_partition(M, N, nnz, rowptr, col, v)
    finally:
        os.chdir(cwd)
    f = t.contents
    d = {k: getattr(f, k) for k in FORMAT_KEYS}
    s = f.dia_shapes
    d["xStart"] = _take(f.xStart, s)
    d["yStart"] = _take(f.yStart, s)
    d["xStop"] = _take(f.xStop, s)
    d["nDiasPtr"] = _take(f.nDiasPtr, s + 1) if s > 0 else np.zeros(0, np.int32)
    d["neg_offsets"] = _take(f.neg_offsets, f.num_negs)
    if f.csrRow:
        d["csrRow"] = _take(f.csrRow, M + 1)
        d["csrCol"] = _take(f.csrCol, int(d["csrRow"][M]))
    else:
        d["csrRow"] = None
        d["csrCol"] = None
    R.ref_free_taichi_new(t)
    R.ref_clear_shapes()
    return d, v[:nnz]
