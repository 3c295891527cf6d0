"""taichi_b200 -- B200-native TaiChi binary SpMV.

Python view of libtaichi_b200.so (the C ABI declared in include/taichi_b200.h),
used by the tests and the benchmark.  The compute path is the CUDA library:
if it is not built this module raises instead of falling back to anything.

Device vectors may be given as torch CUDA tensors (float32, contiguous) or as
raw device addresses (int).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtaichi_b200.so")
_LIB = None

TC_FLAG_NO_PARTITION = 0x1
TC_FLAG_KEEP_HOST = 0x2
TC_FLAG_NO_PDL = 0x4
TC_FLAG_ROWS_STRIDED = 0x8
TC_FLAG_NO_DIRECT = 0x10
TC_FLAG_NO_WIDE = 0x20
TC_FLAG_NO_WINDOW = 0x40
TC_FLAG_WINDOW = 0x80
TC_FLAG_WIDE_BOUNDS = 0x100
TC_FLAG_WIDE_FIXED = 0x200
TC_FLAG_ROWS = 0x400
TC_FLAG_NO_ROWS = 0x800
TC_FLAG_NO_PREFETCH = 0x2000
TC_FLAG_NO_PARAM_STARTS = 0x4000
TC_FLAG_HOST_Y_MAPPED = 0x8000

_IP = C.POINTER(C.c_int)


class TcError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("taichi_b200 status %d: %s" % (status, msg))
        self.status = status


class Params(C.Structure):
    _fields_ = [("thumb_height", C.c_int), ("open_len", C.c_int), ("eye_size", C.c_int),
                ("min_contour", C.c_int), ("min_shape_side", C.c_int), ("density", C.c_double),
                ("tile_rows", C.c_int), ("tile_nnz", C.c_int), ("max_lanes", C.c_int),
                ("ctas_per_sm", C.c_int), ("tile_mode", C.c_int), ("flags", C.c_int), ("rows_w", C.c_int)]


class Format(C.Structure):
    _fields_ = [("dia_shapes", C.c_int), ("num_negs", C.c_int), ("dense_nnz", C.c_int),
                ("zero_elements", C.c_int), ("sparse_nnz", C.c_int), ("row_start", C.c_int),
                ("row_stop", C.c_int), ("xStart", _IP), ("yStart", _IP), ("xStop", _IP),
                ("nDiasPtr", _IP), ("neg_offsets", _IP), ("csrRow", _IP), ("csrCol", _IP)]


class PlanInfo(C.Structure):
    _fields_ = [("M", C.c_int), ("N", C.c_int), ("dia_shapes", C.c_int), ("num_negs", C.c_int),
                ("dense_nnz", C.c_int), ("zero_elements", C.c_int), ("sparse_nnz", C.c_int),
                ("row_start", C.c_int), ("row_stop", C.c_int), ("nnz_input", C.c_int64),
                ("nnz_csr", C.c_int64), ("ntiles", C.c_int), ("ntiles_vector", C.c_int),
                ("ntiles_long", C.c_int), ("device_bytes", C.c_int64), ("spmv_bytes", C.c_int64),
                ("partition_ms", C.c_double), ("num_contours", C.c_int), ("nwtiles", C.c_int),
                ("window_lo", C.c_int), ("window_hi", C.c_int), ("kernel", C.c_int)]


KERNEL_NAMES = {0: "tiles", 1: "grid", 2: "lean", 3: "wide", 4: "stream", 5: "rows", 6: "window"}


# extern "C" symbols declared in include/taichi_b200.h (checked by the tests)
EXPORTS = (
    "tc_params_default", "tc_last_error", "tc_status_string", "tc_plan_create",
    "tc_plan_from_format", "tc_plan_destroy", "tc_plan_info_get", "tc_plan_export",
    "tc_plan_thumbnail", "tc_plan_check", "tc_plan_save", "tc_plan_load", "tc_spmv", "tc_spmv_f64", "tc_spmv_host",
    "tc_spmv_host_async",
    "tc_spmm", "tc_getsdf",
    "tc_trace_contours", "tc_read_mtx", "tc_free", "tc_batch_create", "tc_batch_run",
    "tc_batch_graph_launch", "tc_batch_destroy", "tc_tune", "tc_tune_cache_clear",
    "tc_serve_config_default", "tc_server_create", "tc_server_admit", "tc_server_evict",
    "tc_server_hbm_used", "tc_server_run", "tc_server_destroy", "tc_thumbnail_noalloc",
    "tc_server_start", "tc_server_submit", "tc_server_poll", "tc_server_wait", "tc_server_stats",
    "tc_server_stop", "tc_read_mtx_device", "tc_device_free",
)


class TuneResult(C.Structure):
    _fields_ = [("params", Params), ("spmv_us", C.c_double), ("default_us", C.c_double),
                ("trials", C.c_int), ("cached", C.c_int), ("fingerprint", C.c_uint64)]


def lib():
    """The loaded CUDA library; raises if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libtaichi_b200.so is not built (python -m taichi_b200.build)")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.tc_params_default.argtypes = [C.POINTER(Params)]
        L.tc_params_default.restype = None
        L.tc_last_error.restype = C.c_char_p
        L.tc_status_string.restype = C.c_char_p
        L.tc_status_string.argtypes = [C.c_int]
        L.tc_plan_create.argtypes = [C.c_int, C.c_int, C.c_int64, vp, vp, vp, C.c_int,
                                     C.POINTER(Params), vp, C.POINTER(vp)]
        L.tc_plan_from_format.argtypes = [C.c_int, C.c_int, C.POINTER(Format),
                                          C.POINTER(Params), vp, C.POINTER(vp)]
        L.tc_plan_destroy.argtypes = [vp]
        L.tc_plan_info_get.argtypes = [vp, C.POINTER(PlanInfo)]
        L.tc_plan_export.argtypes = [vp] + [vp] * 7
        L.tc_plan_thumbnail.argtypes = [vp, vp, _IP, vp, _IP]
        L.tc_plan_check.argtypes = [vp]
        L.tc_plan_save.argtypes = [vp, C.c_char_p]
        L.tc_plan_load.argtypes = [C.c_char_p, C.POINTER(Params), vp, C.POINTER(vp)]
        L.tc_spmv.argtypes = [vp, vp, vp, vp]
        L.tc_spmv_f64.argtypes = [vp, vp, vp, vp]
        L.tc_spmv_host.argtypes = [vp, vp, vp, vp]
        L.tc_spmv_host_async.argtypes = [vp, vp, vp, C.c_int, vp]
        L.tc_spmm.argtypes = [vp, vp, C.c_int, C.c_int, vp, C.c_int, vp]
        L.tc_getsdf.argtypes = [C.c_int, C.c_int, vp, vp, C.POINTER(Params), _IP, _IP, vp,
                                C.c_int, _IP, vp, vp]
        L.tc_trace_contours.argtypes = [vp, C.c_int, C.c_int, vp, vp, C.c_int, _IP]
        L.tc_thumbnail_noalloc.argtypes = [C.c_int, C.c_int, vp, vp, C.POINTER(Params), vp,
                                           _IP, vp]
        L.tc_read_mtx.argtypes = [C.c_char_p, _IP, _IP, C.POINTER(C.c_int64), C.POINTER(_IP),
                                  C.POINTER(_IP), C.POINTER(C.POINTER(C.c_float)), _IP]
        L.tc_free.argtypes = [vp]
        L.tc_read_mtx_device.argtypes = [C.c_char_p, _IP, _IP, C.POINTER(C.c_int64), C.POINTER(vp),
                                         C.POINTER(vp), C.POINTER(vp), _IP, C.POINTER(C.c_double),
                                         C.POINTER(C.c_double), vp]
        L.tc_device_free.argtypes = [vp]
        L.tc_device_free.restype = None
        L.tc_gen_rmat.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                  C.c_uint64, C.c_int, _IP, C.POINTER(_IP), C.POINTER(_IP)]
        L.tc_gen_banded.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(_IP),
                                    C.POINTER(_IP)]
        L.tc_batch_create.argtypes = [C.c_int, vp, vp, vp, C.POINTER(vp)]
        L.tc_batch_run.argtypes = [vp, vp]
        L.tc_batch_graph_launch.argtypes = [vp, vp]
        L.tc_batch_destroy.argtypes = [vp]
        L.tc_tune.argtypes = [C.c_int, C.c_int, C.c_int64, vp, vp, C.POINTER(Params), C.c_int, vp,
                              C.POINTER(TuneResult)]
        L.tc_tune_cache_clear.argtypes = []
        L.tc_tune_cache_clear.restype = None
        L.tc_serve_config_default.argtypes = [C.POINTER(ServeConfig)]
        L.tc_serve_config_default.restype = None
        L.tc_server_create.argtypes = [C.POINTER(ServeConfig), C.POINTER(vp)]
        L.tc_server_admit.argtypes = [vp, vp, C.POINTER(C.c_int)]
        L.tc_server_evict.argtypes = [vp, C.c_int]
        L.tc_server_hbm_used.argtypes = [vp]
        L.tc_server_hbm_used.restype = C.c_int64
        L.tc_server_run.argtypes = [vp, C.c_int, vp, vp, vp, vp, C.c_int, vp,
                                    C.POINTER(ServeStats)]
        L.tc_server_destroy.argtypes = [vp]
        L.tc_server_start.argtypes = [vp, C.c_int]
        L.tc_server_submit.argtypes = [vp, C.c_int, vp, vp, C.POINTER(C.c_uint64)]
        L.tc_server_poll.argtypes = [vp, C.c_uint64, C.POINTER(C.c_int)]
        L.tc_server_wait.argtypes = [vp, C.c_uint64, C.c_double]
        L.tc_server_stats.argtypes = [vp, C.POINTER(ServeStats)]
        L.tc_server_stop.argtypes = [vp]
        _LIB = L
    return _LIB


def check(status):
    if status != 0:
        raise TcError(status, lib().tc_last_error().decode(errors="replace"))


def params(**over):
    p = Params()
    lib().tc_params_default(C.byref(p))
    for k, v in over.items():
        setattr(p, k, v)
    return p


def _ptr(a):
    """Device address of a torch tensor / raw int, or host address of numpy."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        assert a.is_contiguous(), "tensor must be contiguous"
        return a.data_ptr()
    raise TypeError("unsupported array type %r" % type(a))


def _stream(s):
    if s is None:
        return None
    if isinstance(s, int):
        return s
    return s.cuda_stream


class ServeConfig(C.Structure):
    _fields_ = [("hbm_budget", C.c_int64), ("arena_bytes", C.c_int64), ("contexts", C.c_int),
                ("max_batch", C.c_int), ("max_plans", C.c_int), ("max_inflight", C.c_int),
                ("max_pending", C.c_int), ("solo_bytes", C.c_int64)]


class ServeStats(C.Structure):
    _fields_ = [("requests", C.c_int64), ("batches", C.c_int64), ("seconds", C.c_double),
                ("spmv_per_s", C.c_double), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("mean_ms", C.c_double), ("max_ms", C.c_double), ("mean_batch", C.c_double),
                ("mean_service_ms", C.c_double), ("mean_launch_us", C.c_double)]


SERVE_DEVICE_VECTORS = 2     # tc_server_run mode bit: requests carry device x / y


class Server:
    """Resident matrices + continuous batching of SpMV requests (tc_server)."""

    def __init__(self, **cfg):
        L = lib()
        c = ServeConfig()
        L.tc_serve_config_default(C.byref(c))
        for k, v in cfg.items():
            setattr(c, k, v)
        self._h = C.c_void_p()
        check(L.tc_server_create(C.byref(c), C.byref(self._h)))
        self._plans = {}

    def admit(self, plan):
        i = C.c_int()
        check(lib().tc_server_admit(self._h, plan.handle, C.byref(i)))
        self._plans[i.value] = plan
        return i.value

    def evict(self, mid):
        check(lib().tc_server_evict(self._h, mid))
        self._plans.pop(mid, None)

    def hbm_used(self):
        return lib().tc_server_hbm_used(self._h)

    def run(self, arrival_s, matrix, xs, ys, mode=0):
        """xs / ys: per-request host arrays (numpy or pinned torch, float32,
        contiguous); device tensors with mode | SERVE_DEVICE_VECTORS.
        Returns (stats dict, latency_ms array)."""
        n = len(matrix)
        arr = np.ascontiguousarray(arrival_s, np.float64)
        mat = np.ascontiguousarray(matrix, np.int32)
        X = (C.c_void_p * n)(*[_ptr(a) for a in xs])
        Y = (C.c_void_p * n)(*[_ptr(a) for a in ys])
        lat = np.zeros(n, np.float64)
        st = ServeStats()
        check(lib().tc_server_run(self._h, n, arr.ctypes.data, mat.ctypes.data, X, Y, mode,
                                  lat.ctypes.data, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServeStats._fields_}, lat

    # -- online requests (tc_server_start / submit / poll / wait / stop) ----
    def start(self, device_vectors=True):
        check(lib().tc_server_start(self._h, 1 if device_vectors else 0))

    def submit(self, mid, x, y):
        """Queues y = A_mid x; returns a ticket (x / y: device tensors after
        start(device_vectors=True), pinned host tensors otherwise)."""
        t = C.c_uint64()
        check(lib().tc_server_submit(self._h, mid, _ptr(x), _ptr(y), C.byref(t)))
        return t.value

    def poll(self, ticket):
        d = C.c_int()
        check(lib().tc_server_poll(self._h, ticket, C.byref(d)))
        return bool(d.value)

    def wait(self, ticket, timeout_s=-1.0):
        check(lib().tc_server_wait(self._h, ticket, timeout_s))

    def stats(self):
        st = ServeStats()
        check(lib().tc_server_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServeStats._fields_}

    def stop(self):
        check(lib().tc_server_stop(self._h))

    def close(self):
        if self._h:
            lib().tc_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tune(M, N, rowptr, col, prm=None, max_trials=32, stream=None):
    """Autotunes the partition threshold and tile shape for a host CSR;
    returns a TuneResult (params usable with Plan.from_csr)."""
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    r = TuneResult()
    check(lib().tc_tune(M, N, int(rowptr[M]), rowptr.ctypes.data, col.ctypes.data,
                        C.byref(prm) if prm is not None else None, max_trials, _stream(stream),
                        C.byref(r)))
    return r


def _take_csr(M, rp, ci):
    L = lib()
    nnz = rp[M]
    out = (np.ctypeslib.as_array(rp, shape=(M + 1,)).copy(),
           np.ctypeslib.as_array(ci, shape=(max(nnz, 1),))[:nnz].copy())
    L.tc_free(C.cast(rp, C.c_void_p))
    L.tc_free(C.cast(ci, C.c_void_p))
    return out


def gen_rmat(scale, edge_factor=16, a=0.499, b=0.001, c=0.001, seed=1, self_loops=False):
    """R-MAT pattern from the library's multi-threaded generator: (M, rowptr, col)."""
    M, rp, ci = C.c_int(), _IP(), _IP()
    check(lib().tc_gen_rmat(scale, edge_factor, a, b, c, seed, int(self_loops), C.byref(M),
                            C.byref(rp), C.byref(ci)))
    return (M.value,) + _take_csr(M.value, rp, ci)


def gen_banded(n, k, per_row, seed):
    """Banded-plus-random pattern: (rowptr, col)."""
    rp, ci = _IP(), _IP()
    check(lib().tc_gen_banded(n, k, per_row, seed, C.byref(rp), C.byref(ci)))
    return _take_csr(n, rp, ci)


def read_mtx_device(path, stream=None):
    """Matrix Market -> CSR built on the GPU (tc_read_mtx_device).  Returns
    ((M, N, rowptr, col, val), (parse_ms, build_ms)) with rowptr / col / val
    as torch CUDA tensors (copied from the library's arrays, which are then
    freed)."""
    import torch
    L = lib()
    M, N, nnz, code = C.c_int(), C.c_int(), C.c_int64(), C.c_int()
    ptrs = [C.c_void_p(), C.c_void_p(), C.c_void_p()]
    pm, bm = C.c_double(), C.c_double()
    st = L.tc_read_mtx_device(path.encode(), C.byref(M), C.byref(N), C.byref(nnz), C.byref(ptrs[0]),
                              C.byref(ptrs[1]), C.byref(ptrs[2]), C.byref(code), C.byref(pm), C.byref(bm),
                              _stream(stream))
    if st != 0:
        raise TcError(st, "%s (reference code %d)" % (L.tc_last_error().decode(), code.value))
    m, z = M.value, nnz.value
    rt = C.CDLL("libcudart.so.12")
    rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
    out = []
    for ptr, n, dt in zip(ptrs, (m + 1, z, z), (torch.int32, torch.int32, torch.float32)):
        t = torch.empty(n, dtype=dt, device="cuda")
        if n:
            assert rt.cudaMemcpy(t.data_ptr(), ptr.value, 4 * n, 3) == 0     # device to device
        out.append(t)
        L.tc_device_free(ptr)
    return (m, N.value) + tuple(out), (pm.value, bm.value)


def read_mtx(path):
    """Matrix Market -> (M, N, rowptr, col, val) numpy arrays (readMtx)."""
    L = lib()
    M, N, nnz, code = C.c_int(), C.c_int(), C.c_int64(), C.c_int()
    rp, ci, va = _IP(), _IP(), C.POINTER(C.c_float)()
    st = L.tc_read_mtx(path.encode(), C.byref(M), C.byref(N), C.byref(nnz), C.byref(rp),
                       C.byref(ci), C.byref(va), C.byref(code))
    if st != 0:
        raise TcError(st, "%s (reference code %d)" % (L.tc_last_error().decode(), code.value))
    m, z = M.value, nnz.value
    out = (m, N.value, np.ctypeslib.as_array(rp, shape=(m + 1,)).copy(),
           np.ctypeslib.as_array(ci, shape=(max(z, 1),))[:z].copy(),
           np.ctypeslib.as_array(va, shape=(max(z, 1),))[:z].copy())
    for p in (rp, ci, va):
        L.tc_free(C.cast(p, C.c_void_p))
    return out


class Plan:
    """A matrix formatted and resident in device memory (tc_plan)."""

    def __init__(self, handle):
        self._h = handle

    # -- construction -------------------------------------------------------
    @classmethod
    def from_csr(cls, M, N, rowptr, col, val=None, prm=None, on_device=False, stream=None,
                 partition=True, keep_host=False):
        p = prm or params()
        if not partition:
            p.flags |= TC_FLAG_NO_PARTITION
        if keep_host:
            p.flags |= TC_FLAG_KEEP_HOST
        keep = []
        if not on_device:
            rowptr = np.ascontiguousarray(rowptr, np.int32)
            col = np.ascontiguousarray(col, np.int32)
            keep += [rowptr, col]
            if val is not None:
                val = np.ascontiguousarray(val, np.float32)
                keep.append(val)
        nnz = int(rowptr[M]) if not on_device else int(rowptr[M].item())
        h = C.c_void_p()
        check(lib().tc_plan_create(M, N, nnz, _ptr(rowptr), _ptr(col), _ptr(val),
                                   1 if on_device else 0, C.byref(p), _stream(stream),
                                   C.byref(h)))
        return cls(h)

    @classmethod
    def from_format(cls, M, N, fmt, prm=None, stream=None):
        """fmt: dict with the TaiChi_new fields (numpy arrays)."""
        f = Format()
        keep = {}
        for k in ("dia_shapes", "num_negs", "dense_nnz", "zero_elements", "sparse_nnz",
                  "row_start", "row_stop"):
            setattr(f, k, int(fmt[k]))
        for k in ("xStart", "yStart", "xStop", "nDiasPtr", "neg_offsets", "csrRow", "csrCol"):
            a = fmt.get(k)
            if a is None:
                continue
            a = np.ascontiguousarray(a, np.int32)
            if a.size == 0:
                a = np.zeros(1, np.int32)
            keep[k] = a
            setattr(f, k, a.ctypes.data_as(_IP))
        h = C.c_void_p()
        check(lib().tc_plan_from_format(M, N, C.byref(f), C.byref(prm or params()),
                                        _stream(stream), C.byref(h)))
        return cls(h)

    def close(self):
        if self._h:
            lib().tc_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # -- queries ------------------------------------------------------------
    def info(self):
        i = PlanInfo()
        check(lib().tc_plan_info_get(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in PlanInfo._fields_}

    def export(self):
        """Host copy of the plan's format as a dict (TaiChi_new fields)."""
        i = self.info()
        s, ng, M = i["dia_shapes"], i["num_negs"], i["M"]
        arrs = {"xStart": np.zeros(max(s, 1), np.int32), "yStart": np.zeros(max(s, 1), np.int32),
                "xStop": np.zeros(max(s, 1), np.int32), "nDiasPtr": np.zeros(s + 1, np.int32),
                "neg_offsets": np.zeros(max(ng, 1), np.int32),
                "csrRow": np.zeros(M + 1, np.int32),
                "csrCol": np.zeros(max(i["nnz_csr"], 1), np.int32)}
        check(lib().tc_plan_export(self._h, *[arrs[k].ctypes.data for k in
                                              ("xStart", "yStart", "xStop", "nDiasPtr",
                                               "neg_offsets", "csrRow", "csrCol")]))
        d = {k: i[k] for k in ("dia_shapes", "num_negs", "dense_nnz", "zero_elements",
                               "sparse_nnz", "row_start", "row_stop")}
        d["xStart"], d["yStart"], d["xStop"] = arrs["xStart"][:s], arrs["yStart"][:s], arrs["xStop"][:s]
        d["nDiasPtr"] = arrs["nDiasPtr"] if s > 0 else np.zeros(0, np.int32)
        d["neg_offsets"] = arrs["neg_offsets"][:ng]
        d["csrRow"] = arrs["csrRow"]
        d["csrCol"] = arrs["csrCol"][:i["nnz_csr"]]
        return d

    def thumbnail(self, height=512):
        W, n = C.c_int(), C.c_int()
        check(lib().tc_plan_thumbnail(self._h, None, C.byref(W), None, C.byref(n)))
        corners = np.zeros((max(n.value, 1), 4), np.int32)
        st = np.zeros((5, height, max(W.value, 1)), np.uint8)
        check(lib().tc_plan_thumbnail(self._h, st.ctypes.data, C.byref(W), corners.ctypes.data,
                                      C.byref(n)))
        return corners[:n.value], st if W.value else None

    # -- multiply -----------------------------------------------------------
    def spmv(self, x, y, stream=None):
        check(lib().tc_spmv(self._h, _ptr(x), _ptr(y), _stream(stream)))

    def spmv_f64(self, x, y, stream=None):
        """y = A x with float64 device vectors (x: N, y: M)."""
        check(lib().tc_spmv_f64(self._h, _ptr(x), _ptr(y), _stream(stream)))

    def check(self):
        """Raises if a multiply of this plan reported a device-side timeout."""
        check(lib().tc_plan_check(self._h))

    # -- plan files ---------------------------------------------------------
    def save(self, path):
        check(lib().tc_plan_save(self._h, os.fsencode(path)))

    @classmethod
    def load(cls, path, prm=None, stream=None):
        h = C.c_void_p()
        check(lib().tc_plan_load(os.fsencode(path), C.byref(prm) if prm is not None else None,
                                 _stream(stream), C.byref(h)))
        return cls(h)

    def spmv_host(self, x, y, stream=None):
        check(lib().tc_spmv_host(self._h, _ptr(x), _ptr(y), _stream(stream)))

    def spmv_host_async(self, x, y, slot, stream):
        """Enqueue copy-in, multiply, copy-out through staging slot 0..3;
        y is ready once `stream` has reached this point."""
        check(lib().tc_spmv_host_async(self._h, _ptr(x), _ptr(y), slot, _stream(stream)))

    def spmm(self, X, Y, k=None, ldx=None, ldy=None, stream=None):
        if k is None:
            k = X.shape[1]
        ldx = ldx or X.shape[1]
        ldy = ldy or Y.shape[1]
        check(lib().tc_spmm(self._h, _ptr(X), ldx, k, _ptr(Y), ldy, _stream(stream)))
