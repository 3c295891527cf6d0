"""The reference's own GPU multiply on this machine's GPU (context for the
benchmark's reference arm; test infrastructure, never the product).

Runs the unmodified reference (TaiChi.cu, built from its sources into
oracle/_ref by oracle/build.py): partition_shapes on the host, then
taichi_SpMV (TaiChi.cu:1331-1456), which uploads the format, makes 10 warm-up
and 500 event-timed launches and prints their mean as `spmv_time=<ms>`.
taichi_SpMV ends with cudaDeviceReset, so this runs in its own process:

    python -m oracle.ref_gpu --workload rmat20

prints one JSON line: the printed times, the GB/s of the printed multiply
time over the same algorithmic bytes as the benchmark, and the result's
normwise error against the FP64 oracle.
"""
import argparse
import json
import os
import re
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def matrix(name):
    from taichi_b200 import matgen
    if name == "rmat20":
        return matgen.rmat(20, 16, 0.499, 0.001, 0.001, seed=1)
    if name == "small":
        return matgen.diag_plus_random(65536, seed=0)
    raise SystemExit("unknown workload " + name)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="rmat20")
    args = ap.parse_args()
    import ctypes as C
    import oracle
    R = oracle.ref_lib()
    if R is None:
        print(json.dumps({"unavailable": "oracle/_ref was not built"}))
        return
    M, N, rp, col = matrix(args.workload)
    x = np.random.default_rng(0).uniform(-1, 1, N).astype(np.float32)
    rp = np.array(rp, np.int32, copy=True)
    col = np.array(col, np.int32, copy=True)
    val = np.ones(max(int(rp[M]), 1), np.float32)
    R.ref_clear_shapes()                       # getSdf: the oracle's restatement of the morphology
    work = tempfile.mkdtemp()
    cwd = os.getcwd()
    os.chdir(work)                             # partition_shapes appends to ./nnz_density.txt
    try:
        t = R.ref_partition(M, N, int(rp[M]), rp, col, val)
    finally:
        os.chdir(cwd)
    y = np.zeros(M, np.float32)
    # taichi_SpMV prints with printf: capture this process's stdout at the fd
    sys.stdout.flush()
    r, w = os.pipe()
    saved = os.dup(1)
    os.dup2(w, 1)
    try:
        R.ref_taichi_spmv(M, N, t, x, y)
        C.CDLL(None).fflush(None)
    finally:
        os.dup2(saved, 1)
        os.close(w)
    out = os.read(r, 1 << 16).decode(errors="replace")
    os.close(r)
    m = re.search(r"transfer_time:([0-9.]+)\s+spmv_time=([0-9.]+)", out)
    if not m:
        print(json.dumps({"unavailable": "no timing line from taichi_SpMV: " + out.strip()[-200:]}))
        return
    transfer_ms, spmv_ms = float(m.group(1)), float(m.group(2))
    y64 = oracle.spmv_csr_f64(M, rp, col, x.astype(np.float64))
    rel = float(np.linalg.norm(y - y64) / np.linalg.norm(y64))
    nbytes = 4 * (M + 1) + 4 * int(rp[M]) + 4 * N + 4 * M
    print(json.dumps({"workload": args.workload, "spmv_time_ms": spmv_ms, "transfer_time_ms": transfer_ms,
                      "gbs": round(nbytes / (spmv_ms * 1e-3) / 1e9, 1) if spmv_ms > 0 else None,
                      "normwise_rel_err_vs_fp64": rel,
                      "timing": "TaiChi.cu:1400-1420: mean of 500 event-timed launches after 10 warm-ups",
                      "build": "TaiChi.cu compiled unmodified for sm_100a (oracle/build.py)"}))


if __name__ == "__main__":
    main()
