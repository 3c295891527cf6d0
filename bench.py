"""Benchmark of the B200 TaiChi binary SpMV.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload rmat20|rmat20_selfloops|mesh|small]

A step is one SpMV y = A x of the workload's matrix.  Default workload: the
R-MAT scale-20 graph (1,048,576 rows, edge factor 16, a=0.499, b=c=0.001,
seed 1, self-loops and duplicates removed), formatted by the GPU partitioner,
FP32 x uniform in [-1, 1].

`value` is SpMV GB/s (algorithmic bytes / device time per SpMV), inputs
resident in HBM; the timed region replays a CUDA graph of back-to-back SpMVs
that rotate over enough resident copies of the matrix and vectors (> 2x the
126 MB L2) that every SpMV reads its operands from HBM.  `e2e` is the same
metric through the host-vector API: every step copies its x in from pinned
host memory and gets its y out, through tc_spmv_host_async with 2-4 staging
slots on as many streams, y either copied out ("copy") or stored by the
multiply straight into the pinned buffer ("mapped", TC_FLAG_HOST_Y_MAPPED);
the fastest (form, slots) is the headline and all are listed;
`e2e.sync_value` is the synchronous tc_spmv_host, one step at a time.
With --impl reference the reference's CPU SpMV loop (main.cu:61-69, restated
in the oracle) runs on all host cores on the same matrix.

One JSON line on stdout (rank 0).  Multi-GPU (torchrun): independent replicas,
one per GPU, max time over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from taichi_b200 import replicas, workloads  # noqa: E402  (plain Python; loads no CUDA library)

METRIC = "SpMV GB/s (% of HBM peak) at R-MAT scale 20"
L2_BYTES = 126 * 2 ** 20


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def make_matrix(name):
    from taichi_b200 import matgen
    if name == "rmat20":
        return matgen.rmat(20, 16, 0.499, 0.001, 0.001, seed=1), \
            "R-MAT scale 20, ef 16, a=0.499 b=c=0.001, seed 1, no self-loops/duplicates"
    if name == "rmat20_selfloops":
        return matgen.rmat(20, 16, 0.499, 0.001, 0.001, seed=1, self_loops=True), \
            "R-MAT scale 20 with self-loops kept (diagonal variant)"
    if name == "mesh":
        return matgen.mesh9(2048, 0.02, seed=2), "9-point stencil 2048^2, 2% rows permuted, seed 2"
    if name == "small":
        return matgen.diag_plus_random(65536, seed=0), "n=65536, diagonals -3..+4 + 10 random/row, seed 0"
    raise SystemExit("unknown workload " + name)


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None

    def stop(self):
        if not self.p:
            return None
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
            out, _ = self.p.communicate()
        rows = [r.split(", ") for r in out.strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def graph_len(steps, cap=4096, least=256):
    """SpMVs per captured graph: all `steps` when that is at most `cap`, else
    the largest divisor of `steps` in [least, cap] (so whole replays make
    exactly `steps`), else all `steps` in one graph."""
    if steps <= cap:
        return steps
    for d in range(cap, least - 1, -1):
        if steps % d == 0:
            return d
    return steps


def cpu_baseline(M, N, rp, col, x, seconds, threads):
    """The reference's CPU SpMV loop (main.cu:61-69, restated in the oracle)
    on a bounded sample: as many whole SpMVs as fit in `seconds`."""
    import oracle
    y = np.empty(M, np.float32)
    nbytes = 4 * (M + 1) + 4 * int(rp[M]) + 4 * N + 4 * M
    reps = 0
    t0 = time.perf_counter()
    while True:
        if threads == 1:
            oracle.lib().or_spmv_csr_f32_serial(M, rp, col, x, y)
        else:
            oracle.lib().or_spmv_csr_f32_omp(M, rp, col, x, y, threads)
        reps += 1
        dt = time.perf_counter() - t0
        if dt >= seconds:
            break
    return nbytes * reps / dt / 1e9, reps, dt


def run_reference(args, rank):
    """--impl reference: the reference's CPU SpMV on all host cores."""
    if rank != 0:
        return
    (M, N, rp, col), desc = make_matrix(args.workload)
    x = np.random.default_rng(0).uniform(-1, 1, N).astype(np.float32)
    threads = os.cpu_count() or 1
    import oracle
    y = np.empty(M, np.float32)
    for _ in range(max(args.warmup, 3)):
        oracle.lib().or_spmv_csr_f32_omp(M, rp, col, x, y, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        oracle.lib().or_spmv_csr_f32_omp(M, rp, col, x, y, threads)
    dt = time.perf_counter() - t0
    nbytes = 4 * (M + 1) + 4 * int(rp[M]) + 4 * N + 4 * M
    val = nbytes * args.steps / dt / 1e9
    line = {"impl": "reference", "metric": METRIC, "value": round(val, 3), "unit": "GB/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic: " + desc,
            "config": {"workload": args.workload + "_cpu_csr_spmv", "M": M, "N": N,
                       "nnz": int(rp[M]), "bytes_per_spmv": nbytes},
            "cpu_baseline": {"value": round(val, 3), "unit": "GB/s", "cores": threads,
                             "kind": "port",
                             "sample": "%d whole SpMVs of the workload (main.cu:61-69 loop, "
                                       "rows split over %d OpenMP threads)" % (args.steps, threads)},
            "e2e": {"value": round(val, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    # the partition on the host, as the reference runs it (partition_shapes,
    # TaiChi.cu:313-612, with getSdf's thumbnail, morphology and contours):
    # one whole partition of the workload by the oracle's sequential
    # restatement, beside the GPU partitioner's partition_ms of the other arm
    t0 = time.perf_counter()
    fmt, _ = oracle.partition(M, N, rp, col)
    line["partition_baseline"] = {"ms": round((time.perf_counter() - t0) * 1e3, 1), "cores": 1,
                                  "kind": "port", "dia_shapes": int(fmt["dia_shapes"]),
                                  "sample": "one partition_shapes of the workload (oracle restatement, "
                                            "sequential)"}
    if args.workload in ("rmat20", "small") and os.path.exists("/dev/nvidiactl") and not args.no_ref_gpu:
        line["reference_gpu"] = reference_gpu(args.workload)
    print(json.dumps(line), flush=True)


def reference_gpu(workload):
    """Context beside the reference arm: the reference's own CUDA multiply
    (TaiChi.cu compiled unmodified for sm_100a, oracle/_ref) on the same
    matrix, timed by the reference itself (its printed spmv_time), in a child
    process because taichi_SpMV ends with cudaDeviceReset."""
    try:
        r = subprocess.run([sys.executable, "-m", "oracle.ref_gpu", "--workload", workload], cwd=ROOT,
                           stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, timeout=300)
    except subprocess.TimeoutExpired:
        return {"unavailable": "oracle.ref_gpu did not finish in 300 s"}
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if r.returncode != 0 or not lines:
        return {"unavailable": "oracle.ref_gpu exited %d: %s" % (r.returncode, r.stderr.strip()[-300:])}
    return json.loads(lines[-1])


def run_ours(args, rank, world, local_rank):
    import torch
    import taichi_b200 as tc

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    (M, N, rp, col), desc = make_matrix(args.workload)
    rng = np.random.default_rng(0)
    x_host = rng.uniform(-1, 1, N).astype(np.float32)

    # format build + GPU partition (timed once; not part of a step)
    stream = torch.cuda.Stream(dev)
    t0 = time.perf_counter()
    over = {} if args.tile_mode is None else {"tile_mode": args.tile_mode}
    if args.tile_rows is not None:
        over["tile_rows"] = args.tile_rows
    if args.rows_strided:
        over["flags"] = tc.TC_FLAG_ROWS_STRIDED
    if args.no_direct:
        over["flags"] = over.get("flags", 0) | tc.TC_FLAG_NO_DIRECT
    if args.no_window:
        over["flags"] = over.get("flags", 0) | tc.TC_FLAG_NO_WINDOW
    if args.window:
        over["flags"] = over.get("flags", 0) | tc.TC_FLAG_WINDOW
    if args.wide_fixed:
        over["flags"] = over.get("flags", 0) | tc.TC_FLAG_WIDE_FIXED
    if args.wide_bounds:
        over["flags"] = over.get("flags", 0) | tc.TC_FLAG_WIDE_BOUNDS
    for on, f in ((args.rows, tc.TC_FLAG_ROWS), (args.no_rows, tc.TC_FLAG_NO_ROWS),
                  (args.no_prefetch, tc.TC_FLAG_NO_PREFETCH), (args.no_param_starts, tc.TC_FLAG_NO_PARAM_STARTS)):
        if on:
            over["flags"] = over.get("flags", 0) | f
    if args.tile_nnz is not None:
        over["tile_nnz"] = args.tile_nnz
    if args.rows_w is not None:
        over["rows_w"] = args.rows_w
    if args.ctas_per_sm is not None:
        over["ctas_per_sm"] = args.ctas_per_sm
    prm = tc.params(**over)
    plan0 = tc.Plan.from_csr(M, N, rp, col, prm=prm, stream=stream)
    partition = "gpu"
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t0
    info = plan0.info()
    bytes_per = info["spmv_bytes"]
    fmt = plan0.export()

    # rotating resident copies so that every SpMV reads from HBM
    ncopy = max(2, int(np.ceil(2.0 * L2_BYTES / bytes_per)))
    ncopy = min(ncopy, 64)
    plans = [plan0] + [tc.Plan.from_format(M, N, fmt, prm=prm, stream=stream) for _ in range(ncopy - 1)]
    xs = [torch.from_numpy(x_host).to(dev) for _ in range(ncopy)]
    ys = [torch.empty(M, dtype=torch.float32, device=dev) for _ in range(ncopy)]

    # correctness guard on the benchmark input (FP64 oracle only in tests;
    # here the integer-exact identity y(x=1) = row lengths)
    ones = torch.ones(N, device=dev)
    yo = torch.empty(M, device=dev)
    plan0.spmv(ones, yo, stream=stream)
    torch.cuda.synchronize()
    assert np.array_equal(yo.cpu().numpy(), np.diff(rp).astype(np.float32)), "SpMV check failed"

    with torch.cuda.stream(stream):
        for i in range(max(args.warmup, 3)):
            plans[i % ncopy].spmv(xs[i % ncopy], ys[i % ncopy], stream=stream)
    torch.cuda.synchronize()

    # The timed multiplies are captured in a CUDA graph and replayed on the
    # device back to back.  Up to 8192 steps: one graph of LEAD untimed
    # multiplies, exactly --steps timed ones and LEAD untimed ones.  The two
    # timing events are graph nodes on a side branch: each is recorded when
    # the multiply before it has completed, without holding back the next
    # multiply, which starts under programmatic dependent launch while its
    # predecessor drains.  The span runs from the completion of the last
    # multiply before the timed ones to the completion of the last timed
    # one -- exactly --steps multiplies in steady state, with neither the
    # host's graph submission nor the graph's start-up in it.  (Events on
    # the chain itself would make the first timed multiply wait for its
    # predecessor to finish: that figure is reported beside it as
    # `chain_bracket_gbs`.)  More steps: a graph of G multiplies (G the
    # largest divisor of steps up to 4096) replayed steps / G times between
    # two stream events, after one untimed replay that keeps the device busy
    # while the host submits the timed ones.
    LEAD = 16
    in_graph = args.steps <= 8192
    G = args.steps if in_graph else graph_len(args.steps)
    reps = args.steps // G
    ev0 = torch.cuda.Event(enable_timing=True, external=in_graph)
    ev1 = torch.cuda.Event(enable_timing=True, external=in_graph)
    side = torch.cuda.Stream(device=dev)

    def spmv_i(i):
        plans[i % ncopy].spmv(xs[i % ncopy], ys[i % ncopy], stream=torch.cuda.current_stream())

    def mark(ev):
        """Records ev on a side branch after everything captured so far."""
        f = torch.cuda.Event()
        f.record(stream)
        side.wait_event(f)
        ev.record(side)

    g_main = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g_main, stream=stream):
        if in_graph:
            for i in range(LEAD):
                spmv_i(i)
            mark(ev0)
            for i in range(args.steps):
                spmv_i(LEAD + i)
            mark(ev1)
            for i in range(LEAD):
                spmv_i(LEAD + args.steps + i)
            j = torch.cuda.Event()
            j.record(side)
            stream.wait_event(j)
        else:
            for i in range(G):
                spmv_i(i)
    with torch.cuda.stream(stream):
        g_main.replay()
    torch.cuda.synchronize()

    clocks = Clocks(local_rank)
    clocks.start()
    time.sleep(0.3)
    replicas.barrier(world)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):        # graph replays run on the current stream
        if in_graph:
            g_main.replay()
        else:
            g_main.replay()
            ev0.record(stream)
            for _ in range(reps):
                g_main.replay()
            ev1.record(stream)
    torch.cuda.synchronize()
    replicas.barrier(world)
    ms = ev0.elapsed_time(ev1)
    cl = clocks.stop()
    chain_ms = None
    if in_graph:                            # context: the events on the chain itself
        c0 = torch.cuda.Event(enable_timing=True, external=True)
        c1 = torch.cuda.Event(enable_timing=True, external=True)
        g_chain = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g_chain, stream=stream):
            for i in range(LEAD):
                spmv_i(i)
            c0.record()
            for i in range(args.steps):
                spmv_i(LEAD + i)
            c1.record()
        with torch.cuda.stream(stream):
            g_chain.replay()
            torch.cuda.synchronize()
            g_chain.replay()
        torch.cuda.synchronize()
        chain_ms = c0.elapsed_time(c1)
        del g_chain
    ms = replicas.max_over_ranks(ms, world, device=dev)    # the slowest replica bounds the job
    ms_step = ms / args.steps
    gbs = bytes_per / (ms_step * 1e-3) / 1e9 * world
    peak, peak_kind = load_peaks()

    # warm-L2 figure (same copy every time) for context
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    gw = torch.cuda.CUDAGraph()
    with torch.cuda.graph(gw, stream=stream):
        for _ in range(256):
            plan0.spmv(xs[0], ys[0], stream=torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        gw.replay()
        torch.cuda.synchronize()
        ev0.record(stream)
        gw.replay()
        ev1.record(stream)
    torch.cuda.synchronize()
    warm_ms = ev0.elapsed_time(ev1) / 256

    # end to end through the public host API (pinned host buffers): every step
    # copies its x in and gets its y out.  Two forms of the same call,
    # tc_spmv_host_async with S staging slots on as many streams: "copy" (the
    # multiply writes a device y, a copy brings it out) and "mapped" (a plan
    # with TC_FLAG_HOST_Y_MAPPED: the multiply stores y straight into the
    # pinned host buffer over the host link).  Each form runs with S = 2, 3
    # and 4 slots (or --e2e-slots alone), 400 pipelined calls each; the
    # headline is the fastest (form, S) on this box, and every pair is
    # reported, with the synchronous tc_spmv_host of each form beside them.
    slot_counts = [args.e2e_slots] if args.e2e_slots else [2, 3, 4]
    Smax = max(slot_counts)
    streams = [stream] + [torch.cuda.Stream(dev) for _ in range(Smax - 1)]
    hxs = [torch.from_numpy(x_host).pin_memory() for _ in range(Smax)]
    hys = [torch.empty(M, dtype=torch.float32).pin_memory() for _ in range(Smax)]
    e2e_steps = 400
    plan_m = tc.Plan.from_format(M, N, fmt, prm=tc.params(**dict(over, flags=over.get("flags", 0) |
                                                                  tc.TC_FLAG_HOST_Y_MAPPED)), stream=stream)
    e2e_forms, e2e_y = {}, {}
    for form, pl in (("copy", plan0), ("mapped", plan_m)):
        for _ in range(3):
            pl.spmv_host(hxs[0], hys[0], stream=stream)
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            pl.spmv_host(hxs[0], hys[0], stream=stream)
        sync_s = (time.perf_counter() - t0) / e2e_steps
        for S in slot_counts:
            for i in range(2 * S):
                pl.spmv_host_async(hxs[i % S], hys[i % S], i % S, streams[i % S])
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for i in range(e2e_steps):
                pl.spmv_host_async(hxs[i % S], hys[i % S], i % S, streams[i % S])
            for st_ in streams[:S]:
                st_.synchronize()
            e2e_s = (time.perf_counter() - t0) / e2e_steps
            pl.check()
            for k in range(1, S):
                assert np.array_equal(hys[0].numpy(), hys[k].numpy()), "pipelined host multiply mismatch"
            e2e_forms["%s/%d" % (form, S)] = {"gbs": bytes_per / e2e_s / 1e9 * world, "ms": e2e_s * 1e3,
                                              "sync_gbs": bytes_per / sync_s / 1e9 * world}
        e2e_y[form] = hys[0].numpy().copy()
    assert np.array_equal(e2e_y["copy"], e2e_y["mapped"]), "mapped-y multiply mismatch"
    plan_m.close()
    e2e_best = max(e2e_forms, key=lambda f: e2e_forms[f]["gbs"])
    e2e_gbs = e2e_forms[e2e_best]["gbs"]
    e2e_s = e2e_forms[e2e_best]["ms"] * 1e-3
    e2e_sync_gbs = e2e_forms[e2e_best]["sync_gbs"]

    # DRAM bytes per launch of the multiply from one ncu capture of this
    # workload with the default parameters (profiles/traffic.json)
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf) and not over:
        with open(tf) as f:
            traffic = json.load(f).get(args.workload)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, n, dt = cpu_baseline(M, N, rp, col, x_host, args.cpu_seconds, 1)
        cpu = {"value": round(v, 3), "unit": "GB/s", "cores": 1, "kind": "port",
               "sample": "%d whole SpMVs in %.1f s (main.cu:61-69 serial FP32 loop)" % (n, dt)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(gbs, 2), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: " + desc,
            "config": {"workload": args.workload + "_plain_hybrid_spmv", "M": M, "N": N,
                       "nnz": int(rp[M]), "partition": partition,
                       "dia_shapes": info["dia_shapes"], "num_negs": info["num_negs"],
                       "nnz_csr": info["nnz_csr"], "tiles": info["ntiles"], "kernel": tc.KERNEL_NAMES.get(info["kernel"]), "tile_mode": prm.tile_mode, "tile_rows": prm.tile_rows,
                       "tile_nnz": prm.tile_nnz, "flags": prm.flags,
                       "bytes_per_spmv": bytes_per,
                       # the same time over the plain-CSR bytes of the matrix
                       # (row pointers, every entry's column, x, y)
                       "effective_csr_gbs": round(gbs * (4 * (M + 1) + 4 * int(rp[M]) + 4 * N + 4 * M)
                                                  / bytes_per, 2),
                       "format_build_s": round(build_s, 3),
                       "partition_ms": info["partition_ms"],
                       "timing": ("one CUDA graph: %d untimed SpMVs, %d timed, %d untimed; events are "
                                  "graph nodes on a side branch after the last untimed and the last timed "
                                  "SpMV (steady state, completion to completion)" % (LEAD, args.steps, LEAD)
                                  if in_graph else
                                  "%d replays of a %d-SpMV graph after an untimed replay, stream events"
                                  % (reps, G)),
                       "l2": "rotating %d resident copies (%.0f MB) > 2x L2" % (
                           ncopy, ncopy * bytes_per / 1e6),
                       "warm_l2_gbs": round(bytes_per / (warm_ms * 1e-3) / 1e9, 1),
                       "chain_bracket_gbs": (round(bytes_per * args.steps / (chain_ms * 1e-3) / 1e9, 1)
                                             if chain_ms else None),
                       "parallelism": "replicas" if world > 1 else "single"},
            "roofline": {"bound": "hbm", "achieved": round(gbs / world, 2), "peak": peak,
                         "unit": "GB/s", "frac": round(gbs / world / peak, 4),
                         "peak_kind": peak_kind + " hbm_gbs (copy)", "traffic": traffic},
            "e2e": {"value": round(e2e_gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 4 * N,
                    "d2h_bytes_per_step": 4 * M, "ms_per_step": e2e_s * 1e3,
                    "api": "tc_spmv_host_async, %s form, %s slots on as many streams" % tuple(
                        e2e_best.split("/")),
                    "steps": e2e_steps,
                    "forms": {f: {"value": round(v["gbs"], 3), "ms_per_step": round(v["ms"], 4),
                                  "sync_value": round(v["sync_gbs"], 3)} for f, v in e2e_forms.items()},
                    "sync_value": round(e2e_sync_gbs, 3), "sync_api": "tc_spmv_host"},
            "gpu_launches": args.steps,
            "clocks": cl,
            "cpu_baseline": cpu,
        }
        if world == 1 and not args.no_forms and not over and args.workload == "rmat20":
            # the batched, served and SpMM forms, each measured on its own workload
            # with its own clocks record (GPU 0 only; replicas runs skip them)
            for p in plans:
                p.close()
            plans = []
            torch.cuda.empty_cache()
            line["spmm"] = spmm_record(args)
            line["batched"] = batched_record(args)
            line["served"] = served_record(args)
        print(json.dumps(line), flush=True)
    for p in plans:
        p.close()


def _events(torch, stream):
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    return a, b


def spmm_record(args):
    """Batched right-hand sides: Y = A X, X 4,194,304 x 64 FP32 row-major,
    uniform in [-1, 1], A the R-MAT scale-22 graph (a = 0.499, b = c =
    0.001, edge factor 16), formatted by the GPU partitioner."""
    import torch
    import taichi_b200 as tc
    dev = torch.device("cuda", 0)
    M, rp, col = tc.gen_rmat(22, 16, 0.499, 0.001, 0.001, seed=1)
    N, k = M, 64
    plan = tc.Plan.from_csr(M, N, rp, col)
    info = plan.info()
    X = torch.empty((N, k), device=dev).uniform_(-1, 1)       # 1 GiB, larger than L2
    Y = torch.empty((M, k), device=dev)
    stream = torch.cuda.Stream(dev)
    for _ in range(max(args.warmup, 3)):
        plan.spmm(X, Y, stream=stream)
    torch.cuda.synchronize()
    clocks = Clocks(0)
    clocks.start()
    time.sleep(0.2)
    a, b = _events(torch, stream)
    steps = max(3, min(args.steps, 200))
    a.record(stream)
    for _ in range(steps):
        plan.spmm(X, Y, stream=stream)
    b.record(stream)
    torch.cuda.synchronize()
    cl = clocks.stop()
    ms = a.elapsed_time(b) / steps
    nbytes = 4 * (M + 1) + 4 * info["nnz_csr"] + 4 * k * N + 4 * k * M
    peak, kind = load_peaks()
    gbs = nbytes / (ms * 1e-3) / 1e9
    plan.close()
    return {"metric": "SpMM GB/s (k=64) at R-MAT scale 22", "value": round(gbs, 1), "unit": "GB/s",
            "ms_per_step": ms, "steps": steps, "frac_of_hbm": round(gbs / peak, 4), "peak": peak,
            "peak_kind": kind, "clocks": cl,
            "config": {"workload": "rmat22_spmm_k64", "M": M, "nnz": int(rp[M]), "k": k,
                       "bytes_per_spmm": nbytes, "dia_shapes": info["dia_shapes"],
                       "l2": "X and Y are 1 GiB each, larger than L2"}}


def batched_record(args):
    """256 binary matrices of uneven size, each autotuned, multiplied by one
    replay of a CUDA graph of the batch launch (one work list over every
    matrix's tiles), against a graph of one launch per matrix."""
    import ctypes as C
    import torch
    import taichi_b200 as tc
    dev = torch.device("cuda", 0)
    mats = workloads.pool_matrices("batch", 256, 7)
    t0 = time.perf_counter()
    plans, xs, ys, nbytes, tuned = [], [], [], 0, 0
    for name, M, rp, col in mats:
        r = tc.tune(M, M, rp, col, max_trials=args.tune_trials) if args.tune_trials > 0 else None
        prm = r.params if r is not None else tc.params()
        tuned += r is not None
        p = tc.Plan.from_csr(M, M, rp, col, prm=prm)
        plans.append(p)
        xs.append(torch.empty(M, device=dev).uniform_(-1, 1))
        ys.append(torch.empty(M, device=dev))
        nbytes += p.info()["spmv_bytes"]
    build_s = time.perf_counter() - t0
    n = len(plans)
    H = (C.c_void_p * n)(*[p.handle.value for p in plans])
    X = (C.c_void_p * n)(*[x.data_ptr() for x in xs])
    Yp = (C.c_void_p * n)(*[y.data_ptr() for y in ys])
    b = C.c_void_p()
    tc.check(tc.lib().tc_batch_create(n, H, X, Yp, C.byref(b)))
    stream = torch.cuda.Stream(dev)
    for _ in range(3):
        tc.check(tc.lib().tc_batch_graph_launch(b, C.c_void_p(stream.cuda_stream)))
    torch.cuda.synchronize()
    steps = max(3, min(args.steps, 500))
    clocks = Clocks(0)
    clocks.start()
    time.sleep(0.2)
    a, e = _events(torch, stream)
    a.record(stream)
    for _ in range(steps):
        tc.check(tc.lib().tc_batch_graph_launch(b, C.c_void_p(stream.cuda_stream)))
    e.record(stream)
    torch.cuda.synchronize()
    ms_batch = a.elapsed_time(e) / steps
    # plain: one multiply launch per matrix, back to back (captured in a graph)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        for p, x, y in zip(plans, xs, ys):
            p.spmv(x, y, stream=torch.cuda.current_stream())
    with torch.cuda.stream(stream):
        g.replay()
        torch.cuda.synchronize()
        a.record(stream)
        for _ in range(steps):
            g.replay()
        e.record(stream)
    torch.cuda.synchronize()
    cl = clocks.stop()
    ms_plain = a.elapsed_time(e) / steps
    tc.check(tc.lib().tc_batch_destroy(b))
    del g
    for p in plans:
        p.close()
    return {"metric": "SpMVs/s over 256 uneven matrices (one graph replay per batch)",
            "matrices": n, "rows": int(sum(m[1] for m in mats)),
            "nnz": int(sum(int(m[2][-1]) for m in mats)),
            "batch_ms": ms_batch, "plain_ms": ms_plain,
            "batch_spmv_per_s": round(n / (ms_batch * 1e-3)),
            "plain_spmv_per_s": round(n / (ms_plain * 1e-3)),
            "batch_gbs": round(nbytes / (ms_batch * 1e-3) / 1e9, 1),
            "plain_gbs": round(nbytes / (ms_plain * 1e-3) / 1e9, 1),
            "speedup": round(ms_plain / ms_batch, 2), "tuned": tuned, "tune_trials": args.tune_trials,
            "build_s": round(build_s, 1), "steps": steps, "clocks": cl}


def highest_passing_rate(serve_at, rates, bisect_steps, limit_ms=2.0):
    """Sweeps `rates` (increasing) until two rates in a row reach a p99 of
    limit_ms (one failure alone may be a passing stall of the host, so the
    sweep goes on), then bisects between the highest passing rate and the
    first failing rate above it.  serve_at(rate) -> stats dict.  Returns
    (stats of the best passing run or None, list of (rate, stats) of every
    run)."""
    runs, best, fails = [], None, 0
    for rate in rates:
        st = serve_at(rate)
        runs.append((rate, st))
        if st["p99_ms"] < limit_ms:
            fails = 0
            if best is None or st["spmv_per_s"] > best[1]["spmv_per_s"]:
                best = (rate, st)
        else:
            fails += 1
            if fails == 2:
                break
    above = [r for r, st in runs if st["p99_ms"] >= limit_ms and best is not None and r > best[0]]
    if best is not None and above and bisect_steps > 0:
        a, b = best[0], min(above)
        for _ in range(bisect_steps):
            mid = 0.5 * (a + b)
            st = serve_at(mid)
            runs.append((mid, st))
            if st["p99_ms"] < limit_ms:
                a = mid
                if st["spmv_per_s"] > best[1]["spmv_per_s"]:
                    best = (mid, st)
            else:
                b = mid
    return (best[1] if best else None), runs


def served_record(args):
    """Poisson arrivals of SpMV requests over a pool of 48 resident matrices
    (Zipf(1.1) choice, a fresh x per request): the highest arrival rate whose
    p99 latency stays under 2 ms, for continuous batching (online submit,
    server-side dispatcher) and for the plain form (one synchronous request
    at a time), with device vectors and with host vectors."""
    import torch
    import taichi_b200 as tc
    dev = torch.device("cuda", 0)
    mats = workloads.pool_matrices("serve", 48, 11)
    srv = tc.Server(contexts=args.serve_contexts, max_batch=args.serve_max_batch,
                    max_inflight=args.serve_inflight, arena_bytes=512 << 20, hbm_budget=96 << 30,
                    solo_bytes=int(args.serve_solo_mb * 2 ** 20))
    plans, ids = [], []
    for name, M, rp, col in mats:
        p = tc.Plan.from_csr(M, M, rp, col)
        plans.append(p)
        ids.append(srv.admit(p))
    rng = np.random.default_rng(5)
    pz = np.arange(1, len(mats) + 1, dtype=np.float64) ** -1.1
    pz /= pz.sum()
    # two x per matrix; enough y per matrix that requests in flight together
    # never share one (at most max_inflight * max_batch are in flight)
    in_flight = args.serve_inflight * args.serve_max_batch
    nbuf = [int(np.ceil(2 * pz[m] * in_flight)) + 2 for m in range(len(mats))]
    xh = [[torch.empty(m[1]).uniform_(-1, 1).pin_memory() for _ in range(2)] for m in mats]
    yh = [[torch.empty(m[1]).pin_memory() for _ in range(nbuf[i])] for i, m in enumerate(mats)]
    xd = [[x.to(dev) for x in pair] for pair in xh]
    yd = [[torch.empty(m[1], device=dev) for _ in range(nbuf[i])] for i, m in enumerate(mats)]
    nreq = args.requests
    keys = ("spmv_per_s", "p50_ms", "p99_ms", "mean_batch", "mean_service_ms", "mean_launch_us")
    out = {"requests": nreq, "pool": len(mats), "pool_rows": int(sum(m[1] for m in mats)),
           "contexts": args.serve_contexts, "max_batch": args.serve_max_batch,
           "max_inflight": args.serve_inflight, "solo_mb": args.serve_solo_mb,
           "bisection_steps": args.rate_search}
    clocks = Clocks(0)
    clocks.start()
    for form, bit, rates, XB, YB in (("device", tc.SERVE_DEVICE_VECTORS, args.device_rates, xd, yd),
                                     ("host", 0, args.rates, xh, yh)):
        rec = {}
        for mode, name in ((0, "batched"), (1, "plain")):
            def serve_at(rate, mode=mode):
                matrix = rng.choice(len(mats), size=nreq, p=pz)
                arrival = np.cumsum(rng.exponential(1.0 / rate, nreq))
                cnt = np.zeros(len(mats), np.int64)
                xs, ys = [], []
                for i, m in enumerate(matrix):
                    xs.append(XB[m][i & 1])
                    ys.append(YB[m][cnt[m] % nbuf[m]])
                    cnt[m] += 1
                st, _ = srv.run(arrival, [ids[m] for m in matrix], xs, ys, mode=mode | bit)
                return st
            best, runs = highest_passing_rate(serve_at, rates, args.rate_search)
            rec[name] = dict({k: round(best[k], 4) for k in keys} if best else {"spmv_per_s": 0.0},
                             runs=[[round(r, 1)] + [round(st[k], 4) for k in keys] for r, st in runs])
        pl = rec["plain"]["spmv_per_s"]
        rec["ratio"] = round(rec["batched"]["spmv_per_s"] / pl, 2) if pl else None
        out[form] = rec
    out["clocks"] = clocks.stop()
    out["runs_columns"] = ["rate"] + list(keys)
    srv.close()
    for p in plans:
        p.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--warmup", type=int, default=50)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rmat20")
    ap.add_argument("--form", default="plain", choices=["plain", "spmm", "batched", "served"],
                    help="plain: the headline line (with the spmm, batched and served records "
                         "unless --no-forms); others: that record alone")
    ap.add_argument("--no-forms", action="store_true",
                    help="plain line only, without the spmm / batched / served records")
    ap.add_argument("--tune-trials", type=int, default=4, help="batched form: tuner trials per matrix")
    ap.add_argument("--requests", type=int, default=20000, help="served form: requests per rate")
    ap.add_argument("--rates", type=float, nargs="+",
                    default=[2000, 4000, 6000, 9000, 13500, 20000, 30000, 45000, 67500, 100000],
                    help="served form, host vectors: arrival rates swept (requests/s)")
    ap.add_argument("--device-rates", type=float, nargs="+",
                    default=[20000, 30000, 45000, 67500, 100000, 150000, 225000, 337500, 506250,
                             759375, 1139062],
                    help="served form, device vectors: arrival rates swept (requests/s)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="reference arm: skip the reference's own GPU multiply (context record)")
    ap.add_argument("--tile-mode", type=int, default=None, help="0 merge, 1 lanes, 2 stream")
    ap.add_argument("--tile-rows", type=int, default=None, help="most rows per multiply tile")
    ap.add_argument("--rows-strided", action="store_true", help="stream tiles: one row per thread")
    ap.add_argument("--tile-nnz", type=int, default=None, help="entry limit of a tile")
    ap.add_argument("--ctas-per-sm", type=int, default=None, help="resident CTAs per SM (persistent grids)")
    ap.add_argument("--no-direct", action="store_true", help="stream tiles only, no direct tiles")
    ap.add_argument("--no-window", action="store_true", help="never the window kernel")
    ap.add_argument("--window", action="store_true", help="the window kernel wherever rows fit its tiles")
    ap.add_argument("--wide-fixed", action="store_true",
                    help="wide plans: tiles of 4096 rows instead of two equal tiles per SM")
    ap.add_argument("--wide-bounds", action="store_true",
                    help="wide plans: tile word ranges in the launch parameters, words staged in shared memory")
    ap.add_argument("--rows", action="store_true", help="stream plans: the rows kernel whatever the row lengths")
    ap.add_argument("--no-rows", action="store_true", help="stream plans: never the rows kernel")
    ap.add_argument("--rows-w", type=int, default=None, help="the rows kernel: words of a row loaded together")
    ap.add_argument("--e2e-slots", type=int, default=None, choices=[1, 2, 3, 4],
                    help="end-to-end figure: staging slots (and streams) of tc_spmv_host_async "
                         "(default: 2, 3 and 4, the fastest reported)")
    ap.add_argument("--no-param-starts", action="store_true",
                    help="wide plans: tile word ranges for the prefetch from the tile records")
    ap.add_argument("--no-prefetch", action="store_true",
                    help="stream / rows kernels: no L2 prefetch of the operands a wave ahead")
    ap.add_argument("--serve-contexts", type=int, default=4, help="served form: launch contexts (streams)")
    ap.add_argument("--serve-max-batch", type=int, default=64, help="served form: most requests per launch")
    ap.add_argument("--serve-inflight", type=int, default=2, help="served form: batches on the GPU at once")
    ap.add_argument("--serve-solo-mb", type=float, default=16.0,
                    help="served form: matrices moving at least this many MB per SpMV get their own launch")
    ap.add_argument("--rate-search", type=int, default=4,
                    help="served form: bisection steps between the last passing and first failing rate")
    args = ap.parse_args()
    if args.impl == "ours" and args.form != "plain":
        rec = {"spmm": spmm_record, "batched": batched_record, "served": served_record}[args.form](args)
        print(json.dumps(dict(form=args.form, **rec)), flush=True)
        return
    rank, world, local_rank = replicas.env()
    if args.impl == "reference":
        run_reference(args, rank)           # rank 0 alone; no process group
        return
    rank, world, local_rank = replicas.init("nccl")
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        replicas.finish(world)


if __name__ == "__main__":
    main()
