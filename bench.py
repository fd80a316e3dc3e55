"""Benchmark of the B200 Sparse BLAS hot path.

Headline workload: FP64 CSR SpMV  y = 1.0*A*x + 0.0*y  on the 4,194,304-row
lognormal power-law matrix (row lengths: mean 16, sigma 1.5, clipped to
[1, 65536]; columns uniform without replacement; values N(0,1); x uniform
[-1,1]; seed 1).  One step = one SpMV over the whole matrix.

Metric: HBM GB/s by the algorithmic byte model
    bytes = nnz*(8 + 8) + (n+1)*8 + |x| + |y|      (int64 indices, FP64)
The inputs (1.18 GB) exceed the 126 MB L2, so no flush is needed between
steps (x, 33.5 MB, is meant to stay L2-resident and is counted once).

Arms:
  default          : this library (C ABI), inputs resident in HBM; plus an
                     end-to-end number through the same C ABI with x copied
                     host->device and y device->host inside every step: a
                     serving loop with two buffer sets, where step i+1's
                     copy-in and step i's copy-out overlap step i's product
                     (the serial copy-in / product / copy-out figure is kept
                     beside it).
  --impl reference : the reference's own serial CPU SpMV (compiled from its
                     sources into oracle/_ref) over all host cores, one
                     reference call per disjoint row block and thread.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SpMV/SpMM HBM GB/s vs ~8 TB/s"
WORKLOAD = "fp64_csr_spmv_powerlaw_4M"


def _env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic_record():
    path = os.path.join(ROOT, "profiles", "seg_kernel_fp64_powerlaw_4M_traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def _host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def max_over_ranks(value: float, world: int, device) -> float:
    """The largest of every rank's `value` (the job's time is its slowest
    rank's); every rank must call it, in the same order."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _matrix(seed=1):
    from asc_cpp_b200 import synthetic
    a = synthetic.power_law(4_194_304, 16.0, 1.5, 65_536, seed=seed, dtype=np.float64)
    rng = np.random.default_rng(seed + 1000)
    x = rng.uniform(-1.0, 1.0, a.cols)
    return a, x


class Clocks:
    """nvidia-smi sampling during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device_index = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.device_index), "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in getattr(self, "lines", []):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": mx or None, "reasons": sorted(reasons),
                "samples": len(sm)}


def run_reference(args, rank, world):
    """--impl reference: the reference's own CPU SpMV on the host cores."""
    if rank != 0:
        return 0
    from oracle import Reference, Restatement, build_oracle
    a, x = _matrix()
    threads = _host_threads()
    kind = "reference"
    if Reference.available():
        ref = Reference()
        handle = ref.blocks_prepare(a.rows, a.cols, a.ptr, a.idx, a.val, threads)
        run = lambda y: ref.blocks_run(handle, np.float64, 1.0, x, 0.0, y)  # noqa: E731
    else:  # compiled reference absent: the C restatement, serial
        kind, threads = "port", 1
        build_oracle.build_restatement()
        rs = Restatement()
        run = lambda y: rs.compat_spmv(a.ptr, a.idx, a.val, 1.0, x, 0.0, y)  # noqa: E731
    y = np.zeros(a.rows)
    sample = "full matrix"
    bytes_ = a.bytes_spmv(8)
    t0 = time.perf_counter()
    run(y)
    t_full = time.perf_counter() - t0
    # keep the whole run within about two minutes: if K full products would
    # take longer, each step runs the reference on a leading row block
    budget = 120.0 / max(1, args.steps + args.warmup)
    if t_full > budget:
        rows = max(1, int(a.rows * budget / t_full))
        nnz = int(a.ptr[rows])
        sub_ptr, sub_idx, sub_val = a.ptr[:rows + 1], a.idx[:nnz], a.val[:nnz]
        bytes_ = nnz * 16 + (rows + 1) * 8 + a.cols * 8 + rows * 8
        sample = f"first {rows} rows ({nnz} nnz) per step"
        if kind == "reference":
            ref.blocks_free(handle, np.float64)
            handle = ref.blocks_prepare(rows, a.cols, sub_ptr, sub_idx, sub_val, threads)
        else:
            run = lambda y: rs.compat_spmv(sub_ptr, sub_idx, sub_val, 1.0, x, 0.0, y)  # noqa: E731
    for _ in range(args.warmup):
        run(y)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        run(y)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * statistics.mean(times)
    gbs = bytes_ / (ms * 1e-3) / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(gbs, 3), "unit": "GB/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "rows": a.rows, "nnz": a.nnz,
                   "alpha": 1.0, "beta": 0.0, "bytes_per_step": bytes_},
        "cpu_baseline": {"value": round(gbs, 3), "unit": "GB/s", "cores": threads,
                         "kind": kind,
                         "sample": sample + ", one reference SpmvReference call per "
                                            "nnz-balanced row block per thread"},
        "e2e": {"value": round(gbs, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def headline_error(a, x, y_best, y_det, mode):
    """Error of the headline product against the FP64 oracle (the C
    restatement of SpmvReference; long double for the bound), and whether
    the DETERMINISTIC product equals the oracle bit for bit."""
    import oracle as orc
    rs = orc.Restatement()
    want = orc.compat_spmv_rows(rs, a.ptr, a.idx, a.val, 1.0, x, 0.0, np.zeros(a.rows))
    exact, absval = orc.extended_rows(rs, a.cols, a.ptr, a.idx, a.val, x)
    rep = orc.error_report(y_best, exact, absval, np.diff(a.ptr), np.float64, 1.0)
    rep.update({"mode": mode, "bitexact": bool(y_best.tobytes() == want.tobytes()),
                "deterministic_bitexact": bool(y_det.tobytes() == want.tobytes()),
                "bound": "|y - y_ref| <= gamma_{n+2} |alpha| sum|a x| per row",
                "oracle": "C restatement of SpmvReference (FP64), long double for the bound"})
    return rep


def spmv_error(a, x, got, transpose):
    """y = A x (or A^T x) from y = 0, DETERMINISTIC and BACKEND_DEFAULT, against
    the oracle: the C restatement in the data's precision for bit-exactness,
    its long-double sums for the bound gamma_{n+2} sum|a x| per output."""
    import oracle as orc
    rs = orc.Restatement()
    op = orc.OP_TRANSPOSE if transpose else orc.OP_NONE
    want = np.zeros(a.cols if transpose else a.rows, dtype=a.val.dtype)
    rs.standard_spmv(orc.CSR, op, a.rows, a.cols, a.ptr, a.idx, a.val, 1.0, x, want)
    exact, absval = rs.extended(op, a.rows, a.cols, a.ptr, a.idx, a.val, x)
    counts = np.bincount(a.idx, minlength=a.cols) if transpose else np.diff(a.ptr)
    rep = orc.error_report(got["default"], exact, absval, counts, a.val.dtype, 1.0)
    rep.update({"mode": "backend_default (plan)",
                "deterministic_bitexact": bool(got["deterministic"].tobytes() == want.tobytes()),
                "bound": "|y - y_ref| <= gamma_{n+2} sum|a x| per output",
                "oracle": "C restatement of asc::Spmv (blas.h:1607-1667), long double for the bound"})
    return rep


def batch_error(g, got, sample):
    """y = A_m x_m for `sample` matrices spread over the batch, both modes,
    against the oracle's compat form (the C restatement of
    CudaCsrSpmv's y = alpha A x + beta y in FP64): DETERMINISTIC bit for bit,
    BACKEND_DEFAULT within gamma_{n+2} sum|a x| per row."""
    import oracle as orc
    rs = orc.Restatement()
    ptr, idx, val, x = (g[k].cpu().numpy() for k in ("ptr", "idx", "val", "x"))
    count = len(g["rows"])
    worst, exact_all, outputs = 0.0, True, 0
    for m in np.linspace(0, count - 1, min(sample, count)).astype(np.int64):
        n, z = int(g["rows"][m]), int(g["nnz"][m])
        pb, nb, rb = int(g["ptr_base"][m]), int(g["nz_base"][m]), int(g["row_base"][m])
        p, i, v, xm = ptr[pb:pb + n + 1], idx[nb:nb + z], val[nb:nb + z], x[rb:rb + n]
        want = rs.compat_spmv(p, i, v, 1.0, xm, 0.0, np.zeros(n))
        exact_all &= got["deterministic"][rb:rb + n].tobytes() == want.tobytes()
        e, a = rs.extended(orc.OP_NONE, n, n, p, i, v, xm)
        rep = orc.error_report(got["default"][rb:rb + n], e, a, np.diff(p), np.float64, 1.0)
        worst = max(worst, rep["max_ratio_to_bound"])
        outputs += n
    return {"mode": "backend_default (batch kernel)", "max_ratio_to_bound": worst,
            "deterministic_bitexact": bool(exact_all), "outputs": outputs,
            "sample": f"{min(sample, count)} matrices spread over the batch",
            "bound": "|y - y_ref| <= gamma_{n+2} sum|a x| per row",
            "oracle": "C restatement of the compat SpMV (FP64), long double for the bound"}


def spmm_error(a, b, c, mode, sample_rows, tensor_cores=False):
    """Error of an SpMM result C = A B (FP32) against the FP64 oracle (the C
    restatement run in FP64 on the same inputs) on the first `sample_rows`
    rows, with the bound gamma_{n+2} sum|a b| (+ the FP64 oracle's own)."""
    import oracle as orc
    rs = orc.Restatement()
    rows = min(a.rows, sample_rows)
    ptr = a.ptr[:rows + 1]
    nnz = int(ptr[-1])
    idx, val = a.idx[:nnz], a.val[:nnz].astype(np.float64)
    b64 = b.astype(np.float64)
    ref = orc.standard_spmm_rows(rs, a.cols, ptr, idx, val, 1.0, b64, np.zeros((rows, b.shape[1])))
    absval = orc.standard_spmm_rows(rs, a.cols, ptr, idx, np.abs(val), 1.0, np.abs(b64),
                                    np.zeros((rows, b.shape[1])))
    counts = np.diff(ptr)[:, None]
    if tensor_cores:  # 3xTF32 on the tensor cores
        bound = ((counts + 64) * 2.0 ** -22 + orc.gamma(counts + 2, np.float64)) * absval
    else:
        bound = (orc.gamma(counts + 2, np.float32) + orc.gamma(counts + 2, np.float64)) * absval
    bound = bound + np.finfo(np.float32).tiny
    err = np.abs(c[:rows].astype(np.float64) - ref)
    return {"mode": mode, "max_abs": float(err.max()),
            "max_ratio_to_bound": float((err / bound).max()),
            "bound": "|c - c_ref| <= gamma_{n+2} sum|a b| per output (tensor-core 3xTF32: "
                     "(n+64) 2^-22 sum|a b|)",
            "sample": f"first {rows} rows", "oracle": "C restatement in FP64"}


def cusparse_leg(a, A, x, stream, bytes_step):
    """cuSPARSE SpMV (torch's CSR mat-vec) on the same device arrays: a
    library comparison, timed like the headline; never the product."""
    import torch
    try:
        with torch.cuda.stream(stream):
            t = torch.sparse_csr_tensor(A.offsets, A.indices, A.values, (a.rows, a.cols))
            torch.mv(t, x)
        stream.synchronize()

        def run():
            with torch.cuda.stream(stream):
                torch.mv(t, x)
        ms = _timer(stream, 20, 3)(run)
    except (RuntimeError, TypeError) as e:  # library refused the operands
        return {"cusparse_csr_mv_unavailable": str(e)[:120]}
    return {"cusparse_csr_mv_gbs": round(bytes_step / (ms * 1e-3) / 1e9, 2),
            "cusparse_csr_mv_ms": round(ms, 4),
            "note": "library comparison on the same arrays (torch CSR mat-vec), not the product"}


def selector_leg(count=40, seed=5, max_rows=1_000_000, reps=10):
    """The learned selector on the drop-in path, re-timed on this GPU: `count`
    matrices of the training families drawn with a seed the selector never saw
    (training used seed 4), each multiplied through CudaCsrSpmv (the C ABI
    entry a reference caller reaches) in BACKEND_DEFAULT mode with the shipped
    selector installed (the context's default), against the default variant
    forced and against exhaustive search on the same path (every candidate
    forced through CudaCsrSpmv and timed)."""
    import ctypes
    import torch
    from asc_cpp_b200 import selector as sel
    from asc_cpp_b200 import sparse_cuda as sc
    from asc_cpp_b200._abi import Determinism, Variant

    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    timed = _timer(stream, reps, 3)
    ctx = sc.SparseCudaContext.Create(0, stream=stream, determinism=Determinism.kBackendDefault)
    rng = np.random.default_rng(seed)
    variants = np.array([v for v, _ in sel.VARIANTS], np.int32)
    lanes = np.array([l for _, l in sel.VARIANTS], np.int32)
    rows = []
    for i in range(count):
        family = sel.FAMILIES[i % len(sel.FAMILIES)]
        n = int(np.exp(rng.uniform(np.log(10_000), np.log(max_rows))))
        dtype = torch.float64 if rng.random() < 0.5 else torch.float32
        with torch.cuda.stream(stream):
            m = sel.family_matrix(family, n, rng, dtype, 20_000_000, dev)
            x = (torch.rand(m.columns, device=dev, dtype=torch.float64) * 2 - 1).to(dtype)
            y = torch.zeros(m.rows, dtype=dtype, device=dev)
        stream.synchronize()
        xv = sc.CudaStridedVectorView(x, m.columns, writable=False)
        yv = sc.CudaStridedVectorView(y, m.rows)
        need = sc.CudaCsrSpmvWorkspaceSize(ctx, m, xv, yv)
        ws = torch.empty(max(need, 1), dtype=torch.uint8, device=dev)

        def product():
            sc.CudaCsrSpmv(ctx, 1.0, m, xv, 0.0, yv, ws, need)
        ctx.set_variant(Variant.kWarpTiles, 0)
        t_default = timed(product)
        ctx.set_variant(Variant.kAuto, 0)
        product()  # first sight of this matrix: the selection is enqueued
        stream.synchronize()
        t_pick = timed(product)  # the pick, once it has landed
        plan = sc.CsrPlan(ctx, m)  # the same selector on a plan: which variant it is
        v, l = ctypes.c_int32(), ctypes.c_int32()
        ctx.check(ctx._lib.asc_sb_plan_variant(plan.handle, ctypes.byref(v), ctypes.byref(l)))
        plan.close()
        # exhaustive on the same path: every candidate forced through CudaCsrSpmv
        forced = []
        for vv, ll in zip(variants, lanes):
            ctx.set_variant(int(vv), int(ll))
            forced.append(timed(product))
        ctx.set_variant(Variant.kAuto, 0)
        rows.append((family, m.rows, m.nnz, t_default, t_pick, float(min(forced)),
                     (int(v.value), int(l.value))))
        del m, x, y, ws
    ctx.close()
    d = np.array([r[3] for r in rows])
    p = np.array([r[4] for r in rows])
    b = np.array([r[5] for r in rows])
    best = np.minimum(b, np.minimum(d, p))
    return {"matrices": count, "seed": seed, "path": "CudaCsrSpmv (asc_sb_csr_spmv), "
            "BACKEND_DEFAULT, shipped selector installed at context creation",
            "geomean_speedup_vs_default": round(float(np.exp(np.log(d / p).mean())), 3),
            "total_time_speedup_vs_default": round(float(d.sum() / p.sum()), 3),
            "geomean_slowdown_vs_exhaustive": round(float(np.exp(np.log(p / best).mean())), 3),
            "within_10pct_of_exhaustive": round(float((p <= 1.1 * best).mean()), 3),
            "picks": {f"{v}/{l}": sum(1 for r in rows if r[6] == (v, l))
                      for v, l in sorted({r[6] for r in rows})}}


def cpu_baseline_sample(a, x):
    """The reference's serial CPU SpMV (1 core) on a bounded row sample."""
    from oracle import Reference, Restatement, build_oracle
    rows = min(a.rows, 1_048_576)
    nnz = int(a.ptr[rows])
    ptr, idx, val = a.ptr[:rows + 1], a.idx[:nnz], a.val[:nnz]
    y = np.zeros(rows)
    if Reference.available():
        ref, kind = Reference(), "reference"
        run = lambda: ref.compat_spmv(rows, a.cols, ptr, idx, val, 1.0, x, 0.0, y)  # noqa
    else:
        build_oracle.build_restatement()
        rs, kind = Restatement(), "port"
        run = lambda: rs.compat_spmv(ptr, idx, val, 1.0, x, 0.0, y)  # noqa
    run()
    times = []
    t_end = time.perf_counter() + 10.0
    while time.perf_counter() < t_end and len(times) < 20:
        t0 = time.perf_counter()
        run()
        times.append(time.perf_counter() - t0)
    bytes_ = nnz * 16 + (rows + 1) * 8 + a.cols * 8 + rows * 8
    gbs = bytes_ / statistics.median(times) / 1e9
    return {"value": round(gbs, 4), "unit": "GB/s", "cores": 1, "kind": kind,
            "sample": f"first {rows} rows ({nnz} nnz), median of {len(times)} calls"}


def run_gpu(args, rank, world):
    import torch
    import torch.distributed as dist
    from asc_cpp_b200 import _abi
    from asc_cpp_b200.sparse_cuda import (CsrPlan, CudaCsrSpmv, CudaCsrSpmvWorkspaceSize,
                                          CudaCsrArray, CudaStridedVectorView,
                                          SparseCudaContext)
    from asc_cpp_b200._abi import Determinism, Variant

    local = _env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    a_h, x_h = _matrix()
    stream = torch.cuda.Stream(device=dev)
    ctx = SparseCudaContext.Create(local, stream=stream, determinism=Determinism.kDeterministic)
    with torch.cuda.stream(stream):
        A = CudaCsrArray(a_h.rows, a_h.cols, torch.from_numpy(a_h.ptr).to(dev),
                         torch.from_numpy(a_h.idx).to(dev), torch.from_numpy(a_h.val).to(dev))
        x = torch.from_numpy(x_h).to(dev)
        y = torch.zeros(a_h.rows, dtype=torch.float64, device=dev)
    stream.synchronize()
    xv = CudaStridedVectorView(x, a_h.cols, writable=False)
    yv = CudaStridedVectorView(y, a_h.rows)
    bytes_step = a_h.bytes_spmv(8)

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        stream.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(steps):
            fn()
        stop.record(stream)
        stop.synchronize()
        torch.cuda.synchronize()
        ms = start.elapsed_time(stop) / steps
        return max_over_ranks(ms, world, dev)

    # -- variants (untimed selection pass, then the headline) --
    plan = CsrPlan(ctx, A)
    detail = {}

    def run_plan():
        plan.csr_spmv(1.0, xv, 0.0, yv)

    # every variant once (untimed selection pass); the fastest is the headline
    choices = {"row_ordered_bitexact": (Determinism.kDeterministic, Variant.kAuto, 0),
               "warp_tiles": (Determinism.kBackendDefault, Variant.kWarpTiles, 0),
               "merge_path": (Determinism.kBackendDefault, Variant.kMergePath, 0),
               "vector_8": (Determinism.kBackendDefault, Variant.kVector, 8),
               "vector_16": (Determinism.kBackendDefault, Variant.kVector, 16),
               "row_split": (Determinism.kBackendDefault, Variant.kRowSplit, 0)}
    if args.probe:
        # profiling aid: a few launches of one variant, nothing timed
        det, var, lanes = choices[args.probe]
        ctx.set_determinism(det)
        ctx.set_variant(var, lanes)
        for _ in range(3):
            run_plan()
        stream.synchronize()
        plan.close()
        ctx.close()
        return None
    for name, (det, var, lanes) in choices.items():
        ctx.set_determinism(det)
        ctx.set_variant(var, lanes)
        detail[name] = bytes_step / (timed(run_plan, 5, 2) * 1e-3) / 1e9
    best = max(detail, key=detail.get)
    det, var, lanes = choices[best]
    ctx.set_determinism(det)
    ctx.set_variant(var, lanes)
    mode = ("deterministic (bit-exact)" if det == Determinism.kDeterministic
            else f"backend_default ({best}, within gamma bound)")

    # -- headline: device-resident inputs --
    launches0 = ctx.launch_count
    with Clocks(local) as clk:
        ms = timed(run_plan, args.steps, args.warmup)
    launches = (ctx.launch_count - launches0) // (args.steps + args.warmup)
    gbs = bytes_step / (ms * 1e-3) / 1e9

    # -- end to end through the C ABI with host buffers --
    x_pin = torch.from_numpy(x_h).pin_memory()
    y_pin = torch.empty(a_h.rows, dtype=torch.float64).pin_memory()
    ws_bytes = CudaCsrSpmvWorkspaceSize(ctx, A, xv, yv)
    ws = torch.empty(max(ws_bytes, 1), dtype=torch.uint8, device=dev)

    def run_e2e():
        with torch.cuda.stream(stream):
            x.copy_(x_pin, non_blocking=True)
            CudaCsrSpmv(ctx, 1.0, A, xv, 0.0, yv, ws, ws_bytes)
            y_pin.copy_(y, non_blocking=True)

    e2e_serial_ms = timed(run_e2e, max(3, args.steps // 2), 2)

    # Serving loop: two buffer sets, so step i+1's x copies in (its own
    # stream) while step i computes on the context stream and its y copies
    # out (a third stream).  Every step still moves its whole x in and its
    # whole y out through pinned host memory.
    h2d = torch.cuda.Stream(device=dev)
    d2h = torch.cuda.Stream(device=dev)
    xs = [x, torch.empty_like(x)]
    ys = [y, torch.empty_like(y)]
    y_pins = [y_pin, torch.empty(a_h.rows, dtype=torch.float64).pin_memory()]
    views = [(CudaStridedVectorView(xs[i], a_h.cols, writable=False),
              CudaStridedVectorView(ys[i], a_h.rows)) for i in range(2)]
    ev = {k: [torch.cuda.Event() for _ in range(2)] for k in ("in", "done", "out")}

    def pipelined(steps):
        for i in range(steps):
            b = i & 1
            with torch.cuda.stream(h2d):
                if i >= 2:
                    h2d.wait_event(ev["done"][b])  # step i-2's product read x[b]
                xs[b].copy_(x_pin, non_blocking=True)
                ev["in"][b].record(h2d)
            stream.wait_event(ev["in"][b])
            if i >= 2:
                stream.wait_event(ev["out"][b])  # step i-2's y[b] has been copied out
            CudaCsrSpmv(ctx, 1.0, A, views[b][0], 0.0, views[b][1], ws, ws_bytes)
            ev["done"][b].record(stream)
            with torch.cuda.stream(d2h):
                d2h.wait_event(ev["done"][b])
                y_pins[b].copy_(ys[b], non_blocking=True)
                ev["out"][b].record(d2h)

    e2e_steps = max(3, args.steps // 2)
    pipelined(2)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(h2d)
    pipelined(e2e_steps)
    stop.record(d2h)
    stop.synchronize()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(start.elapsed_time(stop) / e2e_steps, world, dev)
    e2e_gbs = bytes_step / (e2e_ms * 1e-3) / 1e9
    # the last step's result, read on the host, equals the device product
    last = (e2e_steps - 1) & 1
    e2e_ok = bool(torch.equal(y_pins[last], ys[last].cpu()))

    # the headline's own result against the FP64 oracle (the checker; it runs
    # after every timed region): the best mode's last product, and a
    # DETERMINISTIC product compared bit for bit
    stream.synchronize()
    error = None
    if rank == 0:
        ctx.set_determinism(Determinism.kDeterministic)
        ctx.set_variant(Variant.kAuto, 0)
        y_det = torch.zeros_like(y)
        plan.csr_spmv(1.0, xv, 0.0, CudaStridedVectorView(y_det, a_h.rows))
        stream.synchronize()
        ctx.set_determinism(det)
        ctx.set_variant(var, lanes)
        plan.csr_spmv(1.0, xv, 0.0, yv)
        stream.synchronize()
        error = headline_error(a_h, x_h, y.cpu().numpy(), y_det.cpu().numpy(), best)
    # comparison only (never the product): cuSPARSE through torch's CSR
    # mat-vec on the same arrays, int64 indices
    comparison = cusparse_leg(a_h, A, x, stream, bytes_step) if rank == 0 else None
    selection = selector_leg() if rank == 0 and world == 1 and not args.no_selector else None
    peak, peak_kind = _peaks()
    traffic = _traffic_record().get(WORKLOAD)
    if isinstance(traffic, dict):  # per variant: the one the headline ran
        traffic = traffic.get(best)
    out = None
    if rank == 0:
        cpu = cpu_baseline_sample(a_h, x_h) if world == 1 else None
        out = {
            "metric": METRIC, "value": round(gbs * world, 3), "unit": "GB/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "rows": a_h.rows, "nnz": a_h.nnz,
                       "alpha": 1.0, "beta": 0.0, "bytes_per_step": bytes_step,
                       "l2": "inputs (1.18 GB) larger than L2; no flush",
                       "mode": mode, "parallelism": "replicas" if world > 1 else "single"},
            "roofline": {"bound": "hbm", "achieved": round(gbs, 2), "peak": peak,
                         "unit": "GB/s", "frac": round(gbs / peak, 4),
                         "traffic": traffic, "peak_kind": peak_kind},
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_gbs * world, 3), "unit": "GB/s",
                    "h2d_bytes_per_step": a_h.cols * 8, "d2h_bytes_per_step": a_h.rows * 8,
                    "ms_per_step": round(e2e_ms, 4),
                    "serial_ms_per_step": round(e2e_serial_ms, 4),
                    "serial_value": round(bytes_step / (e2e_serial_ms * 1e-3) / 1e9 * world, 3),
                    "host_result_matches_device": e2e_ok,
                    "note": ("A cloned to HBM once (CudaCloneCsr); every step copies its x in "
                             "and its y out through pinned host memory. value: serving loop "
                             "with two buffer sets, step i+1's copy-in and step i's copy-out "
                             "overlapping step i's product (3 streams); serial_value: copy in, "
                             "product, copy out one after the other")},
            "gpu_launches": int(launches * args.steps),
            "clocks": clk.summary(),
            "detail_gbs": {k: round(v, 2) for k, v in detail.items()},
            "error_vs_fp64_oracle": error,
            "comparison": comparison,
            "selector_drop_in": selection,
        }
    plan.close()
    ctx.close()
    return out


# ---- further workloads (evidence for the other configurations) -------------

EXTRA = ("spmv_powerlaw_4M_f32", "spmv_t_powerlaw_4M_f64", "spmv_t_powerlaw_4M_f32",
         "spmm_stencil_k8", "spmm_stencil_k32", "spmm_stencil_k128", "spmm_stencil96_k32",
         "spmm_block_k8", "spmm_block_k32", "spmm_block_k128", "batched_banded_4096",
         "sptrsv_laplacian_1M_f64", "sptrsv_stencil27_2M_f64", "sptrsv_powerlaw_4M_f64",
         "sptrsv_random_2M_f64", "sptrsv_random_2M_f32",
         "level1_16M_f64", "clone_powerlaw_4M_f64")


def _timer(stream, steps, warmup):
    import torch

    def timed(fn):
        for _ in range(warmup):
            fn()
        stream.synchronize()
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        for _ in range(steps):
            fn()
        stop.record(stream)
        stop.synchronize()
        return start.elapsed_time(stop) / steps
    return timed


def run_extra(args):
    """One JSON line for a workload other than the headline: the same keys,
    both numerical modes timed, the faster one as `value`."""
    import torch
    from asc_cpp_b200 import synthetic
    from asc_cpp_b200._abi import PLAN_TRANSPOSE, Determinism, SparseBlasTranspose
    from asc_cpp_b200 import sparse_cuda as sc

    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    timed = _timer(stream, args.steps, args.warmup)
    ctx = sc.SparseCudaContext.Create(0, stream=stream)
    peak, peak_kind = _peaks()
    w = args.workload
    detail, extra_cfg = {}, {}
    if w.startswith("spmv"):
        transpose = "_t_" in w
        dt = np.float32 if w.endswith("f32") else np.float64
        a_h = synthetic.power_law(4_194_304, 16.0, 1.5, 65_536, seed=1, dtype=dt)
        es = np.dtype(dt).itemsize
        with torch.cuda.stream(stream):
            A = sc.CudaCsrArray(a_h.rows, a_h.cols, torch.from_numpy(a_h.ptr).to(dev),
                                torch.from_numpy(a_h.idx).to(dev), torch.from_numpy(a_h.val).to(dev))
            x = (torch.rand(a_h.rows if transpose else a_h.cols, device=dev,
                            dtype=torch.float64) * 2 - 1).to(A.values.dtype)
            y = torch.zeros(a_h.cols if transpose else a_h.rows, device=dev, dtype=A.values.dtype)
        stream.synchronize()
        xv, yv = sc.CudaStridedVectorView(x, x.numel(), writable=False), sc.CudaStridedVectorView(y, y.numel())
        t0 = time.time()
        plan = sc.CsrPlan(ctx, A, PLAN_TRANSPOSE if transpose else 0)
        stream.synchronize()
        extra_cfg["plan_create_s"] = round(time.time() - t0, 3)
        op = SparseBlasTranspose.kTranspose if transpose else SparseBlasTranspose.kNone
        byts = a_h.nnz * (es + 8) + (a_h.rows + 1) * 8 + (a_h.rows + a_h.cols) * es
        if transpose:
            byts = a_h.nnz * (es + 8) + (a_h.cols + 1) * 8 + (a_h.rows + a_h.cols) * es
        for name, det, use_plan in (("deterministic_plan", Determinism.kDeterministic, True),
                                    ("default_plan", Determinism.kBackendDefault, True),
                                    ("default_scatter", Determinism.kBackendDefault, False)):
            if not transpose and name == "default_scatter":
                continue
            ctx.set_determinism(det)
            ms = timed(lambda: sc.CudaSpmv(ctx, op, 1.0, A, xv, yv, plan=plan if use_plan else None))
            detail[name] = {"ms": round(ms, 4), "gbs": round(byts / ms / 1e6, 1)}
        # one product of each mode through the plan against the oracle (the
        # checker; after every timed region): y = 0 + A x or A^T x
        got = {}
        for name, det in (("deterministic", Determinism.kDeterministic),
                          ("default", Determinism.kBackendDefault)):
            ctx.set_determinism(det)
            with torch.cuda.stream(stream):  # ordered before the product
                y.zero_()
            sc.CudaSpmv(ctx, op, 1.0, A, xv, yv, plan=plan)
            stream.synchronize()
            got[name] = y.cpu().numpy()
        extra_cfg["error_vs_fp64_oracle"] = spmv_error(a_h, x.cpu().numpy(), got, transpose)
        plan.close()
        dtype_s = "f32" if dt == np.float32 else "f64"
        extra_cfg.update({"rows": a_h.rows, "nnz": a_h.nnz, "op": "transpose" if transpose else "none"})
    elif w.startswith("spmm"):
        k = int(w.rsplit("_k", 1)[1])
        # the 27-point stencil on 128^3 (config 3a) or 96^3 (a small case of the
        # same kernels for profiling), or the 16 x 16 block matrix (config 3b)
        if "stencil" in w:
            a_h = synthetic.stencil_27(96 if "stencil96" in w else 128)
        else:
            a_h = synthetic.block_sparse()
        with torch.cuda.stream(stream):
            A = sc.CudaCsrArray(a_h.rows, a_h.cols, torch.from_numpy(a_h.ptr).to(dev),
                                torch.from_numpy(a_h.idx).to(dev), torch.from_numpy(a_h.val).to(dev))
            g = torch.Generator(device=dev)
            g.manual_seed(2)
            B = torch.randn(a_h.cols, k, generator=g, device=dev, dtype=torch.float32)
            C = torch.zeros(a_h.rows, k, device=dev, dtype=torch.float32)
        stream.synchronize()
        byts = a_h.nnz * 12 + (a_h.rows + 1) * 8 + 2 * a_h.rows * k * 4
        flops = 2 * a_h.nnz * k
        bv = sc.DenseMatrixView(B, a_h.cols, k, writable=False)
        cv = sc.DenseMatrixView(C, a_h.rows, k)
        from asc_cpp_b200._abi import PLAN_HAS_ROW_GROUPS, PLAN_HAS_STAGED_SPMM, PLAN_ROW_GROUPS
        # a plan detects dense 16 x 16 blocks (tensor-core path) and builds the
        # TMA-staged tables and row groups (B rows shared by neighbouring rows)
        t0 = time.time()
        plan = sc.CsrPlan(ctx, A, PLAN_ROW_GROUPS)
        stream.synchronize()
        extra_cfg["plan_create_s"] = round(time.time() - t0, 3)
        extra_cfg["dense_blocks16"] = bool(plan.properties() & 2)
        extra_cfg["row_groups_kept"] = bool(plan.properties() & PLAN_HAS_ROW_GROUPS)
        extra_cfg["staged_kept"] = bool(plan.properties() & PLAN_HAS_STAGED_SPMM)
        plain = sc.CsrPlan(ctx, A)
        # the staged kernel at this k (where its stages fit), whatever the
        # plan's default rule would pick
        plan_tag = "_staged"
        if extra_cfg["staged_kept"]:
            from asc_cpp_b200._abi import SPMM_STAGED
            plan.set_spmm(SPMM_STAGED)
        else:
            plan_tag = "_plan_default"
        for name, det in (("deterministic", Determinism.kDeterministic),
                          ("default", Determinism.kBackendDefault)):
            ctx.set_determinism(det)
            for tag, p_ in (("", plain), (plan_tag, plan)):
                ms = timed(lambda: sc.CudaSpmm(ctx, SparseBlasTranspose.kNone, 1.0, A, bv, cv,
                                               plan=p_))
                detail[name + tag] = {"ms": round(ms, 4), "gbs": round(byts / ms / 1e6, 1),
                                      "gflops": round(flops / ms / 1e6, 1)}
        # the faster default-mode path (plain or the plan's) against the FP64
        # oracle on a row sample (the checker; after the timed regions, before
        # the autotuner changes the plan)
        best_default = min(("default", "default" + plan_tag), key=lambda kk: detail[kk]["ms"])
        use = plain if best_default == "default" else plan
        with torch.cuda.stream(stream):  # ordered before the product
            C.zero_()
        sc.CudaSpmm(ctx, SparseBlasTranspose.kNone, 1.0, A, bv, cv, plan=use)
        stream.synchronize()
        extra_cfg["error_vs_fp64_oracle"] = spmm_error(a_h, B.cpu().numpy(), C.cpu().numpy(),
                                                       best_default, 65_536,
                                                       extra_cfg["dense_blocks16"])
        # the SpMM autotuner on this k (row by row, staged, or R rows per
        # group), per mode
        for name, det in (("deterministic", Determinism.kDeterministic),
                          ("default", Determinism.kBackendDefault)):
            ctx.set_determinism(det)
            with torch.cuda.stream(stream):
                scratch = torch.zeros_like(C)
            t_ms, rg = plan.spmm_autotune(1.0, bv, sc.DenseMatrixView(scratch, a_h.rows, k), 5)
            ms = timed(lambda: sc.CudaSpmm(ctx, SparseBlasTranspose.kNone, 1.0, A, bv, cv,
                                           plan=plan))
            detail[name + "_autotuned"] = {"ms": round(ms, 4), "gbs": round(byts / ms / 1e6, 1),
                                           "gflops": round(flops / ms / 1e6, 1),
                                           "rows_per_group": rg,
                                           "tuning_ms": {str(kk): round(vv, 4) for kk, vv in
                                                         plan.spmm_tuning().items()}}
            del scratch
        plan.close()
        plain.close()
        dtype_s = "f32"
        extra_cfg.update({"rows": a_h.rows, "nnz": a_h.nnz, "k": k, "layout": "row-major, ld=k"})
    elif w.startswith("sptrsv"):
        from asc_cpp_b200._abi import PLAN_TRIANGULAR, SparseBlasDiagonal, SparseBlasTriangle
        dt = np.float32 if w.endswith("f32") else np.float64
        es = np.dtype(dt).itemsize
        unit_diagonal = False
        if "laplacian" in w:
            a_h = synthetic.triangle_of(synthetic.laplacian_2d(1000, dtype=dt))
            extra_cfg["wavefronts"] = 2 * 1000 - 1
        elif "stencil27" in w or "powerlaw" in w:
            full = (synthetic.stencil_27(128, dtype=dt) if "stencil27" in w else
                    synthetic.power_law(4_194_304, 16.0, 1.5, 65_536, seed=1, dtype=dt))
            a_h = synthetic.triangle_of(full)
            rows_of = np.repeat(np.arange(a_h.rows), np.diff(a_h.ptr))
            on = a_h.idx == rows_of
            mag = np.bincount(rows_of[~on], weights=np.abs(a_h.val[~on]), minlength=a_h.rows)
            if "stencil27" in w:
                # diagonally dominant: |diagonal| = 1 + sum of the other |entries|
                a_h.val[on] = (1.0 + mag[rows_of[on]]).astype(dt)
                extra_cfg["wavefronts"] = 3 * 127 + 1
            else:
                # the power-law matrix stores almost no diagonal: unit diagonal,
                # entries scaled to row sums below 1/2
                unit_diagonal = True
                a_h.val[:] = (a_h.val / (2.0 * (mag[rows_of] + 1.0))).astype(dt)
        else:
            a_h = synthetic.triangular(np.random.default_rng(11), 2_000_000, lower=True, near=4,
                                       far=2, span=64, dtype=dt)
        n = a_h.rows
        diag = SparseBlasDiagonal.kUnit if unit_diagonal else SparseBlasDiagonal.kNonUnit
        extra_cfg["diagonal"] = "unit" if unit_diagonal else "non-unit"
        with torch.cuda.stream(stream):
            A = sc.CudaCsrArray(n, n, torch.from_numpy(a_h.ptr).to(dev),
                                torch.from_numpy(a_h.idx).to(dev), torch.from_numpy(a_h.val).to(dev))
            b0 = (torch.rand(n, device=dev, dtype=torch.float64) * 2 - 1).to(A.values.dtype)
            xb = b0.clone()
        stream.synchronize()
        plan = sc.CsrPlan(ctx, A, PLAN_TRIANGULAR)
        rhs = sc.DenseMatrixView(xb, n, 1)
        # the solve overwrites its right-hand side: each step restores it
        # (a device copy of n elements, inside the timed region)
        byts = a_h.nnz * (es + 8) + (n + 1) * 8 + 2 * n * es

        def restore():
            with torch.cuda.stream(stream):  # the library's stream, ahead of the solve
                xb.copy_(b0)

        def solve(use_plan):
            restore()
            sc.CudaSparseTriangularSolveMultiple(ctx, SparseBlasTranspose.kNone, 1.0, A,
                                                 SparseBlasTriangle.kLower, diag, rhs,
                                                 plan=plan if use_plan else None)
        copy_ms = timed(restore)
        for name, det, use_plan in (("deterministic", Determinism.kDeterministic, False),
                                    ("default", Determinism.kBackendDefault, False)):
            ctx.set_determinism(det)
            ms = timed(lambda: solve(use_plan)) - copy_ms
            detail[name] = {"ms": round(ms, 4), "gbs": round(byts / ms / 1e6, 1)}
        solved = {}
        t0 = time.perf_counter()
        plan.triangular_analysis(SparseBlasTranspose.kNone, SparseBlasTriangle.kLower)
        stream.synchronize()
        extra_cfg["analysis_ms"] = round((time.perf_counter() - t0) * 1e3, 3)
        for name, det in (("deterministic_levels", Determinism.kDeterministic),
                          ("default_levels", Determinism.kBackendDefault)):
            ctx.set_determinism(det)
            ms = timed(lambda: solve(True)) - copy_ms
            detail[name] = {"ms": round(ms, 4), "gbs": round(byts / ms / 1e6, 1)}
            stream.synchronize()
            solved[name] = xb.cpu().numpy()  # x = A^-1 b0, the same every timed call
        plan.close()
        try:  # the library baseline: cuSPARSE SpSV through torch (not on the product path)
            At = torch.sparse_csr_tensor(A.offsets, A.indices, A.values, (n, n))
            with torch.cuda.stream(stream):
                ms = timed(lambda: torch.triangular_solve(b0.view(n, 1), At, upper=False,
                                                          unitriangular=unit_diagonal))
            detail["cusparse_spsv_via_torch"] = {"ms": round(ms, 4),
                                                 "gbs": round(byts / ms / 1e6, 1)}
        except Exception as e:  # noqa: BLE001
            detail["cusparse_spsv_via_torch"] = {"unavailable": str(e).splitlines()[0][:120]}
        from oracle import Restatement  # the CPU leg only (the oracle as the baseline)
        r = Restatement()
        bh = b0.cpu().numpy()
        t0 = time.perf_counter()
        want = r.triangular_solve(0, 1, int(diag), n, a_h.ptr, a_h.idx, a_h.val, 1.0, bh)
        detail["cpu_oracle_1_thread"] = {"ms": round((time.perf_counter() - t0) * 1e3, 2)}
        # the level-scheduled solves against the oracle's row-by-row solve:
        # DETERMINISTIC bit for bit; BACKEND_DEFAULT by its largest relative
        # difference (a solve's error grows along dependency chains, so no
        # per-row bound is claimed)
        dd = solved["default_levels"].astype(np.float64) - want
        extra_cfg["error_vs_fp64_oracle"] = {
            "deterministic_bitexact": bool(solved["deterministic_levels"].tobytes() == want.tobytes()),
            "default_max_abs": float(np.abs(dd).max()),
            "default_max_rel": float((np.abs(dd) / np.maximum(np.abs(want), 1e-300)).max()),
            "outputs": int(n),
            "oracle": "C restatement of the row-by-row triangular solve, same precision"}
        dtype_s = "f32" if dt == np.float32 else "f64"
        extra_cfg.update({"rows": n, "nnz": a_h.nnz, "op": "none", "triangle": "lower",
                          "rhs_restore_ms_subtracted": round(copy_ms, 4)})
    elif w.startswith("clone"):
        # host -> device clone of the 4M-row power-law matrix (1.18 GB of CSR)
        a_h = synthetic.power_law(4_194_304, 16.0, 1.5, 65_536, seed=1)
        byts = a_h.ptr.nbytes + a_h.idx.nbytes + a_h.val.nbytes
        ptr_p, idx_p, val_p = (torch.from_numpy(a).pin_memory() for a in (a_h.ptr, a_h.idx, a_h.val))
        keep = []

        def clone(pinned):
            src = (ptr_p, idx_p, val_p) if pinned else (a_h.ptr, a_h.idx, a_h.val)
            keep.append(sc.CudaCloneCsr(ctx, a_h.rows, a_h.cols, *src))
            if len(keep) > 2:
                keep.pop(0)

        def torch_pageable():
            keep.append(tuple(torch.from_numpy(a).to(dev) for a in (a_h.ptr, a_h.idx, a_h.val)))
            if len(keep) > 2:
                keep.pop(0)
        for name, fn in (("clone_pageable", lambda: clone(False)),
                         ("clone_pinned", lambda: clone(True)),
                         ("torch_pageable_to_device", torch_pageable)):
            for _ in range(args.warmup):
                fn()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                fn()
            torch.cuda.synchronize()
            ms = (time.perf_counter() - t0) * 1e3 / args.steps
            detail[name] = {"ms": round(ms, 3), "gbs": round(byts / ms / 1e6, 2)}
        dtype_s = "f64"
        extra_cfg.update({"rows": a_h.rows, "nnz": a_h.nnz, "bytes": byts,
                          "timing": "host wall clock around each clone, synchronized"})
        out = {"metric": "host-to-device clone GB/s", "value": detail["clone_pageable"]["gbs"],
               "unit": "GB/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": detail["clone_pageable"]["ms"], "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": dtype_s, "data": "synthetic",
               "config": {"workload": w, **extra_cfg}, "detail": detail}
        ctx.close()
        print(json.dumps(out), flush=True)
        return 0
    elif w.startswith("level1"):
        from asc_cpp_b200._abi import Level1Op
        n, nnz = 64 * 1024 * 1024, 16 * 1024 * 1024
        g = torch.Generator(device=dev)
        g.manual_seed(3)
        with torch.cuda.stream(stream):
            idx = torch.sort(torch.randperm(n, device=dev, generator=g)[:nnz]).values
            val = torch.rand(nnz, device=dev, dtype=torch.float64, generator=g)
            x = torch.rand(n, device=dev, dtype=torch.float64, generator=g)
            res = torch.zeros(1, device=dev, dtype=torch.float64)
        stream.synchronize()
        # bytes: index + value per entry, plus the 32-byte sectors of x touched
        sectors = int(torch.unique(idx // 4).numel()) * 32
        op_bytes = {"dot": nnz * 16 + sectors, "axpy": nnz * 16 + 2 * sectors,
                    "gather": nnz * 24 + sectors, "scatter": nnz * 16 + sectors}
        dv = sc.CudaStridedVectorView(x, n)
        for name, op, det in (("dot_deterministic", Level1Op.kDot, Determinism.kDeterministic),
                              ("dot_default", Level1Op.kDot, Determinism.kBackendDefault),
                              ("axpy", Level1Op.kAxpy, Determinism.kDeterministic),
                              ("gather", Level1Op.kGather, Determinism.kDeterministic),
                              ("scatter", Level1Op.kScatter, Determinism.kDeterministic)):
            ctx.set_determinism(det)
            ms = timed(lambda: sc.CudaLevel1(ctx, op, idx, val, dv, res, 1e-9))
            b = op_bytes[name.split("_")[0]]
            detail[name] = {"ms": round(ms, 4), "gbs": round(b / ms / 1e6, 1)}
        byts = op_bytes["axpy"]
        detail = {"axpy": detail.pop("axpy"), **detail}
        dtype_s = "f64"
        extra_cfg.update({"dense": n, "nnz": nnz, "x_sectors_bytes": sectors})
    else:  # batched
        g = synthetic.banded_batch_device(4096)
        mats, xs, ys = [], [], []
        for m in range(4096):
            n, z = int(g["rows"][m]), int(g["nnz"][m])
            pb, nb, rb = int(g["ptr_base"][m]), int(g["nz_base"][m]), int(g["row_base"][m])
            mats.append(sc.CudaCsrArray(n, n, g["ptr"][pb:pb + n + 1], g["idx"][nb:nb + z],
                                        g["val"][nb:nb + z]))
            xs.append(sc.CudaStridedVectorView(g["x"][rb:rb + n], n, writable=False))
            ys.append(sc.CudaStridedVectorView(g["y"][rb:rb + n], n))
        batch = sc.CudaBatch(ctx, mats, xs, ys)
        got = {}
        byts = int((g["nnz"] * 16 + (g["rows"] + 1) * 8 + 2 * g["rows"] * 8).sum())
        for name, det in (("deterministic", Determinism.kDeterministic),
                          ("default", Determinism.kBackendDefault)):
            ctx.set_determinism(det)
            batch.set_schedule(4, 0)
            per = _timer(stream, max(3, args.steps // 10), args.warmup)(
                lambda: batch.spmv_per_matrix(1.0, 0.0))
            batch.autotune(1.0, 0.0, 3)
            batch.capture(1.0, 0.0)
            ms = timed(lambda: batch.spmv(1.0, 0.0))
            detail[name] = {"ms": round(ms, 4), "gbs": round(byts / ms / 1e6, 1),
                            "per_matrix_ms": round(per, 3), "speedup_vs_per_matrix": round(per / ms, 2),
                            "schedule": batch.schedule()}
            stream.synchronize()
            got[name] = g["y"].cpu().numpy()  # y = A x, the same every timed call
        batch.close()
        extra_cfg["error_vs_fp64_oracle"] = batch_error(g, got, 128)
        dtype_s = "f64"
        extra_cfg.update({"matrices": 4096, "rows": int(g["rows"].sum()), "nnz": int(g["nnz"].sum())})
    if w.startswith("level1"):
        best = "axpy"
    else:
        best = min((k for k in detail if "ms" in detail[k] and not k.startswith(("cusparse", "cpu"))),
                   key=lambda k: detail[k]["ms"])
    ms = detail[best]["ms"]
    gbs = byts / ms / 1e6
    out = {"metric": METRIC, "value": round(gbs, 3), "unit": "GB/s", "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype_s,
           "data": "synthetic", "config": {"workload": w, "bytes_per_step": int(byts),
                                           "best_mode": best, **extra_cfg},
           "roofline": {"bound": "hbm", "achieved": round(gbs, 2), "peak": peak, "unit": "GB/s",
                        "frac": round(gbs / peak, 4), "traffic": None, "peak_kind": peak_kind},
           "detail": detail}
    ctx.close()
    print(json.dumps(out), flush=True)
    return 0


def run_gather_floor(args):
    """The floor under any CSR SpMV of the 4M-row power-law matrix: flat
    (row-less) sums over its own column indices and values with one random
    gather of x per nonzero, the gathers alone and the streamed arrays alone,
    for each load pattern, gather flavour and CTAs per SM
    (csrc/probe/gather_floor.cu).  One JSON line; `value` is the best flat
    sum expressed in the SpMV byte model."""
    import ctypes
    import torch
    from asc_cpp_b200 import build as lib_build

    lib = ctypes.CDLL(lib_build.build_probe())
    lib.ascb_probe_flat.restype = ctypes.c_int
    lib.ascb_probe_flat.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                    ctypes.c_int64, ctypes.c_void_p, ctypes.c_int]
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)
    a_h, x_h = _matrix()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    with torch.cuda.stream(stream):
        idx = torch.from_numpy(a_h.idx).to(dev)
        val = torch.from_numpy(a_h.val).to(dev)
        x = torch.from_numpy(x_h).to(dev)
        out = torch.zeros(sms * 16 * lib.ascb_probe_threads(), dtype=torch.float64, device=dev)
    stream.synchronize()
    nnz = a_h.nnz // 256 * 256
    bytes_step = a_h.bytes_spmv(8)
    timed = _timer(stream, max(5, min(args.steps, 50)), args.warmup)
    names = {0: "flat_16B_lane_runs", 1: "flat_32B_lane_runs", 2: "flat_16B_coalesced",
             3: "gathers_only", 4: "streams_only"}
    flavours = {0: "nc", 1: "nc_L1_no_allocate", 2: "cg"}
    table = {}
    for mode, name in names.items():
        for g, gname in flavours.items():
            if mode == 4 and g > 0:
                continue
            for per_sm in (4, 6, 8, 12, 16):
                def run():
                    rc = lib.ascb_probe_flat(stream.cuda_stream, mode, g, idx.data_ptr(),
                                             val.data_ptr(), x.data_ptr(), nnz, a_h.cols,
                                             out.data_ptr(), sms * per_sm)
                    if rc != 0:
                        raise RuntimeError(f"probe launch failed: {rc}")
                ms = timed(run)
                table[f"{name}/{gname}/{per_sm}"] = round(ms, 4)
    best = {name: min((v, k) for k, v in table.items() if k.startswith(name + "/"))
            for name in names.values()}
    flat = min(best[n] for n in ("flat_16B_lane_runs", "flat_32B_lane_runs", "flat_16B_coalesced"))
    ms = flat[0]
    gbs = bytes_step / (ms * 1e-3) / 1e9
    peak, peak_kind = _peaks()
    line = {"metric": "CSR SpMV gather floor (flat sum, SpMV byte model)", "value": round(gbs, 2),
            "unit": "GB/s", "n_gpus": 1, "steps": max(5, min(args.steps, 50)),
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "gather_floor", "rows": a_h.rows, "nnz": a_h.nnz,
                       "positions_timed": nnz, "bytes_per_step": bytes_step,
                       "best": flat[1]},
            "roofline": {"bound": "hbm", "achieved": round(gbs, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(gbs / peak, 4), "traffic": None, "peak_kind": peak_kind},
            "gathers_per_s_G": round(nnz / (best["gathers_only"][0] * 1e-3) / 1e9, 2),
            "best_ms": {k: v for k, v in best.items()}, "table_ms": table}
    print(json.dumps(line), flush=True)
    return 0


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--no-selector", action="store_true",
                   help="skip the selector leg of the headline run")
    p.add_argument("--probe", default=None,
                   help="profiling aid: run 3 launches of one variant and exit")
    p.add_argument("--workload", default=WORKLOAD,
                   choices=(WORKLOAD,) + EXTRA + ("gather_floor",),
                   help="another configuration's workload (one GPU, this library only)")
    args = p.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = _env_int("RANK", 0)
    world = _env_int("WORLD_SIZE", 1)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "gather_floor":
        return run_gather_floor(args)
    if args.workload != WORKLOAD:
        return run_extra(args)
    import torch.distributed as dist
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        out = run_gpu(args, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
    finally:
        if world > 1:
            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
