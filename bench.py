#!/usr/bin/env python
"""H-matvec throughput on one B200 (or N replicas under torchrun).

Workload (the batching configuration): N = 2^20 points i.i.d. uniform in [0,1]^3
(SplitMix64 seed 1), Matern-3/2 kernel (1 + sqrt3 r/0.2) exp(-sqrt3 r/0.2), leaf
size 128, eta 1.5 (min-diameter admissibility), adaptive ACA eps = 1e-8 with ranks
up to 96, FP32 near-field blocks and mixed-precision low-rank factors (leading terms
FP32, tail terms FP16 / FP8 e4m3 by their share of the block norm), FP32 products
summed in FP64; --prec fp32 / fp64 store every factor in that type.  One step = one
H-matvec y = H x with x ~ U[-1,1] (seed 1001); the error against an FP64 direct sum
over 4,096 rows is reported beside every number (err_vs_fp64).

  value  H-matvecs/s with x and y resident in HBM (device-timed with CUDA events);
  e2e    the same through the host-buffer C-ABI call hmg_matvec_host: x copied
         in from the caller's pageable host memory and y copied out to it, every
         step, inside the timing.
  multi_rhs  products of 32 vectors a pass on the same H-matrix (hmg_matvec_multi,
         CUDA cores), vectors per second.
  batched_tensor_cores  64 vectors a pass on the tensor cores with three-part BF16
         operands at N=2^18 (error <= 1e-6), beside the plain FP64 form at that size
         (the FP64 form of N=2^20 does not fit one B200).
  serve  a short run of the serving workload (60 requests of the Poisson stream over
         8 resident H-matrices, bench.py --workload serve for the full one): p50/p99
         latency of the completed requests.
The stored H-matrix (~95 GB mixed) is far larger than L2, so no L2 flush is needed
between steps.  --impl reference times the FP64 direct product (the reference's
apply_full_mvp, restated by the CPU oracle) on the host cores on a row sample.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = {"workload": "hmatvec_uniform3d_matern32", "n": 1 << 20, "dim": 3, "seed": 1,
            "kernel": "matern32", "rho": 0.2, "leaf": 128, "eta": 1.5, "admissibility": "min",
            "aca_eps": 1e-8, "max_rank": 96}
METRIC = "H-matvecs/s at N=2^20 (err<=1e-6 vs FP64)"
K2_TRAFFIC_RATIO = 1.028  # (dram read + write) / algorithmic bytes of k_tile_matvec, mixed storage


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self, min_samples=1):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_direct_rate(p, x, kind, param, target_s=10.0, threads=None):
    """FP64 direct-sum rows/s on the host cores (the oracle's apply_full_mvp)."""
    from oracle import oracle as O
    threads = threads or os.cpu_count() or 1
    s, o, z = O.order_points(p, 20 if p.shape[0] == 3 else 32)
    xs = np.ascontiguousarray(x[o])
    n = p.shape[1]
    rng = np.random.default_rng(0)
    rows = np.ascontiguousarray(rng.choice(n, size=min(n, 8 * threads), replace=False).astype(np.int32))
    t0 = time.perf_counter()
    O.direct(kind, param, 0.0, z, z, xs, rows=rows, nthreads=threads)
    dt = time.perf_counter() - t0
    nrows = int(min(n, max(len(rows), len(rows) * target_s / max(dt, 1e-6))))
    rows = np.ascontiguousarray(rng.choice(n, size=nrows, replace=False).astype(np.int32))
    t0 = time.perf_counter()
    O.direct(kind, param, 0.0, z, z, xs, rows=rows, nthreads=threads)
    dt = time.perf_counter() - t0
    return nrows / dt, nrows, dt, threads


def run_reference(a, rank, world):
    """The reference arm: FP64 direct product on host cores, bounded row sample per step."""
    from hmglib_b200 import synth
    from oracle import oracle as O
    if rank != 0:
        return 0
    W = WORKLOAD
    n = a.n or W["n"]
    p = synth.uniform_points(n, W["dim"], W["seed"])
    x = synth.rhs_vector(n, W["seed"])
    kind = O.KERNEL_MATERN32
    par = O.kernel_param(kind, W["rho"])
    per_step = max(2.0, 20.0 / max(1, a.steps + a.warmup))
    for _ in range(a.warmup):
        cpu_direct_rate(p, x, kind, par, target_s=per_step / 4)
    rates = []
    for _ in range(a.steps):
        r, nrows, dt, thr = cpu_direct_rate(p, x, kind, par, target_s=per_step)
        rates.append(r)
    rows_per_s = float(np.median(rates))
    value = rows_per_s / n
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "matvec/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1000.0 / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(W, n=n, parallelism="host cores"),
            "cpu_baseline": {"value": value, "unit": "matvec/s", "cores": thr, "kind": "port",
                             "sample": f"{nrows} random rows of the FP64 direct sum per step, scaled to N={n} rows"},
            "e2e": {"value": value, "unit": "matvec/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(values, world, device=None):
    """Element-wise maximum of per-rank timings (the slowest rank sets the step time).
    With one rank the values pass through; otherwise one all-reduce on `device`."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def multi_rhs_timing(torch, H, x, n, nrhs, steps, stream, world, err1):
    """Products of nrhs vectors at once (hmg_matvec_multi): vector products per second,
    device-resident and end to end (pinned host X in, Y out, inside the timing)."""
    rng = np.random.default_rng(11)
    Xh = rng.uniform(-1, 1, (nrhs, n))
    Xh[0] = x
    X = torch.from_numpy(Xh).cuda()
    Y = torch.empty_like(X)
    for _ in range(3):
        H.matvec_multi(X, Y)
    torch.cuda.synchronize()
    # column 0 equals the single-vector product to FP32 rounding
    y1 = torch.empty(n, dtype=torch.float64, device="cuda")
    H.matvec(X[0], y1)
    torch.cuda.synchronize()
    diff = float(torch.linalg.norm(Y[0] - y1) / torch.linalg.norm(y1))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        H.matvec_multi(X, Y)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    Xp = torch.from_numpy(Xh).pin_memory()
    Yp = torch.empty(Xh.shape, dtype=torch.float64).pin_memory()
    e0.record(stream)
    for _ in range(steps):
        X.copy_(Xp, non_blocking=True)
        H.matvec_multi(X, Y)
        Yp.copy_(Y, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1)
    ms, ms_e2e = max_over_ranks([ms, ms_e2e], world, "cuda")
    return {"nrhs": nrhs, "ms_per_product": ms / steps, "value": world * nrhs * 1000.0 * steps / ms,
            "unit": "vector products/s", "e2e_value": world * nrhs * 1000.0 * steps / ms_e2e,
            "err_vs_fp64_col0": err1 + diff, "col0_vs_single": diff}


def onchip_tensor_cores(torch, hmg, H, x, n, steps, stream, world, peak, nrhs=64):
    """64 vectors a pass on the tensor cores over the handle's own (mixed) storage: the
    pass kernels convert factors and near field into three BF16 parts on chip
    (HMG_PREC_BF16X6_ONCHIP).  Error against FP64 direct sums on 2,048 rows of four of
    the vectors; e2e includes copying X in and Y out through pinned host memory."""
    from hmglib_b200 import synth
    t0 = time.perf_counter()
    H.build_bf16_factors(near=hmg.PREC_BF16X6_ONCHIP)
    t_plan = time.perf_counter() - t0
    X = torch.from_numpy(synth.rhs_vector(n, 11, nrhs)).cuda()
    Y = torch.empty_like(X)
    for _ in range(2):
        H.matvec_multi(X, Y)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        e0.record(stream)
        for _ in range(steps):
            H.matvec_multi(X, Y)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks([e0.elapsed_time(e1) / steps], world, "cuda")[0]
    # end to end: X from pinned host memory in, Y out, every step
    Xh = torch.from_numpy(synth.rhs_vector(n, 11, nrhs)).pin_memory()
    Yh = torch.empty(Y.shape, dtype=torch.float64, pin_memory=True)
    e0.record(stream)
    for _ in range(steps):
        X.copy_(Xh, non_blocking=True)
        H.matvec_multi(X, Y)
        Yh.copy_(Y, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1) / steps
    rng = np.random.default_rng(3)
    rows = torch.from_numpy(rng.choice(n, 2048, replace=False).astype(np.int32)).cuda()
    errs = []
    for j in (0, 21, 42, nrhs - 1):
        yd = torch.empty(rows.shape[0], dtype=torch.float64, device="cuda")
        H.full_matvec_rows(X[j], rows, yd)
        torch.cuda.synchronize()
        errs.append(float(torch.linalg.norm(Y[j][rows.long()] - yd) / torch.linalg.norm(yd)))
    info = H.info()
    stored = info["near_bytes"] + info["far_bytes"]
    # the plain FP64 form (FP64 factors and near field, one vector a product) of this
    # H-matrix: its bytes per product and the products/s the measured copy peak allows
    fp64_bytes = 8 * (info["near_entries"] + info["far_entries"]) + 16 * n
    fp64_max = peak * 1e9 / fp64_bytes
    value = nrhs * world * 1000.0 / ms
    return {"n": n, "nrhs": nrhs, "operands": "3 BF16 parts converted on chip from the mixed storage",
            "ms_per_product": ms, "value": value, "unit": "vector products/s",
            "e2e_value": nrhs * world * 1000.0 / ms_e2e, "err_vs_fp64_max": max(errs),
            "err_vs_fp64_cols": errs, "stored_bytes": stored,
            "stored_GBps": stored / (ms * 1e-3) / 1e9, "stored_frac_of_peak": stored / (ms * 1e-3) / 1e9 / peak,
            "plan_s": t_plan, "clocks": clk.summary(),
            "fp64_form_bound": {"bytes_per_product": fp64_bytes, "fits_one_gpu": fp64_bytes < 170e9,
                                "max_value": fp64_max, "unit": "matvec/s",
                                "basis": "FP64 factors and near field read once per product at the measured copy peak"},
            "speedup_vs_fp64_form_bound": value / fp64_max}


def batched_tensor_cores(steps):
    """Batched products on the tensor cores at error <= 1e-6 beside the plain FP64 form,
    at N = 2^18 points of this workload: the largest power of two at which the FP32
    storage and its three-part BF16 operand copy fit one B200 together.  FP32 factors
    and near field, converted to three-part BF16 operands (HMG_PREC_BF16X6), 64 vectors
    a pass (x ~ U[-1,1], seed 11); the plain FP64 form (FP64 factors, near field and
    products, the reference's arithmetic) one vector at a time on the same H-matrix
    structure.  Errors: the largest over 4 vectors of the relative error against FP64
    direct sums over 4,096 rows.  Device-timed with CUDA events; e2e copies X in from
    pinned host memory and Y out, every step."""
    import torch

    import hmglib_b200 as hmg
    from hmglib_b200 import synth
    W = WORKLOAD
    n, nrhs = 1 << 18, 64
    p = synth.uniform_points(n, W["dim"], W["seed"])
    Xh = np.random.default_rng(11).uniform(-1, 1, (nrhs, n))
    X = torch.from_numpy(Xh).cuda()
    rows = torch.from_numpy(np.random.default_rng(7).choice(n, 4096, replace=False).astype(np.int32)).cuda()
    stream = torch.cuda.default_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def build(prec):
        H = hmg.HMatrix(n, n, W["dim"])
        H.set_points(0, p)
        H.set_points(1, p)
        H.setup(W["eta"], W["leaf"], rule=hmg.ADMISSIBLE_MIN)
        H.set_kernel(hmg.KERNEL_MATERN32, W["rho"], 0.0)
        H.precompute_aca(W["max_rank"], W["aca_eps"], prec)
        H.precompute_dense(prec)
        return H

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def max_error(H, Y, cols):
        yd = torch.empty(rows.shape[0], dtype=torch.float64, device="cuda")
        worst = 0.0
        for j in cols:
            H.full_matvec_rows(X[j], rows, yd)
            torch.cuda.synchronize()
            worst = max(worst, float(torch.linalg.norm(Y[j][rows.long()] - yd) / torch.linalg.norm(yd)))
        return worst

    out = {"n": n, "nrhs": nrhs, "operands": "BF16 x3 parts (HMG_PREC_BF16X6)"}
    H = build(hmg.PREC_FP32)
    H.build_bf16_factors(near=hmg.PREC_BF16X6)
    info = H.info()
    Y = torch.empty_like(X)
    with ClockSampler(torch.cuda.current_device()) as clk:
        ms = timed(lambda: H.matvec_multi(X, Y))
        Xp = torch.from_numpy(Xh).pin_memory()
        Yp = torch.empty(Xh.shape, dtype=torch.float64).pin_memory()

        def e2e_step():
            X.copy_(Xp, non_blocking=True)
            H.matvec_multi(X, Y)
            Yp.copy_(Y, non_blocking=True)
        ms_e2e = timed(e2e_step)
    out.update({"ms_per_product": ms, "value": nrhs * 1000.0 / ms, "unit": "vector products/s",
                "e2e_value": nrhs * 1000.0 / ms_e2e, "err_vs_fp64": max_error(H, Y, [0, 1, 31, 63]),
                "operand_bytes": info["tc_bytes"], "fp32_storage_bytes": info["far_bytes"] + info["near_bytes"],
                "clocks": clk.summary()})
    H.close()
    G = build(hmg.PREC_FP64)
    y = torch.empty(n, dtype=torch.float64, device="cuda")
    ms64 = timed(lambda: G.matvec(X[0], y))
    gi = G.info()
    out["fp64_form"] = {"ms_per_product": ms64, "value": 1000.0 / ms64, "unit": "vector products/s",
                        "err_vs_fp64": max_error(G, y.unsqueeze(0), [0]),
                        "storage_bytes": gi["far_bytes"] + gi["near_bytes"]}
    G.close()
    out["speedup_vs_fp64_form"] = out["value"] / out["fp64_form"]["value"]
    return out


def aca_work(H, seconds):
    """Algorithmic work of the adaptive ACA (k_aca, k_aca_warp) per block-size class.
    Rank step l of a block reads its l previous U and V columns twice (the residual
    row / column, then the Frobenius cross terms): 2 l (m1 + m2) FP64 FMAs and as many
    8-byte reads, so a block of rank r costs r (r - 1) (m1 + m2) of each; plus
    (m1 + m2) kernel entries per step."""
    s1l, s1u, s2l, s2u, typ = H.blocks()
    ranks = H.ranks()
    far = typ == 1
    mm = ((s1u - s1l + 1) + (s2u - s2l + 1))[far].astype(np.float64)
    r = ranks[far].astype(np.float64)
    fma = r * (r - 1) * mm
    classes = {}
    for lo, hi in ((0, 512), (512, 2048), (2048, 8192), (8192, 32768), (32768, 1 << 30)):
        sel = (mm >= lo) & (mm < hi)
        classes[f"m1+m2 in [{lo},{hi})"] = {"blocks": int(sel.sum()), "mean_rank": float(r[sel].mean()) if sel.any() else 0.0,
                                            "fp64_gflop": float(2 * fma[sel].sum() / 1e9),
                                            "read_gb": float(8 * fma[sel].sum() / 1e9)}
    total = float(fma.sum())
    return {"fp64_gflop": 2 * total / 1e9, "read_gb": 8 * total / 1e9, "kernel_entries": float((r * mm).sum()),
            "fp64_tflops_achieved": 2 * total / seconds / 1e12 if seconds > 0 else None,
            "read_gbps_achieved": 8 * total / seconds / 1e9 if seconds > 0 else None,
            "by_size": classes}


def run_engine(a, rank, world):
    import torch
    import torch.distributed as dist

    import hmglib_b200 as hmg
    from hmglib_b200 import synth
    from oracle import oracle as O

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    W = WORKLOAD
    n = a.n or W["n"]
    prec = {"fp32": hmg.PREC_FP32, "fp64": hmg.PREC_FP64, "mixed": hmg.PREC_MIXED}[a.prec]
    near_esz = 8 if prec == hmg.PREC_FP64 else 4  # the mixed format stores FP32 near blocks
    p = synth.uniform_points(n, W["dim"], W["seed"])
    x = synth.rhs_vector(n, W["seed"])

    t0 = time.perf_counter()
    H = hmg.HMatrix(n, n, W["dim"])
    H.set_points(0, p)
    H.set_points(1, p)
    H.setup(W["eta"], W["leaf"], rule=hmg.ADMISSIBLE_MIN)
    t_setup = time.perf_counter() - t0
    H.set_kernel(hmg.KERNEL_MATERN32, W["rho"], 0.0)
    t1 = time.perf_counter()
    H.precompute_aca(W["max_rank"], W["aca_eps"], prec)
    t_aca = time.perf_counter() - t1
    near = a.near
    t2 = time.perf_counter()
    if near == "stored":
        try:
            H.precompute_dense(prec)
        except hmg.HmgError as e:
            if e.status != 3:
                raise
            near = "onthefly"
    if near == "onthefly":
        H.set_near_mode(hmg.NEAR_ONTHEFLY)
    t_dense = time.perf_counter() - t2
    H.set_matvec_variant(a.variant)
    H.set_product_precision(hmg.PREC_FP64 if a.arith == "fp64" else hmg.PREC_FP32)
    streaming = a.variant == 0 and near == "stored"
    tile_kernel = "k_tiles_bulk" if streaming else "k_tile_matvec"
    info = H.info()

    dx = torch.from_numpy(x).cuda()
    dy = torch.empty(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.default_stream()
    # the V^T x task size and grid for this H-matrix (hmg_autotune), before any timing
    tuned = H.autotune(reps=3) if not a.no_autotune else None
    for _ in range(max(3, a.warmup)):
        H.matvec(dx, dy)
    H.synchronize()
    # per-kernel device times (events between the product's kernels)
    H.set_profiling(True)
    prof = []
    for _ in range(3):
        H.matvec(dx, dy)
        prof.append(H.profile())
    H.set_profiling(False)
    k2_ms = float(np.median([q["tiles_ms"] for q in prof]))
    k1_ms = float(np.median([q["vtx_ms"] for q in prof]))

    # accuracy vs the FP64 direct sum on a row sample (on the GPU)
    rng = np.random.default_rng(7)
    rows = torch.from_numpy(rng.choice(n, size=min(n, 4096), replace=False).astype(np.int32)).cuda()
    yd = torch.empty(rows.shape[0], dtype=torch.float64, device="cuda")
    H.matvec(dx, dy)
    H.full_matvec_rows(dx, rows, yd)
    H.synchronize()
    err = float(torch.linalg.norm(dy[rows.long()] - yd) / torch.linalg.norm(yd))

    if world > 1:
        dist.barrier()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(a.steps):
            H.matvec(dx, dy)
        ev1.record(stream)
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        # end-to-end through the host-buffer C-ABI call
        xh = np.ascontiguousarray(x)
        yh = np.empty(n)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        H.matvec(xh, yh)
        e0.record(stream)
        for _ in range(a.steps):
            H.matvec(xh, yh)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_e2e = e0.elapsed_time(e1)
        # the same products, each replayed as one captured CUDA graph (hmg_set_graphs)
        H.set_graphs(True)
        H.matvec(dx, dy)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(a.steps):
            H.matvec(dx, dy)
        e1.record(stream)
        torch.cuda.synchronize()
        ms_graph = e0.elapsed_time(e1)
        H.set_graphs(False)
    ms, ms_e2e, ms_graph = max_over_ranks([ms, ms_e2e, ms_graph], world, "cuda")
    ms_step = ms / a.steps
    value = world * 1000.0 / ms_step
    e2e_value = world * 1000.0 * a.steps / ms_e2e

    peak, peak_kind = _peaks()
    # algorithmic bytes of the tile kernel per launch: near entries and U factors
    # streamed once, y written once (plus the permutation read)
    near_b = info["near_entries"] * near_esz if near == "stored" else 0
    u_b = int(info["far_u_bytes"])
    v_b = int(info["far_v_bytes"])
    k2_bytes = near_b + u_b + 12 * n
    traffic_known = a.prec == "mixed" and near == "stored" and not streaming and a.arith == "fp32"
    achieved = k2_bytes / (k2_ms * 1e-3) / 1e9
    whole_bytes = near_b + u_b + v_b + 8 * 2 * n
    line = {
        "metric": METRIC, "value": value, "unit": "matvec/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if (a.prec == "fp64" or a.arith == "fp64") else "f32",
        "data": "synthetic",
        "config": dict(W, n=n, near=near, storage=a.prec, arithmetic="fp64" if a.prec == "fp64" else a.arith,
                       parallelism=f"replicas{world}",
                       l2="inputs larger than L2 (no flush)"),
        "err_vs_fp64": err,
        "e2e": {"value": e2e_value, "unit": "matvec/s", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n},
        "gpu_launches": (3 if streaming else info["matvec_launches"]) * a.steps,
        "roofline": {"bound": "hbm", "kernel": tile_kernel, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     # DRAM bytes / algorithmic bytes of k_tile_matvec measured by ncu on the
                     # N=131072 case of this workload (mixed storage), scaled to this launch
                     "traffic": (K2_TRAFFIC_RATIO * k2_bytes) if traffic_known else None,
                     "traffic_source": "ncu, N=131072 case, scaled by algorithmic bytes" if traffic_known else None,
                     "peak_kind": peak_kind, "bytes_per_launch": k2_bytes, "ms_per_launch": k2_ms},
        "whole_matvec": {"bytes": whole_bytes, "GBps": whole_bytes / (ms_step * 1e-3) / 1e9,
                         "frac": whole_bytes / (ms_step * 1e-3) / 1e9 / peak, "vtx_ms": k1_ms,
                         "tiles_ms": k2_ms},
        "build_s": {"setup": t_setup, "aca": t_aca, "dense": t_dense},
        "aca_work": aca_work(H, t_aca),
        "hmatrix": {k: info[k] for k in ("block_count", "dense_count", "aca_count", "levels", "tile_count",
                                         "max_rank", "near_entries", "far_entries", "near_bytes", "far_bytes")},
        "clocks": clk.summary(),
        "graph_replay": {"ms_per_step": ms_graph / a.steps, "value": world * 1000.0 * a.steps / ms_graph,
                         "unit": "matvec/s"},
        "autotune": tuned,
    }
    if a.nrhs > 1:
        line["multi_rhs"] = multi_rhs_timing(torch, H, x, n, a.nrhs, a.steps, stream, world, err)
        if a.tc:
            modes = {"bf16": ("multi_rhs_tensor_cores", hmg.PREC_BF16),
                     "near-fp32": ("multi_rhs_tensor_cores_near_fp32", hmg.PREC_FP32),
                     "bf16x3": ("multi_rhs_tensor_cores_bf16x3", hmg.PREC_BF16X3),
                     "bf16x6": ("multi_rhs_tensor_cores_bf16x6", hmg.PREC_BF16X6)}
            for name in (modes if a.tc_mode == "all" else [a.tc_mode]):
                key, prec = modes[name]
                H.build_bf16_factors(near=prec)
                line[key] = multi_rhs_timing(torch, H, x, n, a.nrhs, a.steps, stream, world, err)
    if a.nrhs > 1 and not a.no_onchip:
        line["onchip_tensor_cores"] = onchip_tensor_cores(torch, hmg, H, x, n, a.steps, stream, world, peak)
    if rank == 0 and world == 1 and not a.no_cpu:
        kind = O.KERNEL_MATERN32
        rate, nrows, dt, thr = cpu_direct_rate(p, x, kind, O.kernel_param(kind, W["rho"]), target_s=a.cpu_seconds)
        line["cpu_baseline"] = {"value": rate / n, "unit": "matvec/s", "cores": thr, "kind": "port",
                                "sample": f"FP64 direct sum over {nrows} random rows ({dt:.1f} s), scaled to N={n}"}
    H.close()
    if world == 1 and not a.no_batched_tc:
        line["batched_tensor_cores"] = batched_tensor_cores(a.steps)
    if world == 1 and a.serve_in_default > 0:
        # the serving workload, short: p50/p99 latency of products and solves
        r = serve_measure(a, a.serve_in_default, 0, local)
        lat = r["latency"]
        line["serve"] = {"requests": r["requests"], "completed": r["completed"], "refused": r["refused"],
                         "p50_ms": lat.get("all", {}).get("p50_ms"), "p99_ms": lat.get("all", {}).get("p99_ms"),
                         "by_class": {k: v for k, v in lat.items() if k != "all"},
                         "requests_per_s": r["requests_per_s"], "solves": r["solves"],
                         "matvec_batch": r["matvec_batch"], "resident_gb": r["resident_gb"],
                         "latency_targets_s": r["latency_targets_s"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def ridge_feasibility(torch, hmg, H, n, shifts, steps=60, cg_maxit=600, seed=5):
    """Is (H + shift I) positive definite, as CG needs?  Arnoldi on H with FP64-
    arithmetic products (full reorthogonalisation, `steps` vectors) gives V^T H V; its
    symmetric part is the Rayleigh-Ritz projection of S = (H + H^T) / 2, whose
    eigenvalues lie in [lambda_min(S), lambda_max(S)], so its smallest one theta_min
    bounds lambda_min(S) from above, and x^T (H + shift I) x = x^T (S + shift I) x for
    every x.  theta_min + shift < 0 therefore proves that CG can meet p^T A p <= 0;
    the Ritz vector's quadratic form, recomputed with one more FP64 product, confirms
    it.  Then the CG solve (with refinement) at each shift, to 1e-8."""
    H.set_product_precision(hmg.PREC_FP64)
    V = torch.empty(steps + 1, n, dtype=torch.float64, device="cuda")
    g = torch.Generator(device="cpu").manual_seed(seed)
    v = torch.rand(n, generator=g, dtype=torch.float64).cuda() - 0.5
    V[0] = v / torch.linalg.norm(v)
    Hm = torch.zeros(steps + 1, steps, dtype=torch.float64)
    w = torch.empty(n, dtype=torch.float64, device="cuda")
    m = steps
    for j in range(steps):
        H.matvec(V[j], w)
        torch.cuda.synchronize()
        for _ in range(2):  # Gram-Schmidt twice
            c = V[:j + 1] @ w
            w -= V[:j + 1].T @ c
            Hm[:j + 1, j] += c.cpu()
        nb = float(torch.linalg.norm(w))
        Hm[j + 1, j] = nb
        if nb < 1e-12:
            m = j + 1
            break
        V[j + 1] = w / nb
    T = Hm[:m, :m].numpy()
    S = 0.5 * (T + T.T)
    theta, Y = np.linalg.eigh(S)
    x = (V[:m].T @ torch.from_numpy(Y[:, 0]).cuda()).contiguous()
    H.matvec(x, w)
    torch.cuda.synchronize()
    q = float(x @ w) / float(x @ x)
    asym = float(np.abs(T - T.T)[np.triu_indices(m, 2)].max()) if m > 2 else 0.0
    out = {"arnoldi_steps": m, "theta_min": float(theta[0]), "theta_max": float(theta[-1]),
           "rayleigh_min_ritz_vector": q, "hessenberg_above_band_max": asym, "shifts": {}}
    del V
    H.set_product_precision(hmg.PREC_FP32)
    b = torch.from_numpy(np.random.default_rng(seed).uniform(-1, 1, n)).cuda()
    for sh in shifts:
        xs = torch.zeros_like(b)
        t0 = time.perf_counter()
        try:
            it, rel = H.cg_solve(b, xs, sh, tol=1e-8, maxit=cg_maxit, refine=True)
            res = {"iterations": it, "relres": rel, "converged": rel <= 1e-8}
        except hmg.HmgError as e:  # p^T A p <= 0 met by CG
            res = {"error": str(e), "converged": False}
        res["seconds"] = time.perf_counter() - t0
        res["lambda_min_upper_bound"] = float(theta[0]) + sh
        out["shifts"][str(sh)] = res
    return out


def run_precision(a, rank, world):
    """The precision workload: N = 2^21 points in 2D from a 16-component Gaussian
    mixture (seed 2), Gaussian kernel length^2 0.05, ACA eps 1e-6.  Products of 32
    vectors per pass with FP32 factors and with mixed (FP32/FP16/FP8) factors, FP32
    near field, FP32 products summed in FP64 (and on the tensor cores: BF16 copies of the
    FP32 factors; three BF16 parts split on chip from the mixed storage), and a
    kernel-ridge CG solve of
    (K + 1e-3 I) x = b to relative residual 1e-8 with refinement (FP64 residuals,
    relaxed-precision inner products).  Each result's error against FP64 direct sums
    over 2,048 sampled rows is reported."""
    import torch

    import hmglib_b200 as hmg
    from hmglib_b200 import synth
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    n, nrhs = a.n or (1 << 21), 32
    p = synth.gmm_points(n, 2, 2)
    X = torch.from_numpy(synth.rhs_vector(n, 2, nrhs)).cuda()
    rows = torch.from_numpy(np.random.default_rng(9).choice(n, 2048, replace=False).astype(np.int32)).cuda()
    out = {}
    stream = torch.cuda.default_stream()
    for name, prec in (("fp32", hmg.PREC_FP32), ("mixed", hmg.PREC_MIXED)):
        t0 = time.perf_counter()
        H = hmg.HMatrix(n, n, 2)
        H.set_points(0, p)
        H.set_points(1, p)
        H.setup(1.5, 64, rule=hmg.ADMISSIBLE_MIN)
        H.set_kernel(hmg.KERNEL_GAUSSIAN, 0.05, 0.0)
        H.precompute_aca(64, 1e-6, prec)
        H.precompute_dense(hmg.PREC_FP32)
        torch.cuda.synchronize()
        t_build = time.perf_counter() - t0
        Y = torch.empty_like(X)
        for _ in range(2):
            H.matvec_multi(X, Y)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(a.steps):
            H.matvec_multi(X, Y)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.steps
        errs = []
        for j in range(0, nrhs, 8):
            yd = torch.empty(rows.shape[0], dtype=torch.float64, device="cuda")
            H.full_matvec_rows(X[j], rows, yd)
            torch.cuda.synchronize()
            errs.append(float(torch.linalg.norm(Y[j][rows.long()] - yd) / torch.linalg.norm(yd)))
        info = H.info()
        if prec == hmg.PREC_FP32:
            # tensor cores: BF16 factors with the near field in FP32 on the CUDA cores (the
            # configuration as specified), then with the near field in BF16 as well
            tc = {}
            for near in (hmg.PREC_FP32, hmg.PREC_BF16):
                H.build_bf16_factors(near=near)
                Yt = torch.empty_like(X)
                for _ in range(2):
                    H.matvec_multi(X, Yt)
                torch.cuda.synchronize()
                e0.record(stream)
                for _ in range(a.steps):
                    H.matvec_multi(X, Yt)
                e1.record(stream)
                torch.cuda.synchronize()
                ms_tc = e0.elapsed_time(e1) / a.steps
                errs_tc = []
                for j in range(0, nrhs, 8):
                    yd = torch.empty(rows.shape[0], dtype=torch.float64, device="cuda")
                    H.full_matvec_rows(X[j], rows, yd)
                    torch.cuda.synchronize()
                    errs_tc.append(float(torch.linalg.norm(Yt[j][rows.long()] - yd) / torch.linalg.norm(yd)))
                tc["near_fp32_cuda_cores" if near == hmg.PREC_FP32 else "near_bf16_tensor_cores"] = {
                    "ms_per_32_vectors": ms_tc, "vectors_per_s": nrhs * 1000.0 / ms_tc, "err_vs_fp64_max": max(errs_tc)}
        res = {"ms_per_32_vectors": ms, "vectors_per_s": nrhs * 1000.0 / ms, "err_vs_fp64_max": max(errs),
               "build_s": t_build, "far_gb": info["far_bytes"] / 1e9, "near_gb": info["near_bytes"] / 1e9,
               "max_rank": info["max_rank"]}
        if prec == hmg.PREC_FP32:
            res["bf16_tensor_cores"] = tc
        if prec == hmg.PREC_MIXED:
            # tensor cores over the same mixed storage, every operand split into three
            # BF16 parts on chip (no copy; error <= 1e-6 territory)
            t0 = time.perf_counter()
            H.build_bf16_factors(near=hmg.PREC_BF16X6_ONCHIP)
            t_plan = time.perf_counter() - t0
            Yt = torch.empty_like(X)
            for _ in range(2):
                H.matvec_multi(X, Yt)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(a.steps):
                H.matvec_multi(X, Yt)
            e1.record(stream)
            torch.cuda.synchronize()
            ms_oc = e0.elapsed_time(e1) / a.steps
            errs_oc = []
            for j in range(0, nrhs, 8):
                yd = torch.empty(rows.shape[0], dtype=torch.float64, device="cuda")
                H.full_matvec_rows(X[j], rows, yd)
                torch.cuda.synchronize()
                errs_oc.append(float(torch.linalg.norm(Yt[j][rows.long()] - yd) / torch.linalg.norm(yd)))
            res["onchip_tensor_cores"] = {"ms_per_32_vectors": ms_oc, "vectors_per_s": nrhs * 1000.0 / ms_oc,
                                          "err_vs_fp64_max": max(errs_oc), "plan_s": t_plan}
        if name == "fp32" and not a.no_feasibility:
            res["ridge_feasibility"] = ridge_feasibility(torch, hmg, H, n, [1e-3, 1e-2, 1e-1, 1.0],
                                                         cg_maxit=a.cg_maxit)
        if name == "fp32":
            b = X[0].clone()
            x = torch.zeros_like(b)
            t0 = time.perf_counter()
            it, rel = H.cg_solve(b, x, 1e-3, tol=1e-8, maxit=a.cg_maxit, refine=True)
            t_cg = time.perf_counter() - t0
            yx = torch.empty(rows.shape[0], dtype=torch.float64, device="cuda")
            H.full_matvec_rows(x, rows, yx)
            torch.cuda.synchronize()
            r_ex = float(torch.linalg.norm(b[rows.long()] - (yx + 1e-3 * x[rows.long()])) / torch.linalg.norm(b[rows.long()]))
            res["cg"] = {"iterations": it, "relres_operator": rel, "relres_exact_kernel_rows": r_ex, "seconds": t_cg,
                         "tol": 1e-8, "maxit": a.cg_maxit}
        out[name] = res
        H.close()
    line = {"metric": "32-vector H-matvecs at N=2^21 (GMM 2D, Gaussian l^2 0.05, eps 1e-6)",
            "value": out["fp32"]["vectors_per_s"], "unit": "vector products/s", "n_gpus": 1, "steps": a.steps,
            "warmup": 2, "ms_per_step": out["fp32"]["ms_per_32_vectors"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "precision_gmm2d_2m_32rhs", "n": n, "nrhs": nrhs, "aca_eps": 1e-6,
                       "near": "fp32"},
            "results": out}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_group(a, rank, world):
    """Many independent H-matrices (512 sets, sizes log-uniform in [2^10, 2^16], half 2D
    and half 3D, Gaussian length^2 U[0.01, 0.2], FP32 factors, ACA eps 1e-5): one
    grouped H-matrix multiplied in one set of launches, against the same sets
    compressed and multiplied one handle at a time.  One step = every set once.
    Clustering is timed both ways: hmg_setup per set then hmg_group_create, and
    hmg_group_setup (every set ordered and clustered in the same launches)."""
    import torch

    import hmglib_b200 as hmg
    from hmglib_b200 import synth
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    count = a.group_count
    sets = synth.group_sets(count, 3)
    leaf = [64 if p.shape[0] == 2 else 128 for p, _ in sets]

    def handles():
        out = []
        for p, l2 in sets:
            dim, n = p.shape
            H = hmg.HMatrix(n, n, dim)
            H.set_points(0, p)
            H.set_points(1, p)
            H.set_kernel(hmg.KERNEL_GAUSSIAN, l2, 0.0)
            out.append(H)
        return out
    t0 = time.perf_counter()
    hs = handles()
    t_handles = time.perf_counter() - t0
    # clustering one set at a time (hmg_setup per set, then hmg_group_create) ...
    t0 = time.perf_counter()
    for H, c in zip(hs, leaf):
        H.setup(1.5, c, rule=hmg.ADMISSIBLE_MIN)
    t_setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    G = hmg.group(hs)
    t_group = time.perf_counter() - t0
    # ... and every set in the same launches (hmg_group_setup): the same handle
    raw = handles()
    t0 = time.perf_counter()
    G1 = hmg.group_setup(raw, 1.5, leaf, rule=hmg.ADMISSIBLE_MIN)
    t_group_setup = time.perf_counter() - t0
    same_tree = all(bool(np.array_equal(u, v)) for u, v in zip(G.blocks(), G1.blocks())) and \
        all(bool(np.array_equal(G.order(w), G1.order(w))) for w in (0, 1))
    G1.close()
    for H in raw:
        H.close()
    off = G.offsets(0)
    n = int(off[-1])
    x = synth.rhs_vector(n, 3)
    stream = torch.cuda.default_stream()

    # one handle at a time: compression and products in a loop over the sets
    t0 = time.perf_counter()
    for H in hs:
        H.precompute_aca(64, 1e-5, hmg.PREC_FP32)
        H.precompute_dense(hmg.PREC_FP32)
    torch.cuda.synchronize()
    t_build_loop = time.perf_counter() - t0
    dx = torch.from_numpy(x).cuda()
    dy_loop = torch.empty_like(dx)
    xs = [dx[off[i]:off[i + 1]] for i in range(count)]
    ys = [dy_loop[off[i]:off[i + 1]] for i in range(count)]

    def loop_step():
        for H, xi, yi in zip(hs, xs, ys):
            H.matvec(xi, yi)
    for _ in range(a.warmup):
        loop_step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        loop_step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_loop = e0.elapsed_time(e1) / a.steps
    # accuracy on 8 sets against their FP64 direct sums
    errs = []
    for i in range(0, count, max(1, count // 8)):
        yd = torch.empty_like(xs[i])
        hs[i].full_matvec(xs[i], yd)
        torch.cuda.synchronize()
        errs.append(float(torch.linalg.norm(ys[i] - yd) / torch.linalg.norm(yd)))
    y_loop = dy_loop.clone()
    for H in hs:
        H.close()

    # the group: one compression and one product launch set for all sets
    t0 = time.perf_counter()
    G.precompute_aca(64, 1e-5, hmg.PREC_FP32)
    G.precompute_dense(hmg.PREC_FP32)
    torch.cuda.synchronize()
    t_build_group = time.perf_counter() - t0
    info = G.info()
    dy = torch.empty_like(dx)
    for _ in range(a.warmup):
        G.matvec(dx, dy)
    torch.cuda.synchronize()
    same = bool(torch.equal(dy, y_loop))
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(a.steps):
            G.matvec(dx, dy)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    # end to end: x from pinned host memory in, y out
    xp = torch.from_numpy(x).pin_memory()
    yp = torch.empty(n, dtype=torch.float64).pin_memory()
    e0.record(stream)
    for _ in range(a.steps):
        dx.copy_(xp, non_blocking=True)
        G.matvec(dx, dy)
        yp.copy_(dy, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1) / a.steps
    peak, peak_kind = _peaks()
    bytes_ = info["matvec_bytes"]
    line = {
        "metric": f"grouped H-matvecs/s ({count} sets, every set once per step)", "value": 1000.0 / ms,
        "unit": "group products/s", "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"group{count}_gauss_mixed2d3d", "sets": count, "points": n, "aca_eps": 1e-5,
                   "max_rank": 64, "storage": "fp32", "l2": "inputs larger than L2 (no flush)"},
        "loop_one_handle_at_a_time": {"ms_per_step": ms_loop, "speedup_group": ms_loop / ms,
                                      "build_s": t_build_loop},
        "group_equals_loop": same, "err_vs_fp64_sets": max(errs),
        "e2e": {"value": 1000.0 / ms_e2e, "unit": "group products/s", "h2d_bytes_per_step": 8 * n,
                "d2h_bytes_per_step": 8 * n},
        "gpu_launches": info["matvec_launches"] * a.steps,
        "roofline": {"bound": "hbm", "kernel": "whole product", "achieved": bytes_ / (ms * 1e-3) / 1e9,
                     "peak": peak, "unit": "GB/s", "frac": bytes_ / (ms * 1e-3) / 1e9 / peak, "traffic": None,
                     "peak_kind": peak_kind, "bytes_per_launch": bytes_},
        "build_s": {"handles": t_handles, "setup_sets": t_setup, "group_create": t_group,
                    "group_setup": t_group_setup, "group_setup_equals_setup_sets": same_tree,
                    "aca_dense_group": t_build_group},
        "hmatrix": {k: info[k] for k in ("block_count", "dense_count", "aca_count", "tile_count", "max_rank",
                                         "near_bytes", "far_bytes")},
        "clocks": clk.summary(),
    }
    G.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


SERVE_SIZES = [1 << 16] * 4 + [1 << 17, 1 << 18, 1 << 19, 1 << 20]


def serve_measure(a, n_requests, n_baseline, local=0):
    """The serving workload: 8 resident H-matrices (four of 2^16 points, then 2^17, 2^18,
    2^19, 2^20; uniform 3D, Matern-3/2 rho 0.2, leaf 64, ACA eps 1e-4, mixed storage:
    ~96 GB) and a Poisson stream at 2000 requests/s (seed 4): 80% single-vector
    products, 15% 8-vector kernel-ridge solves (shift 1e-3 N, relative residual 1e-4,
    the library's block CG with FP64 refinement), 5% new point sets of 2^14-2^18
    points, under a 120 GB budget, with latency targets (--serve-slo-matvec,
    --serve-slo-solve seconds): a request whose predicted completion misses its target
    is refused on arrival.  Returns p50/p99 latency of the completed requests, the
    refused counts and (n_baseline > 0) throughput against the plain FP64
    one-request-at-a-time path (FP64 products, one vector per call, solves by
    hmg_cg_solve per column) on the same H-matrices and the first n_baseline requests."""
    import torch

    import hmglib_b200 as hmg
    from hmglib_b200 import serve, synth
    sizes = SERVE_SIZES
    t0 = time.perf_counter()
    slo = {"matvec": a.serve_slo_matvec, "solve": a.serve_slo_solve}
    srv = serve.Server(budget_bytes=120e9, slo_s=slo)
    for i, n in enumerate(sizes):
        st = torch.cuda.Stream()
        H = serve.build_hmatrix(synth.uniform_points(n, 3, 4000 + i), hmg.KERNEL_MATERN32, 0.2, 1e-4,
                                hmg.PREC_MIXED, stream=st.cuda_stream, leaf=64)
        srv.add(H, st)
    t_build = time.perf_counter() - t0
    resident = srv.used_bytes()
    reqs = serve.poisson_requests(n_requests, 2000.0, sizes, seed=4, eps=1e-4, shift_per_point=1e-3,
                                  tol=1e-4)
    print(f"serve: resident {srv.used_bytes() / 1e9:.1f} GB built in {t_build:.1f} s; {len(reqs)} requests",
          file=sys.stderr, flush=True)
    # warm-up: a product and three solve iterations on every resident matrix (seeds the
    # service-time estimates the latency targets are checked against)
    warm = [serve.Matvec(m, np.zeros(n)) for m, n in enumerate(sizes)]
    warm += [serve.Solve(m, synth.uniform01(77 + m, 8 * n).reshape(8, n), 1e-3 * n, tol=1e-12, maxit=3)
             for m, n in enumerate(sizes)]
    srv.run(warm)
    srv.iters_per_solve = 30.0  # the warm-up solves stop at 3 iterations: not a solve length
    with ClockSampler(local) as clk:
        done, wall = srv.run(reqs, time_limit=300.0)
    print(f"serve: {len(reqs)} requests served in {wall:.1f} s", file=sys.stderr, flush=True)
    lat = serve.latency_summary(done)
    solves = [q for q in done if isinstance(q, serve.Solve) and q.done is not None and q.rejected is None]
    solve_stats = {"iters_mean": float(np.mean([q.iters for q in solves])) if solves else None,
                   "converged": int(sum(bool((q.relres <= q.tol).all()) for q in solves)),
                   "count": len(solves)}
    builds = [q for q in done if isinstance(q, serve.Build)]
    build_stats = {"admitted": sum(q.mid is not None for q in builds), "refused": sum(q.rejected is not None for q in builds)}
    n_done = sum(q.done is not None and getattr(q, "rejected", None) is None for q in done)
    n_refused = sum(getattr(q, "rejected", None) is not None for q in done)
    batches = [q.batch for q in done if isinstance(q, serve.Matvec) and q.rejected is None]
    out = {
        "requests": len(reqs), "completed": n_done, "seconds": wall, "requests_per_s": n_done / wall,
        "latency": lat, "refused": n_refused, "admitted_fraction": 1.0 - n_refused / max(1, len(reqs)),
        "matvec_batch": {"mean": float(np.mean(batches)) if batches else None,
                         "max": int(np.max(batches)) if batches else None},
        "solves": solve_stats, "builds": build_stats, "resident_gb": resident / 1e9, "build_s": t_build,
        "clocks": clk.summary(), "latency_targets_s": slo,
    }
    # the plain path: one request at a time, FP64 products, no batching, no overlap
    nb = min(n_baseline, len(reqs))
    if nb > 0:
        base = reqs[:nb]
        for r in srv.res.values():
            r.H.set_product_precision(hmg.PREC_FP64)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for q in base:
            if isinstance(q, serve.Matvec):
                srv.res[q.mid].H.matvec(q.x)
            elif isinstance(q, serve.Solve):
                H = srv.res[q.mid].H
                for j in range(q.B.shape[0]):
                    b = torch.from_numpy(q.B[j]).cuda()
                    x = torch.zeros_like(b)
                    H.cg_solve(b, x, q.shift, tol=q.tol, maxit=q.maxit, refine=False)
            else:
                Hn = serve.build_hmatrix(q.points, q.kind, q.param, q.eps, hmg.PREC_FP64)
                Hn.close()
        torch.cuda.synchronize()
        t_base = time.perf_counter() - t0
        out["plain_fp64_one_at_a_time"] = {"requests": nb, "seconds": t_base, "requests_per_s": nb / t_base,
                                           "throughput_ratio_served_vs_plain": (n_done / wall) / (nb / t_base)}
    for mid in list(srv.res):
        srv.res.pop(mid).H.close()
    return out


def run_serve(a, rank, world):
    """The serving workload on its own (serve_measure), as its own JSON line."""
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    r = serve_measure(a, a.serve_requests, a.serve_baseline, local)
    line = {
        "metric": "served requests/s (8 resident H-matrices, Poisson 2000 req/s); p50/p99 latency",
        "value": r["requests_per_s"], "unit": "requests/s", "n_gpus": 1, "steps": r["requests"], "warmup": 16,
        "ms_per_step": 1000.0 * r["seconds"] / max(1, r["completed"]), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "serve_8resident_matern3d_poisson2000", "sizes": SERVE_SIZES, "aca_eps": 1e-4,
                   "leaf": 64, "storage": "mixed", "budget_gb": 120, "requests": r["requests"],
                   "mix": [0.8, 0.15, 0.05], "latency_targets_s": r["latency_targets_s"]},
        "e2e": {"value": r["requests_per_s"], "unit": "requests/s", "h2d_bytes_per_step": None,
                "d2h_bytes_per_step": None},
    }
    line.update({k: v for k, v in r.items() if k not in ("requests_per_s", "latency_targets_s")})
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_legacy(a, rank, world):
    """The reference's own configurations (tests/golden: config 1, N=16384 2D, exp(-r^2)
    with coordinates scaled by 1/sqrt(0.1), leaf 64, max rule, fixed rank 64; and the
    N=8192 3D case of its Bessel-Y kernel, rank 16), in its arithmetic (FP64 factors and
    near field, fixed-rank ACA): the engine's setup, compression, near-field fill and
    H-matvec timed with CUDA events, beside the reference's own GPU build timed on a
    B200 by the fixture generator (the same inputs; tests/golden/make_golden.py)."""
    import torch

    import hmglib_b200 as hmg
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests"))
    from golden.make_golden import CASES, case_inputs
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    stream = torch.cuda.default_stream()
    out = {}
    for name in ("config1_parity", "uniform3d_matern"):
        c = CASES[name]
        p1, p2, x = case_inputs(c)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(10)]
        H = hmg.HMatrix(p1.shape[1], p2.shape[1], p1.shape[0])
        ev[0].record(stream)
        H.set_points(0, p1)
        H.set_points(1, p2)
        H.setup(c["eta"], c["c_leaf"], rule=hmg.ADMISSIBLE_MAX)
        H.set_kernel(c["kernel"], 0.0, 0.0)
        ev[1].record(stream)
        H.precompute_aca(c["k"], 0.0, hmg.PREC_FP64)
        ev[2].record(stream)
        H.precompute_dense(hmg.PREC_FP64)
        ev[3].record(stream)
        dx = torch.from_numpy(x).cuda()
        dy = torch.empty(p1.shape[1], dtype=torch.float64, device="cuda")
        for _ in range(a.warmup):
            H.matvec(dx, dy)
        ev[4].record(stream)
        for _ in range(a.steps):
            H.matvec(dx, dy)
        ev[5].record(stream)
        H.full_matvec(dx, dy)
        ev[6].record(stream)
        torch.cuda.synchronize()
        g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", name + ".npz"))
        ref = [float(v) for v in g["timings_ms"]]
        out[name] = {
            "n": int(p1.shape[1]), "dim": int(p1.shape[0]), "rank": c["k"], "leaf": c["c_leaf"],
            "engine_ms": {"setup": ev[0].elapsed_time(ev[1]), "precompute_aca": ev[1].elapsed_time(ev[2]),
                          "precompute_dense": ev[2].elapsed_time(ev[3]),
                          "apply": ev[4].elapsed_time(ev[5]) / a.steps, "apply_full": ev[5].elapsed_time(ev[6])},
            "reference_gpu_ms": {"setup": ref[0], "precompute_aca": ref[1], "precompute_dense": ref[2],
                                 "apply": ref[3], "apply_full": ref[4]},
        }
        out[name]["apply_speedup"] = ref[3] / out[name]["engine_ms"]["apply"]
        H.close()
    c1 = out["config1_parity"]
    line = {"metric": "H-matvecs/s, the reference's configuration 1 (N=16384 2D, FP64, fixed rank 64)",
            "value": 1000.0 / c1["engine_ms"]["apply"], "unit": "matvec/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": c1["engine_ms"]["apply"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "reference_configurations", "cases": list(out)}, "results": out}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--n", type=int, default=0, help="override the point count (default 2^20)")
    ap.add_argument("--prec", default="mixed", choices=["fp32", "fp64", "mixed"])
    ap.add_argument("--near", default="stored", choices=["stored", "onthefly"])
    ap.add_argument("--nrhs", type=int, default=32,
                    help="also time products of this many vectors at once (hmg_matvec_multi)")
    ap.add_argument("--tc-mode", default="all", choices=["all", "bf16", "near-fp32", "bf16x3", "bf16x6"],
                    help="tensor-core operand modes --tc measures")
    ap.add_argument("--tc", action="store_true",
                    help="with --nrhs and --prec fp32: also time the tensor-core path (BF16 factor copy)")
    ap.add_argument("--arith", default="fp32", choices=["fp32", "fp64"],
                    help="arithmetic of the products over FP32/mixed storage")
    ap.add_argument("--variant", type=int, default=1, choices=[0, 1],
                    help="product kernels: 1 plain 16-byte loads (default), 0 bulk-copy streaming")
    ap.add_argument("--workload", default="uniform3d", choices=["uniform3d", "group", "serve", "precision", "legacy"],
                    help="uniform3d: the N=2^20 headline; group: many small H-matrices as one; "
                         "serve: the request loop over resident H-matrices")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default V^T x task size and grid")
    ap.add_argument("--serve-requests", type=int, default=300)
    ap.add_argument("--serve-in-default", type=int, default=60,
                    help="requests of the short serving run added to the default line (0: none)")
    ap.add_argument("--serve-slo-matvec", type=float, default=1.0, help="latency target of a product, seconds")
    ap.add_argument("--serve-slo-solve", type=float, default=10.0, help="latency target of a solve, seconds")
    ap.add_argument("--cg-maxit", type=int, default=600)
    ap.add_argument("--no-feasibility", action="store_true",
                    help="precision workload: skip the positive-definiteness study of H + shift I")
    ap.add_argument("--serve-baseline", type=int, default=60)
    ap.add_argument("--group-count", type=int, default=512)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-onchip", action="store_true",
                    help="skip the 64-vector tensor-core products over the mixed storage (on-chip operands)")
    ap.add_argument("--no-batched-tc", action="store_true",
                    help="skip the tensor-core batched products at N=2^18 beside the FP64 form")
    a = ap.parse_args(argv)
    a.warmup = max(3, a.warmup)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if a.impl == "reference":
        return run_reference(a, rank, world)
    if a.workload == "group":
        return run_group(a, rank, world) if rank == 0 else 0
    if a.workload == "serve":
        return run_serve(a, rank, world) if rank == 0 else 0
    if a.workload == "legacy":
        return run_legacy(a, rank, world)
    if a.workload == "precision":
        return run_precision(a, rank, world) if rank == 0 else 0
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        return run_engine(a, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
