#!/usr/bin/env python
"""Benchmark: FP64 multifrontal numeric factorization + supernodal solve.

Workload (default): the 64^3 7-point Laplacian generated exactly as the
reference's taucs_ccs_generate_mesh3d(64,64,64) (n = 262,144), AMD ordering,
one right-hand side b = A x_true with x_true ~ U(-1,1) (seed 0).  One STEP is
one numeric factorization on the analysed pattern plus one solve -- the
reference's taucs_ccs_factor_llt_numeric + taucs_supernodal_solve_llt
(src/taucs_sn_llt.c:2169-2209, :2844-2885).  Ordering and symbolic analysis
happen once, before the timed region, as in the reference's pattern-reuse
path (src/taucs_linsolve.c:433-453).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line (rank 0).  `value` is whole-job systems/s with the
matrix values and b resident in device memory; `e2e` is the same metric
through the C ABI with pinned host buffers (values, b in; x out) copied
inside every step.  Under torchrun every rank factors its own replica (no
collective on the data path; max over ranks for time).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fp64 numeric factor + solve throughput (64^3 7-point Laplacian, AMD)"
UNIT = "systems/s"

KC = dict(small_front=0, build=1, potrf=2, trsm=3, gemm_panel=4, gemm_u=5, solve_fwd=6, solve_bwd=7)
TENSOR_KC = {"gemm_panel", "gemm_u", "trsm", "potrf"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=64, help="mesh side (64 = the benchmark configuration)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def scaled_residual(A, x, b):
    r = A.matvec(x) - b
    return float(np.max(np.abs(r)) / (A.inf_norm() * np.max(np.abs(x)) + np.max(np.abs(b))))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def fp64_gemm_peak():
    """cuBLAS DGEMM 8192^3, best of 5 (FP64 has no entry in MEASURED_PEAKS.json)."""
    import torch
    n = 8192
    a = torch.randn(n, n, device="cuda", dtype=torch.float64)
    b = torch.randn(n, n, device="cuda", dtype=torch.float64)
    best = 0.0
    for _ in range(6):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        a @ b
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    del a, b
    torch.cuda.empty_cache()
    return best


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def cpu_baseline(grid, n_threads):
    """The reference's own CPU multifrontal path (oracle/_ref), one numeric
    factorization + one solve of the same system, on this host's cores."""
    from oracle.bindings import Port, Ref, ref_available
    if ref_available():
        R = Ref(threads=n_threads)
        R.set_threads(n_threads)
        n, cp, ri, va = R.mesh3d(grid, grid, grid)
        perm, iperm = R.order(n, cp, ri, va, "amd")
        _, pc, pr, pv = R.permute(n, cp, ri, va, perm, iperm)
        L = R.symbolic(n, pc, pr, pv)
        xt = np.random.default_rng(0).uniform(-1, 1, n)
        b = Port().spmv(n, pc, pr, pv, xt)
        t0 = time.perf_counter()
        assert R.numeric(L, n, pc, pr, pv) == 0
        x = R.solve(L, b)
        dt = time.perf_counter() - t0
        R.free(L)
        return {"value": 1.0 / dt, "unit": UNIT, "cores": n_threads, "kind": "reference",
                "seconds_per_system": dt,
                "sample": f"one taucs_ccs_factor_llt_numeric + one taucs_supernodal_solve_llt of the same "
                          f"{grid}^3 system (reference sources + OpenBLAS 0.3.15, {n_threads} threads)",
                "max_abs_err": float(np.max(np.abs(x - xt)))}
    # fallback: the plain-C restatement on a smaller sample, scaled by flops
    import taucs_b200 as tb
    P = Port()
    g = max(8, grid // 2)
    A = tb.mesh3d(g)
    perm, iperm = tb.order(A, "amd")
    Pm = A.permute(perm, iperm)
    h = P.analyze(*Pm.arrays()[:3])
    t0 = time.perf_counter()
    P.numeric(h, Pm.colptr, Pm.rowind, Pm.values)
    P.solve(h, Pm.matvec(np.ones(A.n)))
    dt = time.perf_counter() - t0
    flops_s = tb.factor_symbolic(Pm).info().flops
    Af = tb.mesh3d(grid)
    pf, ipf = tb.order(Af, "amd")
    flops_f = tb.factor_symbolic(Af.permute(pf, ipf)).info().flops
    P.free(h)
    dt_full = dt * flops_f / flops_s
    return {"value": 1.0 / dt_full, "unit": UNIT, "cores": 1, "kind": "port", "seconds_per_system": dt_full,
            "sample": f"oracle restatement on {g}^3, time scaled by the flop ratio to {grid}^3"}


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return
    n_threads = os.cpu_count() or 1
    os.environ["OPENBLAS_NUM_THREADS"] = str(n_threads)
    from oracle.bindings import Port, Ref, ref_available
    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libtaucs_ref.so was not built"}))
        return
    R = Ref(threads=n_threads)
    R.set_threads(n_threads)
    g = args.grid
    n, cp, ri, va = R.mesh3d(g, g, g)
    perm, iperm = R.order(n, cp, ri, va, "amd")
    _, pc, pr, pv = R.permute(n, cp, ri, va, perm, iperm)
    L = R.symbolic(n, pc, pr, pv)
    xt = np.random.default_rng(0).uniform(-1, 1, n)
    b = Port().spmv(n, pc, pr, pv, xt)
    sym = R.dump_symbolic(L)
    # each step is one full system: about 15-25 s of CPU work at 64^3, so the
    # run is bounded to 1 warm-up step and at most 3 timed steps
    warm = min(args.warmup, 1)
    steps = max(1, min(args.steps, 3))
    x = None
    for _ in range(warm):
        R.numeric(L, n, pc, pr, pv)
        x = R.solve(L, b)
        R.free_numeric(L)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        assert R.numeric(L, n, pc, pr, pv) == 0
        x = R.solve(L, b)
        times.append(time.perf_counter() - t0)
        R.free_numeric(L)
    R.free(L)
    tot = sum(times)
    val = steps / tot
    out = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world,
           "steps": steps, "warmup": warm, "ms_per_step": 1e3 * tot / steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": f"mesh3d {g}^3 7-point Laplacian (reference generator), AMD, "
                                  f"numeric factor + 1-RHS solve", "n": n, "nnz_lower": int(cp[-1]),
                      "flops": sym.flops()},
           "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "cpu_baseline": {"value": val, "unit": UNIT, "cores": n_threads, "kind": "reference",
                            "sample": f"{steps} timed steps of the full {g}^3 system after {warm} warm-up "
                                      f"(reference sources + OpenBLAS 0.3.15, {n_threads} threads)"},
           "max_abs_err": float(np.max(np.abs(x - xt)))}
    print(json.dumps(out))


def run_ours(args):
    import torch
    import taucs_b200 as tb

    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    stream = torch.cuda.current_stream()
    tb.set_stream(stream.cuda_stream)
    g = args.grid

    # ---- setup (untimed): generator, AMD, permutation, symbolic analysis
    A = tb.mesh3d(g)
    perm, iperm = tb.order(A, "amd")
    P = A.permute(perm, iperm)
    F = tb.factor_symbolic(P)
    info = F.info()
    n, nnz = A.n, P.nnz
    xt = np.random.default_rng(0).uniform(-1, 1, n)
    b = P.matvec(xt)
    d_vals = torch.from_numpy(P.values).cuda()
    d_b = torch.from_numpy(b).cuda()
    d_x = torch.empty_like(d_b)
    # pinned host buffers for the end-to-end path
    h_vals = torch.empty(nnz, dtype=torch.float64, pin_memory=True).numpy()
    h_vals[:] = P.values
    Ph = tb.Matrix(n, P.colptr, P.rowind, h_vals)
    h_b = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    h_b[:] = b
    h_x = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()

    def step_device():
        if tb.lib().taucs_b200_factor_numeric_device_async(F.h, d_vals.data_ptr()) != 0:
            raise RuntimeError("numeric launch failed: " + tb.last_error())
        if F.solve_device(1, d_x.data_ptr(), d_b.data_ptr(), n) != 0:
            raise RuntimeError("solve launch failed: " + tb.last_error())

    def step_e2e():
        if F.numeric(Ph) != 0:
            raise RuntimeError("numeric failed: " + tb.last_error())
        if tb.lib().taucs_supernodal_solve_llt(F.h, h_x, h_b) != 0:
            raise RuntimeError("solve failed: " + tb.last_error())

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident timing
    for _ in range(max(args.warmup, 3)):
        step_device()
    assert tb.lib().taucs_b200_factor_status(F.h) == 0, tb.last_error()
    clocks = ClockSampler(local_rank)
    barrier()
    clocks.start()
    tb.launch_count(reset=True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step_device()
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    launches = tb.launch_count(reset=True) // max(args.steps, 1)
    ms = max_over_ranks(e0.elapsed_time(e1))
    ok = tb.lib().taucs_b200_factor_status(F.h) == 0
    x_dev = d_x.cpu().numpy()
    res_dev = scaled_residual(P, x_dev, b)

    # ---- end-to-end through the C ABI with pinned host buffers
    for _ in range(2):
        step_e2e()
    barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        step_e2e()
    f1.record(stream)
    barrier()
    ms_e2e = max_over_ranks(f0.elapsed_time(f1))
    res_e2e = scaled_residual(P, h_x, b)

    # ---- roofline: CUDA events around every launch, separate profiled steps
    tb.lib().taucs_b200_profile(1)
    nprof = max(2, min(args.steps, 5))
    for _ in range(nprof):
        step_device()
    torch.cuda.synchronize()
    import ctypes as C
    kern = {}
    rd = tb.lib().taucs_b200_profile_read
    for name, kc in KC.items():
        t, nl, fl, by = C.c_double(), C.c_long(), C.c_double(), C.c_double()
        rd(kc, C.byref(t), C.byref(nl), C.byref(fl), C.byref(by))
        if nl.value:
            kern[name] = {"ms_per_step": t.value / nprof, "launches_per_step": nl.value // nprof,
                          "gflop_per_step": fl.value / nprof / 1e9, "gb_per_step": by.value / nprof / 1e9}
    tb.lib().taucs_b200_profile(0)

    peaks = measured_peaks()
    fp64_peak = fp64_gemm_peak()
    hbm_peak = peaks.get("hbm_gbs")
    dom = max(kern.items(), key=lambda kv: kv[1]["ms_per_step"])[0] if kern else None
    roof = None
    if dom:
        d = kern[dom]
        per_launch_ms = d["ms_per_step"] / max(d["launches_per_step"], 1)
        if dom in TENSOR_KC:
            ach = d["gflop_per_step"] / d["ms_per_step"]  # GFLOP/ms = TFLOP/s
            roof = {"kernel": dom, "bound": "tensor", "achieved": ach, "peak": fp64_peak, "unit": "TFLOP/s",
                    "frac": ach / fp64_peak,
                    "peak_source": "FP64: cuBLAS DGEMM 8192^3 measured in this run (of measured)",
                    "algorithmic_per_launch": d["gflop_per_step"] / max(d["launches_per_step"], 1) * 1e9,
                    "avg_launch_ms": per_launch_ms, "traffic": None}
        else:
            ach = d["gb_per_step"] / d["ms_per_step"] * 1e3
            roof = {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s",
                    "frac": ach / hbm_peak if hbm_peak else None,
                    "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                    "algorithmic_per_launch": d["gb_per_step"] / max(d["launches_per_step"], 1) * 1e9,
                    "avg_launch_ms": per_launch_ms, "traffic": None}
    for v in kern.values():
        if v["gflop_per_step"] > 0:
            v["tflop_s"] = v["gflop_per_step"] / v["ms_per_step"]
        if v["gb_per_step"] > 0:
            v["gb_s"] = v["gb_per_step"] / v["ms_per_step"] * 1e3

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(g, os.cpu_count() or 1)
        except Exception as exc:  # report, never hide
            cpu = {"error": repr(exc)}

    steps = args.steps
    out = {
        "metric": METRIC, "value": world * steps / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
        "steps": steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"mesh3d {g}^3 7-point Laplacian (reference generator), AMD, "
                               f"FP64 numeric factor + 1-RHS solve", "n": n, "nnz_lower": nnz,
                   "flops": info.flops, "supernodes": info.n_live, "levels": info.n_levels,
                   "max_front": info.max_front, "l_gb": info.l_bytes / 1e9, "u_arena_gb": info.u_bytes / 1e9,
                   "l2_policy": "inputs larger than L2 (L and update arena > 4 GB touched per step)",
                   "parallelism": f"replicas x{world}"},
        "clocks": clk,
        "e2e": {"value": world * steps / (ms_e2e * 1e-3), "unit": UNIT, "ms_per_step": ms_e2e / steps,
                "h2d_bytes_per_step": 8 * nnz + 8 * n, "d2h_bytes_per_step": 8 * n + 4},
        "gpu_launches": int(launches),
        "roofline": roof,
        "kernels": kern,
        "cpu_baseline": cpu,
        "factor_tflop_s": info.flops / (ms / steps * 1e-3) / 1e12,
        "scaled_residual": {"device": res_dev, "e2e": res_e2e},
        "status_ok": bool(ok),
    }
    if rank == 0:
        print(json.dumps(out))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    F.free()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
