#!/usr/bin/env python
"""Benchmark of the multifrontal Cholesky factor + solve path.

Default workload (--workload mixed80): the precision configuration -- a 3D
7-point operator on an 80^3 grid (n = 512,000) whose edge conductances are
exp(2 N(0,1)) times an anisotropy of 1:1:100 in x:y:z (seeded generator,
taucs_b200_generate_lognormal), AMD ordering, 8 right-hand sides ~ U(-1,1)
(seed 0).  One STEP factors the analysed pattern with FP32 fronts (diagonal
scaling, tcgen05 FP16x3 products; --split-format 0 for TF32x3) and refines all 8 solutions in FP64 to a
scaled residual ||Ax-b||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= 1e-12 --
the FP32+refinement form.  The plain FP64 path (FP64 fronts, one solve of the
8 right-hand sides) is timed beside it on the same inputs and reported as
`fp64` with the speed-up.  Ordering and symbolic analysis happen once, before
the timed region, as in the reference's pattern-reuse path
(src/taucs_linsolve.c:433-453; numeric = src/taucs_sn_llt.c:2169-2209, solve
= :2844-2885).

--workload fp64-64: the 64^3 7-point Laplacian of the reference's
taucs_ccs_generate_mesh3d, AMD, FP64 numeric factor + one 1-RHS solve.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line (rank 0).  `value` is whole-job systems/s with values
and right-hand sides resident in device memory; `e2e` is the same metric
through the C ABI with pinned host buffers (values, B in; X out) copied
inside every step.  Under torchrun every rank factors its own replica (no
collective on the data path; max over ranks for time).
"""
import argparse
import ctypes as C
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

UNIT = "systems/s"
METRIC_MIXED = ("FP32+refine vs FP64 factor+solve time at 1e-12 residual "
                "(80^3 lognormal sigma=2, aniso 1:1:100, AMD, 8 RHS): FP32+refine systems/s")
METRIC_FP64 = "fp64 numeric factor + solve throughput (64^3 7-point Laplacian, AMD)"
NRHS = 8
TOL = 1e-12
SAMPLE_GRID = 56          # bounded CPU sample of the lognormal workload

KC = dict(small_front=0, build=1, leaf=2, dinv=3, gemm_panel=4, gemm_u=5, solve_fwd=6, solve_bwd=7)
# kernel classes whose roofline is the tensor pipe; the others (the panel
# leaves among them: a latency-bound chain) are held against HBM
TENSOR_KC = {"gemm_panel", "gemm_u"}
# DRAM traffic per algorithmic byte of a kernel class, from one ncu capture
# of a 56^3 update-matrix launch (FP32 fronts, FP16x3 products, the largest
# update product of the 56^3 factorization: one front, 630 tiles): dram read
# + write 101.1 + 11.0 MB against 129.9 MB of L21 read once and U read and
# written once; the bench scales it to its own per-launch algorithmic bytes
TRAFFIC_PER_ALG_BYTE = {"gemm_u": (112.1 / 129.9, "ncu dram__bytes_read.sum + dram__bytes_write.sum of one 56^3 "
                                                  "update-matrix launch (python -m taucs_b200.profile_case "
                                                  "update-gemm 56), scaled by algorithmic bytes (L21 read once, "
                                                  "U read and written once) to this launch size")}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mixed80", choices=["mixed80", "fp64-64", "batch4096"])
    ap.add_argument("--batch-count", type=int, default=BATCH_COUNT)
    ap.add_argument("--grid", type=int, default=None, help="grid side (default 80 / 64 per workload)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="duration of the Poisson request stream at 2000 req/s (the configuration's 60 s)")
    ap.add_argument("--split-format", type=int, default=1, choices=[0, 1],
                    help="operand format of the FP32 fronts' tensor-core products: 0 TF32x3, 1 FP16x3")
    ap.add_argument("--refinement", type=int, default=0, choices=[0, 1],
                    help="0 refinement steps (PCG on stall), 1 PCG on the FP32 factor from the first step")
    ap.add_argument("--no-extra-legs", action="store_true",
                    help="skip the fp64-64 and batch4096 legs that the default run reports beside its line")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def scaled_residual(A, x, b):
    r = A.matvec(x) - b
    return float(np.max(np.abs(r)) / (A.inf_norm() * np.max(np.abs(x)) + np.max(np.abs(b))))


def max_over_ranks_of(dist, v, device):
    """The slowest rank's value (timings are reported as the max over ranks);
    dist is torch.distributed or None for one process."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_system(workload, g):
    """(A unpermuted, perm, iperm, PAP^T, B) of the workload."""
    import taucs_b200 as tb
    if workload == "mixed80":
        A = tb.lognormal(g, g, g, 2.0, (1.0, 1.0, 100.0), 0)
        nrhs = NRHS
    else:
        A = tb.mesh3d(g)
        nrhs = 1
    perm, iperm = tb.order(A, "amd")
    P = A.permute(perm, iperm)
    rng = np.random.default_rng(0)
    if workload == "mixed80":
        B = rng.uniform(-1, 1, (A.n, nrhs))
    else:
        B = P.matvec(rng.uniform(-1, 1, A.n)).reshape(-1, 1)
    return A, perm, iperm, P, B


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


def tf32_gemm_peak():
    """cuBLAS TF32 GEMM (FP32 inputs on the tensor cores) 8192^3, best of 5."""
    import torch
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = True
    n = 8192
    a = torch.randn(n, n, device="cuda", dtype=torch.float32)
    b = torch.randn(n, n, device="cuda", dtype=torch.float32)
    best = 0.0
    for _ in range(6):
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        a @ b
        e.record()
        torch.cuda.synchronize()
        best = max(best, 2.0 * n ** 3 / (s.elapsed_time(e) * 1e-3) / 1e12)
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    torch.cuda.empty_cache()
    return best


# ---------------------------------------------------------------- CPU (reference)

def ref_inputs(workload, g):
    """The workload's P A P^T for the reference library, built without the
    product library: the oracle's independent statement of the lognormal
    generator (bit-identical to the product's, tests/test_oracle.py) or the
    reference's own mesh3d, then the reference's AMD ordering and symmetric
    permutation.  Returns (Ref, n, colptr, rowind, values, B)."""
    from oracle.bindings import Port, Ref, ref_available
    if not ref_available():
        raise RuntimeError("oracle/_ref/libtaucs_ref.so was not built")
    R, port = Ref(), Port()
    if workload == "mixed80":
        n, cp, ri, va = port.lognormal(g, g, g, 2.0, (1.0, 1.0, 100.0), 0)
    else:
        n, cp, ri, va = R.mesh3d(g, g, g)
    perm, iperm = R.order(n, cp, ri, va, "amd")
    _, pc, pr, pv = R.permute(n, cp, ri, va, perm, iperm)
    rng = np.random.default_rng(0)
    if workload == "mixed80":
        B = rng.uniform(-1, 1, (n, NRHS))
    else:
        B = port.spmv(n, pc, pr, pv, rng.uniform(-1, 1, n)).reshape(-1, 1)
    return R, port, n, pc, pr, pv, B


def ref_steps(R, L, n, pc, pr, pv, B, steps, threads):
    """`steps` runs of the reference's pattern-reuse path (numeric factor on
    the analysed pattern, src/taucs_sn_llt.c:2169-2209, then one
    taucs_supernodal_solve_llt per right-hand side, :2844-2885) with
    `threads` OpenBLAS threads.  Returns (factor s, solve s) per step and the
    last step's X."""
    R.set_threads(threads)
    tf, ts, X = [], [], None
    for _ in range(steps):
        t0 = time.perf_counter()
        if R.numeric(L, n, pc, pr, pv) != 0:
            raise RuntimeError("reference numeric factorization failed")
        t1 = time.perf_counter()
        X = np.empty_like(B)
        for q in range(B.shape[1]):       # the reference solves one right-hand side per call
            X[:, q] = R.solve(L, np.ascontiguousarray(B[:, q]))
        ts.append(time.perf_counter() - t1)
        tf.append(t1 - t0)
        R.free_numeric(L)
    return tf, ts, X


def lower_inf_norm(n, cp, ri, va):
    """||A||_inf of the symmetric matrix stored as its lower triangle."""
    col = np.repeat(np.arange(n), np.diff(cp))
    a = np.abs(va)
    rs = np.zeros(n)
    np.add.at(rs, ri, a)
    np.add.at(rs, col[ri != col], a[ri != col])
    return float(rs.max())


def x_checksum(X):
    """Per-column sums and max-abs of a solution block (compared across arms)."""
    return {"sum": [float(v) for v in X.sum(axis=0)], "max_abs": [float(v) for v in np.abs(X).max(axis=0)]}


def cpu_baseline_sample(workload, g_full, flops_full, threads_list, g_sample=SAMPLE_GRID):
    """The bounded CPU-baseline leg of this arm: the reference (sources +
    OpenBLAS 0.3.15) on a smaller grid of the same generator, one factor + all
    solves per thread count, its time scaled by the reference's flop count to
    the full grid.  Returns the cpu_baseline object."""
    if workload != "mixed80":
        g_sample = g_full
    R, _, n, pc, pr, pv, B = ref_inputs(workload, g_sample)
    L = R.symbolic(n, pc, pr, pv)
    fl = R.dump_symbolic(L).flops()
    scale = flops_full / fl if workload == "mixed80" else 1.0
    out = {}
    for th in threads_list:
        tf, ts, _ = ref_steps(R, L, n, pc, pr, pv, B, 1, th)
        out[th] = (tf[0] + ts[0]) * scale, tf[0] + ts[0]
    R.free(L)
    th0 = threads_list[0]
    what = (f"reference FP64 numeric factor + {B.shape[1]} one-RHS solves of the {g_sample}^3 system of the same "
            f"generator (sigma=2, aniso 1:1:100, AMD)") if workload == "mixed80" else \
        f"reference FP64 numeric factor + 1-RHS solve of the full {g_full}^3 system"
    res = {"value": 1.0 / out[th0][0], "unit": UNIT, "cores": th0, "kind": "reference",
           "sample": what + (f", scaled by the reference's flop count x{scale:.2f} to {g_full}^3" if scale != 1.0
                             else "") + "; sources + OpenBLAS 0.3.15",
           "per_thread_count": {str(th): {"systems_per_s": 1.0 / v[0], "sample_s": v[1]} for th, v in out.items()}}
    return res


def run_reference(args):
    """The reference's own CPU multifrontal path on the FULL workload (no
    sampling, no scaling), in a process that loads only the oracle libraries
    (oracle/_ref): numeric factor + solves of the same seeded system, timed at
    all host threads; one more step at one OpenBLAS thread is reported beside
    it.  Each step takes about a minute on the box, so at most two timed
    steps run (no warm-up: nothing is compiled or cached between steps; the
    reference allocates its fronts afresh every time)."""
    rank, _, world = dist_env()
    if rank != 0:
        return
    if args.workload == "batch4096":
        return run_reference_batch(args, world)
    g = args.grid or (80 if args.workload == "mixed80" else 64)
    nproc = os.cpu_count() or 1
    try:
        t_setup = time.perf_counter()
        R, port, n, pc, pr, pv, B = ref_inputs(args.workload, g)
        L = R.symbolic(n, pc, pr, pv)
        sym = R.dump_symbolic(L)
        flops = sym.flops()
        t_setup = time.perf_counter() - t_setup
        steps = max(1, min(args.steps, 2))
        tf, ts, X = ref_steps(R, L, n, pc, pr, pv, B, steps, nproc)
        tf1, ts1, _ = ref_steps(R, L, n, pc, pr, pv, B, 1, 1)
        R.free(L)
    except Exception as exc:  # one line, never a traceback
        print(json.dumps({"impl": "reference", "unavailable": repr(exc)}))
        return
    anorm = lower_inf_norm(n, pc, pr, pv)
    res = max(float(np.max(np.abs(port.spmv(n, pc, pr, pv, X[:, q]) - B[:, q])) /
                    (anorm * np.max(np.abs(X[:, q])) + np.max(np.abs(B[:, q])))) for q in range(B.shape[1]))
    sec = (sum(tf) + sum(ts)) / steps
    sec1 = tf1[0] + ts1[0]
    val = 1.0 / sec
    metric = METRIC_MIXED if args.workload == "mixed80" else METRIC_FP64
    desc = (f"reference FP64 numeric factor + {B.shape[1]} one-RHS solves of the full {g}^3 system "
            f"({steps} timed steps at {nproc} threads); sources + OpenBLAS 0.3.15")
    out = {"impl": "reference", "metric": metric, "value": val, "unit": UNIT, "n_gpus": world,
           "steps": steps, "warmup": 0, "ms_per_step": 1e3 * sec, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": workload_config(args.workload, g, n, len(pv), B.shape[1]),
           "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "cpu_baseline": {"value": val, "unit": UNIT, "cores": nproc, "kind": "reference", "sample": desc},
           "steps_note": (f"{args.steps} steps requested; each full step takes about a minute of CPU time, so "
                          f"{steps} are timed"),
           "factor_s": sum(tf) / steps, "solve_s": sum(ts) / steps, "setup_s": t_setup,
           "factor_gflop_s": flops / (sum(tf) / steps) / 1e9, "flops": flops,
           "supernodes": int(np.count_nonzero(sym.sn_size)),
           "one_thread": {"value": 1.0 / sec1, "unit": UNIT, "factor_s": tf1[0], "solve_s": ts1[0],
                          "factor_gflop_s": flops / tf1[0] / 1e9},
           "scaled_residual": res, "x_checksum": x_checksum(X)}
    print(json.dumps(out))


def run_reference_batch(args, world):
    try:
        import taucs_b200 as tb
        systems, bs = batch_systems(tb, args.batch_count)
        flops = 0.0
        for A in systems:
            p, ip = tb.order(A, "amd")
            F = tb.factor_symbolic(A.permute(p, ip))
            flops += F.info().flops
            F.free()
        n_threads = os.cpu_count() or 1
        t_s, fl_s, ns = cpu_reference_batch(systems, bs, n_threads)
        sec = t_s * flops / fl_s
    except Exception as exc:
        print(json.dumps({"impl": "reference", "unavailable": repr(exc)}))
        return
    val = args.batch_count / sec
    desc = (f"reference FP64 factor + solve of {ns} evenly spaced systems of the batch one at a time "
            f"({t_s:.2f} s), scaled by the reference's flop count to all {args.batch_count} systems; "
            f"sources + OpenBLAS 0.3.15, {n_threads} threads")
    print(json.dumps({"impl": "reference", "metric": METRIC_BATCH, "value": val, "unit": UNIT, "n_gpus": world,
                      "steps": 1, "warmup": 0, "ms_per_step": 1e3 * sec, "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                      "config": {"workload": f"{args.batch_count} systems"},
                      "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                      "cpu_baseline": {"value": val, "unit": UNIT, "cores": n_threads, "kind": "reference",
                                       "sample": desc}}))


def workload_config(workload, g, n, nnz, nrhs):
    """The `config` object both arms print (it names the workload only)."""
    return {"workload": workload_name(workload, g), "n": int(n), "nnz_lower": int(nnz), "nrhs": int(nrhs)}


def workload_name(workload, g):
    if workload == "mixed80":
        return (f"lognormal {g}^3 7-point (sigma=2, aniso 1:1:100, seed 0), AMD, {NRHS} RHS; "
                f"numeric factor + solve to scaled residual <= {TOL:g}")
    return f"mesh3d {g}^3 7-point Laplacian (reference generator), AMD, FP64 numeric factor + 1-RHS solve"


# ---------------------------------------------------------------- serving

class ServeStream:
    """Seeded request stream of the serving configuration: Poisson arrivals;
    70% 2D 5-point lognormal grids with n ~ U[1000, 20000] (side = floor(sqrt n)),
    25% 3D 7-point grids with side ~ U{16..40}, 5% 3D 64^3; sigma = 1; of all
    requests 50% bring new coefficients on a pattern already seen, 20% new
    right-hand sides (1-32 columns) for a matrix already seen, the rest a
    freshly drawn size with new coefficients.  The 64^3 requests take their
    coefficients from 8 generated sets, each scaled by a distinct factor per
    request (a new SPD matrix every time, without 16 MB of generation per
    request).  Right-hand sides are views of one seeded U(-1,1) pool."""

    def __init__(self, tb, seed=0):
        self.tb = tb
        self.rng = np.random.default_rng(seed)
        self.base = {}          # pattern -> Matrix (colptr/rowind shared by all its requests)
        self.big_sets = []
        self.seen_pat, self.seen_mat = [], []
        self.pool = self.rng.uniform(-1, 1, 64 ** 3 * 32 + 1)

    def _pattern(self):
        v = self.rng.random()
        if v < 0.70:
            s = int(np.sqrt(self.rng.integers(1000, 20001)))
            return (s, s, 0)
        if v < 0.95:
            s = int(self.rng.integers(16, 41))
            return (s, s, s)
        return (64, 64, 64)

    def _new_matrix(self, pk):
        tb = self.tb
        if pk == (64, 64, 64):
            if not self.big_sets:
                self.big_sets = [tb.lognormal(64, 64, 64, 1.0, (1, 1, 1), 1000 + i) for i in range(8)]
            M = self.big_sets[int(self.rng.integers(8))]
            c = 1.0 + float(self.rng.random())
            return tb.Matrix(M.n, M.colptr, M.rowind, M.values * c)
        return tb.lognormal(pk[0], pk[1], pk[2], 1.0, (1, 1, 1), int(self.rng.integers(1 << 30)))

    def draw(self, n_req):
        out = []
        for _ in range(n_req):
            u = self.rng.random()
            nrhs = 1
            if u < 0.20 and self.seen_mat:
                A, pk = self.seen_mat[int(self.rng.integers(len(self.seen_mat)))]
                nrhs = int(self.rng.integers(1, 33))
            elif u < 0.70 and self.seen_pat:
                pk = self.seen_pat[int(self.rng.integers(len(self.seen_pat)))]
                A = self._new_matrix(pk)
            else:
                pk = self._pattern()
                if pk not in self.seen_pat:
                    self.seen_pat.append(pk)
                A = self._new_matrix(pk)
            self.seen_mat.append((A, pk))
            off = int(self.rng.integers(0, len(self.pool) - A.n * nrhs))
            B = self.pool[off:off + A.n * nrhs].reshape(nrhs, A.n).T     # column-major view
            out.append((A, B, pk))
        return out


def serve_stream(tb, S, reqs, rate, rng):
    """Submits reqs at Poisson arrival times (rate req/s) and waits for all;
    returns per-request results, the span first submit -> last completion,
    and the client's worst lag behind the arrival schedule."""
    gaps = rng.exponential(1.0 / rate, len(reqs))
    t_arr = np.cumsum(gaps)
    ids, lag = [], 0.0
    t0 = time.perf_counter()
    for (A, B, _), ta in zip(reqs, t_arr):
        now = time.perf_counter() - t0
        if ta > now:
            time.sleep(ta - now)
        else:
            lag = max(lag, now - ta)
        ids.append(S.submit(A, B, TOL))
    res = [S.wait(i) for i in ids]
    span = time.perf_counter() - t0
    return res, span, lag


def fp64_one_at_a_time(tb, reqs):
    """The same requests solved one after another through the FP64 C API
    (patterns analysed beforehand, as the server caches them): permute,
    factor, solve, un-permute per request.  Two untimed passes over the
    sample first, so that every factor replays its recorded launch sequences
    in the timed pass (the steady state of a long-running caller, as for the
    server)."""
    cache = {}
    for A, _, pk in reqs:
        if pk not in cache:
            p, ip = tb.order(A, "amd")
            F = tb.factor_symbolic(A.permute(p, ip))
            F.set_precision(0)
            cache[pk] = (p, ip, F)

    def one_pass():
        for A, B, pk in reqs:
            p, ip, F = cache[pk]
            if F.numeric(A.permute(p, ip)) != 0:
                raise RuntimeError("FP64 factor failed")
            X = np.empty_like(B)
            X[p, :] = F.solve(np.ascontiguousarray(B[p, :]))

    one_pass()
    one_pass()
    t0 = time.perf_counter()
    one_pass()
    dt = time.perf_counter() - t0
    for _, _, F in cache.values():
        F.free()
    return len(reqs) / dt


def run_serving(tb, seconds=2.0, rate=2000.0, sustain_rate=250.0, sustain_seconds=4.0, workers=16,
                budget=120e9, fp64_sample=200, warm_requests=1500):
    rng = np.random.default_rng(1)
    gen = ServeStream(tb, seed=0)
    n_main = int(seconds * rate)
    n_sus = int(sustain_seconds * sustain_rate)
    main = gen.draw(n_main)
    sus = gen.draw(n_sus)
    S = tb.Server(workers=workers, budget_bytes=budget)
    # warm-up, untimed: analyse every pattern of the streams once
    seen = {}
    for A, _, pk in main + sus + gen.draw(0):
        if pk not in seen:
            seen[pk] = A
    for A in seen.values():
        S.wait(S.submit(A, np.ones(A.n), TOL))
    # warm-up stream of the same mix, untimed: factor instances and recorded
    # launch sequences exist before the timed stream, as in a long-running
    # server
    warm = gen.draw(warm_requests)
    for i in [S.submit(A, B, TOL) for A, B, _ in warm]:
        S.wait(i)
    del warm
    st0 = S.stats()
    res, span, lag = serve_stream(tb, S, main, rate, rng)
    st1 = S.stats()
    res_s, span_s, lag_s = serve_stream(tb, S, sus, sustain_rate, rng)
    S.close()
    lat = np.array([r[2] for r in res]) * 1e3
    lat_s = np.array([r[2] for r in res_s]) * 1e3
    cols = sum(B.shape[1] for _, B, _ in main)
    fails = sum(1 for r in res + res_s if r[0] != 0)
    worst = max(r[4] for r in res + res_s)
    served = len(main) / span
    fp64 = fp64_one_at_a_time(tb, main[:fp64_sample])
    return {
        "workload": (f"Poisson {rate:g} req/s for {seconds:g} s ({n_main} requests): 70% 2D n in [1k,20k], "
                     f"25% 3D side 16-40, 5% 64^3, sigma=1; 50% new coefficients on a seen pattern, 20% new RHS "
                     f"(1-32) on a seen matrix; FP32 fronts + FP64 refinement to {TOL:g}"),
        "workers": workers, "budget_gb": budget / 1e9, "patterns": len(seen),
        "warm_up": f"{warm_requests} requests of the same mix, untimed, before the timed streams",
        "requests_per_s": served, "rhs_columns_per_s": cols / span,
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "note": "offered rate above capacity: latencies include queueing of the backlog",
        "client_max_lag_ms": lag * 1e3,
        "sustained": {"rate": sustain_rate, "requests": n_sus, "requests_per_s": n_sus / span_s,
                      "p50_ms": float(np.percentile(lat_s, 50)), "p99_ms": float(np.percentile(lat_s, 99)),
                      "client_max_lag_ms": lag_s * 1e3},
        "fp64_one_at_a_time_requests_per_s": fp64, "speedup_vs_fp64_one_at_a_time": served / fp64,
        "factorizations": st1["factorizations"] - st0["factorizations"],
        "resident_solves": st1["resident_solves"] - st0["resident_solves"],
        "evictions": st1["evictions"], "failed": fails, "worst_scaled_residual": worst,
    }



# ---------------------------------------------------------------- batches

BATCH_COUNT = 4096
METRIC_BATCH = ("batch of 4096 SPD systems (2048 2D 5-point side 8-96, 2048 3D 7-point side 4-24, lognormal "
                "sigma=1, 1 RHS each): FP32+refine factor+solve systems/s")


def batch_systems(tb, count=BATCH_COUNT, seed=0):
    """The batch configuration: half 2D 5-point grids with side ~ U{8..96},
    half 3D 7-point grids with side ~ U{4..24}; lognormal(0, 1) edge
    conductances (system i uses generator seed i); b_i ~ U(-1, 1)."""
    rng = np.random.default_rng(seed)
    systems, bs = [], []
    for i in range(count):
        if i < count // 2:
            s = int(rng.integers(8, 97))
            A = tb.lognormal(s, s, 0, 1.0, (1, 1, 1), i)
        else:
            s = int(rng.integers(4, 25))
            A = tb.lognormal(s, s, s, 1.0, (1, 1, 1), i)
        systems.append(A)
    for A in systems:
        bs.append(rng.uniform(-1, 1, A.n))
    return systems, bs


def cpu_reference_batch(systems, bs, n_threads, sample=96):
    """The reference's CPU multifrontal path, one system at a time (its only
    mode), on an evenly spaced sample of the batch; scaled to the batch by
    the flop ratio."""
    import taucs_b200 as tb
    from oracle.bindings import Ref, ref_available
    os.environ["OPENBLAS_NUM_THREADS"] = str(n_threads)
    if not ref_available():
        raise RuntimeError("oracle/_ref/libtaucs_ref.so was not built")
    R = Ref(threads=n_threads)
    R.set_threads(n_threads)
    idx = np.linspace(0, len(systems) - 1, sample).astype(int)
    t_tot, fl_s = 0.0, 0.0
    for i in idx:
        A = systems[i]
        perm, iperm = R.order(A.n, A.colptr, A.rowind, A.values, "amd")
        _, pc, pr, pv = R.permute(A.n, A.colptr, A.rowind, A.values, perm, iperm)
        L = R.symbolic(A.n, pc, pr, pv)
        fl_s += R.dump_symbolic(L).flops()
        b = np.ascontiguousarray(bs[i][np.asarray(perm)])
        t0 = time.perf_counter()
        assert R.numeric(L, A.n, pc, pr, pv) == 0
        R.solve(L, b)
        t_tot += time.perf_counter() - t0
        R.free(L)
    return t_tot, fl_s, len(idx)


def run_batch(args):
    import torch
    import taucs_b200 as tb
    rank, local_rank, world = dist_env()
    torch.cuda.set_device(local_rank)
    stream = torch.cuda.current_stream()
    tb.set_stream(stream.cuda_stream)
    lib = tb.lib()
    count = args.batch_count
    t0 = time.perf_counter()
    systems, bs = batch_systems(tb, count)
    B = tb.Batch(systems)
    t_setup = time.perf_counter() - t0
    info = B.info()
    n = B.n
    d_vals = torch.from_numpy(B.combined_values()).cuda()
    d_b = torch.from_numpy(B.combined_rhs(bs)).cuda()
    d_x = torch.empty_like(d_b)
    res = np.empty(count, np.float64)

    def step_mixed():
        B.set_precision(1)
        if lib.taucs_b200_factor_numeric_device(B.h, d_vals.data_ptr()) != 0:
            raise RuntimeError("batch numeric failed: " + tb.last_error())
        its = lib.taucs_b200_solve_refine_device(B.h, 1, C.c_void_p(d_x.data_ptr()), C.c_void_p(d_b.data_ptr()),
                                                  n, TOL, 10, res)
        if its < 0:
            raise RuntimeError("batch refinement failed: " + tb.last_error())
        return its

    def step_fp64():
        B.set_precision(0)
        if lib.taucs_b200_factor_numeric_device_async(B.h, d_vals.data_ptr()) != 0:
            raise RuntimeError("batch numeric failed: " + tb.last_error())
        if B.solve_device(1, d_x.data_ptr(), d_b.data_ptr(), n) != 0:
            raise RuntimeError("batch solve failed: " + tb.last_error())

    def timed(step, k):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = None
        for _ in range(k):
            out = step()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    def worst_residual():
        torch.cuda.synchronize()
        xs = B.split(d_x.cpu().numpy())
        return max(scaled_residual(A, x, b) for A, x, b in zip(systems, xs, bs))

    W, K = max(args.warmup, 3), args.steps
    for _ in range(W):
        step_mixed()
    clocks = ClockSampler(local_rank)
    clocks.start()
    tb.launch_count(reset=True)
    ms, its = timed(step_mixed, K)
    clk = clocks.stop()
    launches = tb.launch_count(reset=True) // max(K, 1)
    res_mixed = worst_residual()
    worst_reported = float(res.max())
    for _ in range(W):
        step_fp64()
    ms64, _ = timed(step_fp64, K)
    res64 = worst_residual()

    # end to end through the C ABI: host values and right-hand sides per system
    bptr = (C.c_void_p * count)(*[b.ctypes.data for b in bs])
    xs_h = [np.empty(A.n) for A in systems]
    xptr = (C.c_void_p * count)(*[x.ctypes.data for x in xs_h])
    sptr = (C.POINTER(tb.CCSStruct) * count)(*[C.pointer(A.s) for A in systems])

    def step_e2e():
        B.set_precision(1)
        if lib.taucs_b200_batch_factor(B.h, sptr) != 0:
            raise RuntimeError("batch factor failed: " + tb.last_error())
        if lib.taucs_b200_batch_solve(B.h, xptr, bptr, TOL, 10, res) < 0:
            raise RuntimeError("batch solve failed: " + tb.last_error())
    step_e2e()
    t0 = time.perf_counter()
    for _ in range(K):
        step_e2e()
    ms_e2e = (time.perf_counter() - t0) * 1e3

    # profiled steps for the roofline
    lib.taucs_b200_profile(1)
    nprof = 2
    for _ in range(nprof):
        step_mixed()
    torch.cuda.synchronize()
    kern = read_profile(tb, nprof)
    lib.taucs_b200_profile(0)
    tf32 = tf32_gemm_peak()
    roof = roofline(kern, tf32 / 3.0, f"cuBLAS TF32 GEMM 8192^3 measured in this run ({tf32:.0f} TF/s) / 3 "
                                      f"(TF32x3 products, of measured)", measured_peaks().get("hbm_gbs"))
    B.free()
    torch.cuda.empty_cache()

    # the same systems one at a time on the GPU (FP64, patterns analysed
    # beforehand), on an evenly spaced sample
    idx = np.linspace(0, count - 1, 128).astype(int)
    pre = []
    for i in idx:
        A = systems[i]
        p, ip = tb.order(A, "amd")
        P = A.permute(p, ip)
        F = tb.factor_symbolic(P)
        F.set_precision(0)
        pre.append((F, P, np.ascontiguousarray(bs[i][p])))
    # (every system once untimed: its first call also uploads its plan)
    for F, P, b in pre:
        F.numeric(P)
        F.solve(b)
    t0 = time.perf_counter()
    for F, P, b in pre:
        F.numeric(P)
        F.solve(b)
    t_one = (time.perf_counter() - t0) / len(pre)
    for F, _, _ in pre:
        F.free()

    cpu = None
    if not args.no_cpu_baseline:
        try:
            nth = os.cpu_count() or 1
            t_s, fl_s, ns = cpu_reference_batch(systems, bs, nth)
            sec = t_s * info.flops / fl_s
            cpu = {"value": count / sec, "unit": UNIT, "cores": nth, "kind": "reference",
                   "sample": f"reference FP64 factor + solve of {ns} evenly spaced systems of the batch one at a "
                             f"time ({t_s:.2f} s), scaled by the reference's flop count to all {count} systems; "
                             f"sources + OpenBLAS 0.3.15, {nth} threads"}
        except Exception as exc:
            cpu = {"error": repr(exc)}
    out = {
        "metric": METRIC_BATCH, "value": K * count / (ms * 1e-3), "unit": UNIT, "n_gpus": 1, "steps": K,
        "warmup": W, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64", "data": "synthetic",
        "config": {"workload": f"{count} systems, one block-diagonal level-scheduled factor + solve per step",
                   "rows": n, "nnz_lower": B.nnz, "flops": info.flops, "supernodes": info.n_live,
                   "levels": info.n_levels, "l_gb_fp64": info.l_bytes / 1e9, "setup_s": t_setup,
                   "l2_policy": "inputs larger than L2 (tens of GB of factor and update arena per step)"},
        "clocks": clk,
        "e2e": {"value": K * count / (ms_e2e * 1e-3), "unit": UNIT, "ms_per_step": ms_e2e / K,
                "h2d_bytes_per_step": 8 * B.nnz + 8 * n, "d2h_bytes_per_step": 8 * n + 8 * count},
        "gpu_launches": int(launches),
        "roofline": roof,
        "kernels": kern,
        "cpu_baseline": cpu,
        "refinement_steps": its,
        "scaled_residual": {"worst_system": res_mixed, "worst_reported_by_refinement": worst_reported},
        "fp64": {"value": K * count / (ms64 * 1e-3), "unit": UNIT, "ms_per_step": ms64 / K,
                 "worst_system_scaled_residual": res64},
        "one_at_a_time_fp64_gpu": {"value": 1.0 / t_one, "unit": UNIT,
                                   "sample": "128 evenly spaced systems, FP64 factor + solve each from host "
                                             "arrays, patterns analysed and every system run once beforehand"},
    }
    return out



# ---------------------------------------------------------------- GPU

def read_profile(tb, nsteps):
    kern = {}
    rd = tb.lib().taucs_b200_profile_read
    for name, kc in KC.items():
        t, nl, fl, by = C.c_double(), C.c_long(), C.c_double(), C.c_double()
        rd(kc, C.byref(t), C.byref(nl), C.byref(fl), C.byref(by))
        if nl.value:
            kern[name] = {"ms_per_step": t.value / nsteps, "launches_per_step": nl.value // nsteps,
                          "gflop_per_step": fl.value / nsteps / 1e9, "gb_per_step": by.value / nsteps / 1e9}
    for v in kern.values():
        if v["gflop_per_step"] > 0:
            v["tflop_s"] = v["gflop_per_step"] / v["ms_per_step"]
        if v["gb_per_step"] > 0:
            v["gb_s"] = v["gb_per_step"] / v["ms_per_step"] * 1e3
    return kern


def roofline(kern, tensor_peak, tensor_src, hbm_peak, traffic_table=None, dom=None):
    """The roofline of kernel class dom (default: the dominant one by time).
    traffic_table (kernel class -> (DRAM bytes per algorithmic byte, source))
    is passed only for the run whose kernel and sizes the ncu capture matches
    (FP32 fronts at 80^3)."""
    if not kern:
        return None
    if dom is None:
        dom = max(kern.items(), key=lambda kv: kv[1]["ms_per_step"])[0]
    if dom not in kern:
        return None
    d = kern[dom]
    per_launch_ms = d["ms_per_step"] / max(d["launches_per_step"], 1)
    bytes_per_launch = d.get("gb_per_step", 0.0) / max(d["launches_per_step"], 1) * 1e9
    traffic, traffic_src = None, None
    if traffic_table and dom in traffic_table and bytes_per_launch > 0:
        ratio, traffic_src = traffic_table[dom]
        traffic = ratio * bytes_per_launch
    if dom in TENSOR_KC:
        ach = d["gflop_per_step"] / d["ms_per_step"]  # GFLOP/ms = TFLOP/s
        out = {"kernel": dom, "bound": "tensor", "achieved": ach, "peak": tensor_peak, "unit": "TFLOP/s",
               "frac": ach / tensor_peak, "peak_source": tensor_src,
               "algorithmic_per_launch": d["gflop_per_step"] / max(d["launches_per_step"], 1) * 1e9,
               "avg_launch_ms": per_launch_ms, "traffic": traffic,
               "algorithmic_bytes_per_launch": bytes_per_launch}
        if traffic_src:
            out["traffic_source"] = traffic_src
        return out
    ach = d["gb_per_step"] / d["ms_per_step"] * 1e3
    return {"kernel": dom, "bound": "hbm", "achieved": ach, "peak": hbm_peak, "unit": "GB/s",
            "frac": ach / hbm_peak if hbm_peak else None,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
            "algorithmic_per_launch": d["gb_per_step"] / max(d["launches_per_step"], 1) * 1e9,
            "avg_launch_ms": per_launch_ms, "traffic": None}


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
    mixed = args.workload == "mixed80"
    g = args.grid or (80 if mixed else 64)

    # ---- setup (untimed): generator, AMD, permutation, symbolic analysis
    A, perm, iperm, P, B = make_system(args.workload, g)
    F = tb.factor_symbolic(P)
    tb.lib().taucs_b200_set_split_format(F.h, args.split_format)
    tb.lib().taucs_b200_set_refinement(F.h, args.refinement)
    info = F.info()
    n, nnz, nrhs = A.n, P.nnz, B.shape[1]
    Bf = np.asfortranarray(B)
    d_vals = torch.from_numpy(P.values).cuda()
    d_b = torch.from_numpy(Bf.T.copy()).cuda()        # column-major n x nrhs
    d_x = torch.empty_like(d_b)
    # pinned host buffers for the end-to-end path
    h_vals = torch.empty(nnz, dtype=torch.float64, pin_memory=True).numpy()
    h_vals[:] = P.values
    Ph = tb.Matrix(n, P.colptr, P.rowind, h_vals)
    h_b = torch.empty(nrhs * n, dtype=torch.float64, pin_memory=True).numpy()
    h_b[:] = Bf.T.reshape(-1)
    h_x = torch.empty(nrhs * n, dtype=torch.float64, pin_memory=True).numpy()
    res_buf = np.empty(nrhs, np.float64)
    lib = tb.lib()

    def numeric_device(prec):
        F.set_precision(prec)
        if lib.taucs_b200_factor_numeric_device(F.h, d_vals.data_ptr()) != 0:
            raise RuntimeError("numeric failed: " + tb.last_error())

    def step_mixed():
        numeric_device(1)
        its = lib.taucs_b200_solve_refine_device(F.h, nrhs, C.c_void_p(d_x.data_ptr()), C.c_void_p(d_b.data_ptr()),
                                                  n, TOL, 10, res_buf)
        if its < 0:
            raise RuntimeError("refinement did not reach the target: " + tb.last_error())
        return its

    def step_fp64():
        F.set_precision(0)
        if lib.taucs_b200_factor_numeric_device_async(F.h, d_vals.data_ptr()) != 0:
            raise RuntimeError("numeric launch failed: " + tb.last_error())
        if F.solve_device(nrhs, d_x.data_ptr(), d_b.data_ptr(), n) != 0:
            raise RuntimeError("solve launch failed: " + tb.last_error())

    def step_e2e_mixed():
        F.set_precision(1)
        if F.numeric(Ph) != 0:
            raise RuntimeError("numeric failed: " + tb.last_error())
        its = lib.taucs_b200_solve_refine(F.h, None, nrhs, h_x, h_b, TOL, 10, res_buf)
        if its < 0:
            raise RuntimeError("refinement did not reach the target: " + tb.last_error())

    def step_e2e_fp64():
        F.set_precision(0)
        if F.numeric(Ph) != 0:
            raise RuntimeError("numeric failed: " + tb.last_error())
        if lib.taucs_supernodal_solve_llt(F.h, h_x, h_b) != 0:
            raise RuntimeError("solve failed: " + tb.last_error())

    # autotuner (setup, untimed): per-level GEMM variants from measured times
    t_tune = time.perf_counter()
    tuned = {}
    for prec in ((1, 0) if mixed else (0,)):
        F.set_precision(prec)
        tuned["fp32" if prec else "fp64"] = [int(c) for c in F.autotune(d_vals.data_ptr())]
    t_tune = time.perf_counter() - t_tune

    step_main = step_mixed if mixed else step_fp64
    step_e2e = step_e2e_mixed if mixed else step_e2e_fp64

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v):
        return max_over_ranks_of(dist, v, "cuda")

    def timed(step, k):
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = None
        for _ in range(k):
            out = step()
        e1.record(stream)
        barrier()
        return max_over_ranks(e0.elapsed_time(e1)), out

    def x_host():
        torch.cuda.synchronize()
        return d_x.cpu().numpy().reshape(nrhs, n).T

    W = max(args.warmup, 3)
    K = args.steps
    # ---- the measured form, device-resident
    for _ in range(W):
        step_main()
    clocks = ClockSampler(local_rank)
    clocks.start()
    tb.launch_count(reset=True)
    ms, its = timed(step_main, K)
    clk = clocks.stop()
    launches = tb.launch_count(reset=True) // max(K, 1)
    X = x_host()
    res_main = max(scaled_residual(P, X[:, q], B[:, q]) for q in range(nrhs))
    steps_main = its if mixed else None

    # ---- the plain FP64 path on the same inputs (mixed80 only)
    fp64 = None
    if mixed:
        for _ in range(W):
            step_fp64()
        ms64, _ = timed(step_fp64, K)
        X64 = x_host()
        res64 = max(scaled_residual(P, X64[:, q], B[:, q]) for q in range(nrhs))
        fp64 = {"value": world * K / (ms64 * 1e-3), "unit": UNIT, "ms_per_step": ms64 / K,
                "scaled_residual": res64, "speedup_of_fp32_refine": ms64 / ms,
                "max_rel_diff_x": float(np.max(np.abs(X - X64)) / np.max(np.abs(X64)))}

    # ---- end-to-end through the C ABI with pinned host buffers
    for _ in range(2):
        step_e2e()
    ms_e2e, _ = timed(step_e2e, K)
    Xe = h_x.reshape(nrhs, n).T
    res_e2e = max(scaled_residual(P, Xe[:, q], B[:, q]) for q in range(nrhs))

    # ---- roofline: CUDA events around every launch, separate profiled steps
    lib.taucs_b200_profile(1)
    nprof = max(2, min(K, 3))
    for _ in range(nprof):
        step_main()
    torch.cuda.synchronize()
    kern = read_profile(tb, nprof)
    lib.taucs_b200_profile(0)

    peaks = measured_peaks()
    hbm_peak = peaks.get("hbm_gbs")
    if mixed and args.split_format == 1 and peaks.get("bf16_tflops_sustained"):
        bf16 = peaks["bf16_tflops_sustained"]
        tensor_peak = bf16 / 3.0
        tensor_src = (f"MEASURED_PEAKS.json bf16_tflops_sustained ({bf16:.0f} TF/s; the products run inside a "
                      f"long step) / 3: the FP16x3 products do 3 FP16 MMAs (the bf16 rate) per FP32-accurate "
                      f"product (of measured)")
    elif mixed:
        tf32 = tf32_gemm_peak()
        tensor_peak = tf32 / 3.0
        tensor_src = (f"cuBLAS TF32 GEMM 8192^3 measured in this run ({tf32:.0f} TF/s) / 3: the TF32x3 "
                      f"products do 3 tensor-core MMAs per FP32-accurate product (of measured)")
    else:
        tensor_peak = fp64_gemm_peak()
        tensor_src = "FP64: cuBLAS DGEMM 8192^3 measured in this run (of measured)"
    traffic = TRAFFIC_PER_ALG_BYTE if mixed else None
    roof = roofline(kern, tensor_peak, tensor_src, hbm_peak, traffic)
    # the update-matrix product, the dominant tensor-core kernel, beside it
    roof_gemm = roofline(kern, tensor_peak, tensor_src, hbm_peak, traffic, dom="gemm_u")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline_sample(args.workload, g, info.flops, [os.cpu_count() or 1, 1])
        except Exception as exc:  # report, never hide
            cpu = {"error": repr(exc)}

    serving = None
    if mixed and world == 1 and not args.no_serving:
        F.free()
        torch.cuda.empty_cache()
        try:
            serving = run_serving(tb, seconds=args.serve_seconds)
        except Exception as exc:  # report, never hide
            serving = {"error": repr(exc)}

    h2d = 8 * nnz + 8 * n * nrhs
    d2h = 8 * n * nrhs + (8 * nrhs if mixed else 4)
    out = {
        "metric": METRIC_MIXED if mixed else METRIC_FP64, "value": world * K / (ms * 1e-3), "unit": UNIT,
        "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if mixed else "f64", "data": "synthetic",
        "config": workload_config(args.workload, g, n, nnz, nrhs),
        "problem": {"flops": info.flops, "supernodes": info.n_live, "levels": info.n_levels,
                   "max_front": info.max_front, "l_gb_fp64": info.l_bytes / 1e9,
                   "u_arena_gb_fp64": info.u_bytes / 1e9,
                   "l2_policy": "inputs larger than L2 (several GB of L and update arena touched per step)",
                   "parallelism": f"replicas x{world}",
                   "autotuned_gemm_variants": tuned, "autotune_s": t_tune},
        "clocks": clk,
        "e2e": {"value": world * K / (ms_e2e * 1e-3), "unit": UNIT, "ms_per_step": ms_e2e / K,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches),
        "roofline": roof,
        "roofline_gemm_u": roof_gemm,
        "kernels": kern,
        "cpu_baseline": cpu,
        "scaled_residual": {"device": res_main, "e2e": res_e2e},
        "x_checksum": x_checksum(X),
    }
    if mixed:
        out["refinement_steps"] = steps_main
        out["fp64"] = fp64
        out["serving"] = serving
    else:
        out["factor_tflop_s"] = info.flops / (ms / K * 1e-3) / 1e12
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    F.free()
    torch.cuda.empty_cache()
    # the other configurations' workloads, measured the same way, beside the line
    if mixed and world == 1 and not args.no_extra_legs:
        for key, wl in (("fp64_mesh3d64", "fp64-64"), ("batch4096", "batch4096")):
            a2 = argparse.Namespace(**vars(args))
            a2.workload, a2.grid, a2.no_cpu_baseline, a2.no_serving, a2.no_extra_legs = wl, None, True, True, True
            try:
                out[key] = run_batch(a2) if wl == "batch4096" else run_ours(a2)
            except Exception as exc:  # report, never hide
                out[key] = {"error": repr(exc)}
            torch.cuda.empty_cache()
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    out = run_batch(args) if args.workload == "batch4096" else run_ours(args)
    if dist_env()[0] == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
