"""Benchmark: batched uneven-size Cholesky + cho_solve, matrices per second.

Workload (the batched leg of the headline metric): 100,000 SPD matrices per
GPU, n_i uniform in [8, 128], A_i = G G^T / n + n I with G iid N(0,1), 4
right-hand sides iid N(0,1), float64.  One step = one pass of the batched
factor + solve over the whole batch (plan built once, outside the timing).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank runs its own 100,000-matrix shard (weak
scaling, no collective on the data path); the time is the max over ranks.

Printed: one JSON line on rank 0 with the metric, the device-timed value
(inputs resident in HBM), the end-to-end value through the public API with
host<->device copies, the roofline of the batched kernel against the
measured HBM peak, and the oracle's CPU time on a bounded sample.
`--impl reference` times numax's own CPU algorithm for the path (the oracle,
a C restatement of numax's Array-tier cholesky + cholesky_solve run per
matrix over all host cores) instead.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "batched uneven Cholesky+cho_solve throughput (100k SPD, n~U[8,128], 4 RHS)"
UNIT = "matrices/s"
COUNT = 100_000
NMIN, NMAX, NRHS = 8, 128, 4
SEED = 20260303
PROFILE = os.path.join(ROOT, "profiles", "batched_potrf_f64_100k.md")


def draw_sizes(count, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    return rng.integers(NMIN, NMAX + 1, size=count).astype(np.int32)


def shard(rank, count, world=1):
    """Rank `rank`'s shard (weak scaling): the job draws world x count sizes
    and the library's partitioner (nmx_batched_partition, longest processing
    time first) splits them by predicted cost, every rank computing the same
    split with no communication.  Returns the rank's sizes and the seed of
    its data."""
    if world == 1:
        return draw_sizes(count, SEED), SEED
    from numax_b200.batched import partition
    ns_all = draw_sizes(count * world, SEED)
    dev_of, _ = partition(ns_all, world, NRHS)
    return ns_all[dev_of == rank], SEED + 1000 * rank


def max_over_ranks(x, world, device):
    """The largest x over the job's ranks (a step takes as long as its
    slowest rank); x itself on one rank."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world, per_rank, steps, seconds):
    """Whole-job throughput: every rank's `per_rank` units per step, over
    `steps` steps, in the slowest rank's `seconds`."""
    return world * per_rank * steps / seconds


def make_batch_torch(ns, nrhs, dtype, device, seed):
    """Ragged A (G G^T/n + n I per matrix) and B, generated size group by
    size group with a seeded torch generator on `device`."""
    import torch
    from numax_b200.batched import ragged_offsets
    a_off = torch.from_numpy(ragged_offsets(ns)).to(device)
    total_a = int((ns.astype(np.int64) ** 2).sum())
    total_b = int(ns.astype(np.int64).sum()) * nrhs
    A = torch.empty(total_a, dtype=dtype, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    ns_t = torch.from_numpy(ns).to(device)
    for n in np.unique(ns):
        idx = torch.nonzero(ns_t == int(n)).flatten()
        g = torch.randn((idx.numel(), int(n), int(n)), generator=gen, dtype=torch.float64,
                        device=device)
        m = g @ g.transpose(1, 2) / n + n * torch.eye(int(n), dtype=torch.float64, device=device)
        pos = a_off[idx][:, None] + torch.arange(int(n) * int(n), device=device)[None, :]
        A[pos.flatten()] = m.reshape(-1).to(dtype)
        del g, m, pos
    B = torch.randn(total_b, generator=gen, dtype=torch.float64, device=device).to(dtype)
    return A, B


def algorithmic_bytes(ns, nrhs, esize):
    """Bytes one pass must move: read lower(A), write lower(L), read B,
    write X (n*nrhs each), write info."""
    n = ns.astype(np.int64)
    return int((esize * (n * (n + 1) // 2 * 2 + 2 * nrhs * n)).sum() + 4 * len(ns))


def algorithmic_flops(ns, nrhs):
    n = ns.astype(np.float64)
    return float((n ** 3 / 3 + 2 * nrhs * n ** 2).sum())


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        rows = []
        for line in (self.out or "").strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, flags in rows for i, f in enumerate(flags)
                          if f.lower() == "active"})
        return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": rows[0][1],
                "reasons": reasons, "samples": len(rows)}


def arith_dtype(schedule, io_dtype):
    """The arithmetic type of a batched plan's launches: the tile kernel
    computes in FP64 for both element types, the packed kernel in the batch's
    own type."""
    kinds = {"f64" if (s["threads"] >= 1000 or io_dtype == "f64") else io_dtype for s in schedule}
    return kinds.pop() if len(kinds) == 1 else "+".join(sorted(kinds))


def kernel_name(shape, dtype):
    """The kernel a batched plan's CTA shape code selects."""
    if shape >= 1000:
        w = (shape - 1000) // 32
        return f"potrf_tile_batched_kernel<{w}> (8x8 DMMA tiles, {w} warps per matrix)"
    return f"potrf_potrs_batched_kernel<{'double' if dtype == 'f64' else 'float'}, {shape}>"


def read_traffic():
    """Per-launch DRAM bytes from the committed ncu summary, if any."""
    try:
        text = open(PROFILE).read()
    except OSError:
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", text)
    return float(m.group(1)) if m else None


def cpu_baseline_sample(ns_all, seed, target_s=10.0):
    """Oracle (numax's Array-tier algorithm, C, OpenMP over matrices) on a
    bounded sample of the workload; returns (mats/s, threads, sample text)."""
    from oracle import oracle as O
    threads = O.max_threads()
    rng = np.random.Generator(np.random.PCG64(seed + 7))

    def sample(count):
        ns = ns_all[:count]
        mats, rhs = [], []
        for n in ns:
            g = rng.standard_normal((n, n))
            mats.append((g @ g.T / n + n * np.eye(n)).ravel())
            rhs.append(rng.standard_normal(n * NRHS))
        return ns, np.concatenate(mats), np.concatenate(rhs)

    # The whole workload's size sequence (capped at 100k matrices), repeated
    # passes until about target_s seconds of CPU work.
    count = min(len(ns_all), 100_000)
    ns, A, B = sample(count)
    passes, dt = 0, 0.0
    t0 = time.perf_counter()
    while dt < target_s and passes < 50:
        O.batched_cholesky_solve(ns, A, B, NRHS, want_l=True, threads=threads)
        passes += 1
        dt = time.perf_counter() - t0
    return count * passes / dt, threads, (f"first {count} matrices of the workload's size sequence, "
                                          f"float64, {NRHS} RHS, {passes} passes, {dt:.2f} s")


def run_reference(args):
    """numax's own CPU algorithm for the path (the oracle), rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import build as obuild, oracle as O
    obuild.build()
    threads = O.max_threads()
    ns_all = draw_sizes(COUNT, SEED)
    per_step = int(os.environ.get("NMX_REF_SAMPLE", "8000"))
    rng = np.random.Generator(np.random.PCG64(SEED + 11))
    ns = ns_all[:per_step]
    mats, rhs = [], []
    for n in ns:
        g = rng.standard_normal((n, n))
        mats.append((g @ g.T / n + n * np.eye(n)).ravel())
        rhs.append(rng.standard_normal(n * NRHS))
    A, B = np.concatenate(mats), np.concatenate(rhs)
    for _ in range(args.warmup):
        O.batched_cholesky_solve(ns, A, B, NRHS, want_l=True, threads=threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.batched_cholesky_solve(ns, A, B, NRHS, want_l=True, threads=threads)
    dt = time.perf_counter() - t0
    value = per_step * args.steps / dt
    sample = (f"each step: first {per_step} matrices of the {COUNT}-matrix workload "
              f"(n~U[8,128], float64, {NRHS} RHS), Array-tier cholesky+cholesky_solve per matrix")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (PCG64 seeded)",
        "config": {"workload": "batched uneven Cholesky + cho_solve", "count": COUNT,
                   "n_range": [NMIN, NMAX], "nrhs": NRHS, "parallelism": f"cpu{threads}",
                   "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def haar_torch(n, gen, dev):
    """Haar-distributed orthogonal matrix: Q of a Gaussian's QR with the
    sign fix (data generation only; torch/cuSOLVER)."""
    import torch
    g = torch.randn((n, n), generator=gen, dtype=torch.float64, device=dev)
    q, r = torch.linalg.qr(g)
    q *= torch.sign(torch.diagonal(r))[None, :]
    del g, r
    return q


# Refinement modes per conditioning: (label, mode flags).  Every mode may
# escalate (BF16/FP16 -> BF16X3 -> BF16X6 -> FP64) so that each ends at FP64
# backward error; the final precision is reported beside the time.
IR_MODES = {
    1e2: [("bf16x3", "BF16X3"), ("fp16", "FP16"), ("bf16", "BF16")],
    1e5: [("bf16x6", "BF16X6"), ("bf16x3", "BF16X3"), ("fp16", "FP16")],
    1e8: [("bf16x6", "BF16X6"), ("fp16", "FP16")],
}


def run_lu_ir(n, kappas, dev, seed=SEED):
    """FP64 LU solve vs the low-precision-factor IR solve at order n,
    A = U diag(s) V^T (U, V Haar, s geometric 1..1/kappa), b = A x_true.
    Device time (CUDA events), inputs resident.  Workspaces are reserved
    first (nmx_gesv_ir_reserve); each mode runs twice and both times are
    reported: "cold" (first launch of its kernels) and "warm"."""
    import ctypes as C
    import torch
    from numax_b200 import _lib
    lib = _lib.load()
    ctx = _lib.context(dev.index)
    stream = torch.cuda.current_stream(dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed + 77)
    u = haar_torch(n, gen, dev)
    v = haar_torch(n, gen, dev)
    xt = torch.randn(n, generator=gen, dtype=torch.float64, device=dev)
    flag = lambda p: getattr(_lib, f"NMX_IR_{p}")
    _lib.call("nmx_gesv_ir_reserve", ctx, n, _lib.NMX_IR_BF16 | _lib.NMX_IR_ESCALATE)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    lu = torch.empty((n, n), dtype=torch.float64, device=dev)
    piv = torch.empty(n, dtype=torch.int32, device=dev)
    info = torch.empty(1, dtype=torch.int32, device=dev)
    out = {}
    for ki, kappa in enumerate(kappas):
        s = torch.logspace(0.0, -np.log10(kappa), n, dtype=torch.float64, device=dev)
        a = (u * s[None, :]) @ v.T
        b = a @ xt
        norm_a = float(a.abs().sum(1).max())

        def berr(x):
            r = b - a @ x
            return float(r.abs().max() / (norm_a * x.abs().max() + b.abs().max()))

        # FP64: nmx_getrf_f64 + nmx_getrs_f64 on a copy (the first kappa also
        # runs it once untimed, so the timed call allocates nothing).
        x64 = torch.empty_like(b)

        def fp64_solve():
            lu.copy_(a)
            x64.copy_(b)
            torch.cuda.synchronize(dev)
            e0.record(stream)
            _lib.call("nmx_getrf_f64", ctx, n, lu.data_ptr(), n, piv.data_ptr(), info.data_ptr(),
                      stream.cuda_stream)
            _lib.call("nmx_getrs_f64", ctx, n, 1, lu.data_ptr(), n, piv.data_ptr(),
                      x64.data_ptr(), 1, stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            return e0.elapsed_time(e1)
        if ki == 0:
            fp64_solve()
        t64 = fp64_solve()
        res = {"fp64_lu_solve_ms": t64, "fp64_backward_error": berr(x64)}
        for label, prec in IR_MODES.get(kappa, IR_MODES[1e8]):
            mode = flag(prec) | _lib.NMX_IR_AUTO | _lib.NMX_IR_ESCALATE
            times = []
            for rep in range(2):
                x = torch.empty_like(b)
                st = _lib.IrStats()
                torch.cuda.synchronize(dev)
                e0.record(stream)
                rc = lib.nmx_gesv_ir_f64(ctx, n, C.c_void_p(a.data_ptr()), n,
                                         C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), mode,
                                         1e-14, 60, C.byref(st), C.c_void_p(stream.cuda_stream))
                e1.record(stream)
                torch.cuda.synchronize(dev)
                if rc != 0:
                    res[f"{label}_ir_error"] = _lib.last_error()
                    break
                times.append(e0.elapsed_time(e1))
            if len(times) < 2:
                continue
            fe = float((x - x64).abs().max() / x64.abs().max())
            res[label] = {
                "solve_ms_warm": times[1], "solve_ms_cold": times[0],
                "backward_error": berr(x), "converged": bool(st.converged),
                "final_precision": _lib.IR_PRECISION_NAMES.get(st.final_precision, "?"),
                "iterations": st.iterations, "gmres_iterations": st.gmres_iterations,
                "used_gmres": bool(st.used_gmres), "factor_ms": st.factor_ms,
                "refine_ms": st.refine_ms, "forward_diff_vs_fp64": fe,
                "speedup_fp64_over_ir": t64 / times[1]}
        out[f"{kappa:.0e}"] = res
        del a, b, s
        torch.cuda.empty_cache()
    del lu
    return out


def run_dense(dev, orders=(4096, 8192, 16384), nrhs=16, qr_m=262144, qr_n=256, seed=SEED,
              eigh_n=4096):
    """The dense factorizations at the single-matrix configs: FP64 LU + 16-RHS
    solve and FP64 Cholesky + 16-RHS solve at each order, FP32 Householder QR
    (geqrf, then orgqr) of qr_m x qr_n; FP64 eigh / eigvalsh of one
    eigh_n x eigh_n symmetric matrix (0 skips it).  Device time (CUDA events)
    of one call each after a warm-up call; rates in TF/s (LAPACK flop
    counts)."""
    import torch
    from numax_b200 import _lib
    ctx = _lib.context(dev.index)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed + 31)
    ev = lambda: torch.cuda.Event(enable_timing=True)

    def timed(fn):
        fn()
        torch.cuda.synchronize(dev)
        e0, e1 = ev(), ev()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1)

    out = {"nrhs": nrhs, "lu_f64": {}, "cholesky_f64": {}}
    for n in orders:
        a = torch.randn((n, n), generator=gen, dtype=torch.float64, device=dev)
        b = torch.randn((n, nrhs), generator=gen, dtype=torch.float64, device=dev)
        lu, x = torch.empty_like(a), torch.empty_like(b)
        piv = torch.empty(n, dtype=torch.int32, device=dev)
        info = torch.empty(1, dtype=torch.int32, device=dev)

        def lu_solve():
            lu.copy_(a)
            x.copy_(b)
            _lib.call("nmx_getrf_f64", ctx, n, lu.data_ptr(), n, piv.data_ptr(), info.data_ptr(), sp)
            _lib.call("nmx_getrs_f64", ctx, n, nrhs, lu.data_ptr(), n, piv.data_ptr(),
                      x.data_ptr(), nrhs, sp)
        ms = timed(lu_solve)
        fl = 2 * n ** 3 / 3 + 2 * n * n * nrhs
        berr = float((b - a @ x).abs().max() / (a.abs().sum(1).max() * x.abs().max() + b.abs().max()))
        out["lu_f64"][str(n)] = {"ms": ms, "tflops": fl / ms / 1e9, "backward_error": berr}
        g = torch.randn((n, n), generator=gen, dtype=torch.float64, device=dev)
        spd = g @ g.T / n + torch.eye(n, dtype=torch.float64, device=dev)
        del g

        def chol_solve():
            lu.copy_(spd)
            x.copy_(b)
            _lib.call("nmx_potrf_f64", ctx, n, lu.data_ptr(), n, info.data_ptr(), sp)
            _lib.call("nmx_potrs_f64", ctx, n, nrhs, lu.data_ptr(), n, x.data_ptr(), nrhs, sp)
        ms = timed(chol_solve)
        fl = n ** 3 / 3 + 2 * n * n * nrhs
        berr = float((b - spd @ x).abs().max() /
                     (spd.abs().sum(1).max() * x.abs().max() + b.abs().max()))
        out["cholesky_f64"][str(n)] = {"ms": ms, "tflops": fl / ms / 1e9, "backward_error": berr}
        del a, b, lu, x, spd
        torch.cuda.empty_cache()
    q = torch.randn((qr_m, qr_n), generator=gen, dtype=torch.float32, device=dev)
    f = torch.empty_like(q)
    qq = torch.empty_like(q)
    tau = torch.empty(qr_n, dtype=torch.float32, device=dev)

    def geqrf():
        f.copy_(q)
        _lib.call("nmx_geqrf_f32", ctx, qr_m, qr_n, f.data_ptr(), qr_n, tau.data_ptr(), sp)
    ms = timed(geqrf)
    fl = 2 * qr_m * qr_n ** 2 - 2 * qr_n ** 3 / 3
    ms_q = timed(lambda: _lib.call("nmx_orgqr_f32", ctx, qr_m, qr_n, f.data_ptr(), qr_n,
                                   tau.data_ptr(), qq.data_ptr(), qr_n, sp))
    orth = float((qq.T.double() @ qq.double() - torch.eye(qr_n, dtype=torch.float64, device=dev)).abs().max())
    out["qr_f32"] = {"m": qr_m, "n": qr_n, "geqrf_ms": ms, "tflops": fl / ms / 1e9,
                     "orgqr_ms": ms_q, "q_orthogonality_err": orth}
    del q, f, qq
    torch.cuda.empty_cache()
    if eigh_n:
        out["eigh_f64"] = run_eigh_dense(dev, eigh_n, gen)
    return out


def run_eigh_dense(dev, n, gen):
    """Symmetric eigendecomposition of one n x n FP64 matrix (G + G^T)/2:
    eigh (values and vectors: tridiagonalization, divide and conquer, Q Z)
    and eigvalsh (tridiagonalization, bisection), device time of one call
    after a warm-up call.  The tridiagonalization reads the trailing matrix
    once per column: n^3 / 3 doubles in all, its algorithmic bytes.
    torch.linalg.eigh (cuSOLVER) on the same matrix is timed beside it for
    context only."""
    import torch
    from numax_b200 import linalg as L
    stream = torch.cuda.current_stream(dev)
    g = torch.randn((n, n), generator=gen, dtype=torch.float64, device=dev)
    a = (g + g.T) / 2
    del g

    def timed(fn):
        fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1), out
    ms, r = timed(lambda: L.eigh(a))
    ms_v, w = timed(lambda: L.eigvalsh(a))
    ms_ref, (wr, _) = timed(lambda: torch.linalg.eigh(a))
    V, W = r.vectors, r.values
    resid = float(torch.linalg.matrix_norm(a @ V - V * W, 2) / torch.linalg.matrix_norm(a, 2))
    orth = float((V.T @ V - torch.eye(n, dtype=torch.float64, device=dev)).abs().max())
    tri_bytes = 8.0 * n ** 3 / 3
    return {"n": n, "eigh_ms": ms, "eigvalsh_ms": ms_v, "residual": resid,
            "orthogonality_err": orth,
            "values_err_vs_cusolver": float((W - wr).abs().max() / wr.abs().max()),
            "eigvalsh_err_vs_cusolver": float((w - wr).abs().max() / wr.abs().max()),
            "tridiagonalization_algorithmic_gb": tri_bytes / 1e9,
            "eigvalsh_gbs": tri_bytes / ms_v / 1e6,
            "cusolver_eigh_ms": ms_ref}


def make_eigh_batch(count, dev, seed=SEED):
    """Half harmonic-well Hamiltonians (n = 24 on [-4, 4], omega ~ U[0.5, 2];
    diagonal 1/dx^2 + omega^2 x^2 / 2, off-diagonal -1/(2 dx^2)) and half
    dense (G + G^T)/2 with n ~ U{16..64}; float32, ragged row-major."""
    import torch
    from numax_b200.batched import ragged_offsets
    rng = np.random.Generator(np.random.PCG64(seed + 5))
    half = count // 2
    ns = np.concatenate([np.full(half, 24), rng.integers(16, 65, size=count - half)]).astype(np.int32)
    a_off = ragged_offsets(ns)
    A = torch.empty(int((ns.astype(np.int64) ** 2).sum()), dtype=torch.float32, device=dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed + 9)
    n, dx = 24, 8.0 / 23
    omega = torch.rand(half, generator=gen, dtype=torch.float64, device=dev) * 1.5 + 0.5
    xg = -4.0 + dx * torch.arange(n, dtype=torch.float64, device=dev)
    H = torch.zeros((half, n, n), dtype=torch.float64, device=dev)
    idx = torch.arange(n, device=dev)
    H[:, idx, idx] = 1.0 / dx ** 2 + (omega[:, None] ** 2) * xg[None, :] ** 2 / 2
    H[:, idx[:-1], idx[1:]] = -0.5 / dx ** 2
    H[:, idx[1:], idx[:-1]] = -0.5 / dx ** 2
    A[: half * n * n] = H.reshape(-1).to(torch.float32)
    ns_t = torch.from_numpy(ns).to(dev)
    a_off_t = torch.from_numpy(a_off).to(dev)
    for m in range(16, 65):
        sel = torch.nonzero(ns_t[half:] == m).flatten() + half
        if sel.numel() == 0:
            continue
        g = torch.randn((sel.numel(), m, m), generator=gen, dtype=torch.float64, device=dev)
        sym = (g + g.transpose(1, 2)) / 2
        pos = a_off_t[sel][:, None] + torch.arange(m * m, device=dev)[None, :]
        A[pos.flatten()] = sym.reshape(-1).to(torch.float32)
    return ns, A


def run_eigh(count, dev, steps=3, tol=1e-7, max_sweeps=20):
    """Batched Jacobi eigh throughput (matrices/s) and float32 eigenvalue
    error against float64 LAPACK (cuSOLVER) on a sample."""
    import torch
    import numax_b200 as nb
    from numax_b200.batched import ragged_offsets
    ns, A = make_eigh_batch(count, dev)
    plan = nb.EighBatch(ns, device=dev)
    W = torch.empty(plan.w_elems, dtype=torch.float32, device=dev)
    V = torch.empty(plan.a_elems, dtype=torch.float32, device=dev)
    sw = torch.empty(len(ns), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    schedule = plan.autotune(A, W, V, sw, tol=tol, max_sweeps=max_sweeps, sort=True, reps=2)
    for _ in range(3):
        plan.run(A, W, V, sw, tol=tol, max_sweeps=max_sweeps, sort=True, graph=True)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        plan.run(A, W, V, sw, tol=tol, max_sweeps=max_sweeps, sort=True, graph=True)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / steps
    sweeps = sw.double()
    # Error on a sample: 256 wells + 256 dense.
    ao, wo = ragged_offsets(ns), ragged_offsets(ns, 1)
    worst = 0.0
    half = count // 2
    for i in list(range(0, 256)) + list(range(half, half + 256)):
        n = int(ns[i])
        a = A[ao[i]:ao[i] + n * n].double().reshape(n, n)
        ref = torch.linalg.eigvalsh(a)
        got = W[wo[i]:wo[i] + n].double()
        worst = max(worst, float((got - ref).abs().max() / ref.abs().max()))
    n64 = ns.astype(np.float64)
    swp = sweeps.cpu().numpy()
    flops = float((9.0 * n64 ** 2 * (n64 - 1) * swp).sum())
    bytes_ = float((4 * (2 * n64 ** 2 + n64)).sum())
    return {"count": count, "ms": ms, "matrices_per_s": count / (ms / 1e3),
            "mean_sweeps": float(swp.mean()), "max_sweeps": int(swp.max()),
            "max_rel_eig_err_vs_fp64": worst, "flop_rate_tflops": flops / (ms / 1e3) / 1e12,
            "hbm_gbs": bytes_ / (ms / 1e3) / 1e9, "schedule": schedule,
            "launch": "CUDA graph of the plan (autotuned shapes)"}


def measure_gemm_peaks(dev, n=8192):
    """FP64 and FP32 (no TF32) GEMM rates of the vendor library at n^3 on this
    GPU, best of 3: the measured denominators of the FP64 and FP32 roofline
    fractions (the peak file lists HBM and BF16 only)."""
    import torch
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    out = {}
    try:
        for name, dt in (("fp64_gemm_tflops", torch.float64), ("fp32_gemm_tflops", torch.float32)):
            a = torch.randn((n, n), dtype=dt, device=dev)
            b = torch.randn((n, n), dtype=dt, device=dev)
            best = float("inf")
            for _ in range(4):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                a @ b
                e1.record()
                torch.cuda.synchronize(dev)
                best = min(best, e0.elapsed_time(e1))
            out[name] = 2.0 * n ** 3 / best / 1e9
            del a, b
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev
    return out


def run_chol_ir(n, kappas, dev, seed=SEED):
    """FP64 Cholesky solve (nmx_potrf_f64 + nmx_potrs_f64) vs the
    mixed-precision Cholesky with FP64 refinement (nmx_posv_ir_f64) at order
    n, A = U diag(s) U^T (U Haar, s geometric 1..1/kappa).  Device time,
    inputs resident, workspaces reserved, each mode run twice (cold, warm)."""
    import ctypes as C
    import torch
    from numax_b200 import _lib
    lib = _lib.load()
    ctx = _lib.context(dev.index)
    stream = torch.cuda.current_stream(dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed + 91)
    u = haar_torch(n, gen, dev)
    xt = torch.randn(n, generator=gen, dtype=torch.float64, device=dev)
    _lib.call("nmx_posv_ir_reserve", ctx, n, _lib.NMX_IR_BF16 | _lib.NMX_IR_ESCALATE)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    work = torch.empty((n, n), dtype=torch.float64, device=dev)
    info = torch.empty(1, dtype=torch.int32, device=dev)
    out = {}
    for ki, kappa in enumerate(kappas):
        s = torch.logspace(0.0, -np.log10(kappa), n, dtype=torch.float64, device=dev)
        a = (u * s[None, :]) @ u.T
        a = (a + a.T) / 2
        b = a @ xt
        norm_a = float(a.abs().sum(1).max())

        def berr(x):
            r = b - a @ x
            return float(r.abs().max() / (norm_a * x.abs().max() + b.abs().max()))
        x64 = torch.empty_like(b)

        def fp64_solve():
            work.copy_(a)
            x64.copy_(b)
            torch.cuda.synchronize(dev)
            e0.record(stream)
            _lib.call("nmx_potrf_f64", ctx, n, work.data_ptr(), n, info.data_ptr(),
                      stream.cuda_stream)
            _lib.call("nmx_potrs_f64", ctx, n, 1, work.data_ptr(), n, x64.data_ptr(), 1,
                      stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            return e0.elapsed_time(e1)
        if ki == 0:
            fp64_solve()
        t64 = fp64_solve()
        res = {"fp64_cholesky_solve_ms": t64, "fp64_backward_error": berr(x64)}
        for label, prec in IR_MODES.get(kappa, IR_MODES[1e8]):
            mode = getattr(_lib, f"NMX_IR_{prec}") | _lib.NMX_IR_AUTO | _lib.NMX_IR_ESCALATE
            times = []
            for rep in range(2):
                x = torch.empty_like(b)
                st = _lib.IrStats()
                torch.cuda.synchronize(dev)
                e0.record(stream)
                rc = lib.nmx_posv_ir_f64(ctx, n, C.c_void_p(a.data_ptr()), n,
                                         C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), mode,
                                         1e-14, 60, C.byref(st), C.c_void_p(stream.cuda_stream))
                e1.record(stream)
                torch.cuda.synchronize(dev)
                if rc != 0:
                    res[f"{label}_ir_error"] = _lib.last_error()
                    break
                times.append(e0.elapsed_time(e1))
            if len(times) < 2:
                continue
            res[label] = {
                "solve_ms_warm": times[1], "solve_ms_cold": times[0],
                "backward_error": berr(x), "converged": bool(st.converged),
                "final_precision": _lib.IR_PRECISION_NAMES.get(st.final_precision, "?"),
                "iterations": st.iterations, "gmres_iterations": st.gmres_iterations,
                "factor_ms": st.factor_ms, "refine_ms": st.refine_ms,
                "forward_diff_vs_fp64": float((x - x64).abs().max() / x64.abs().max()),
                "speedup_fp64_over_ir": t64 / times[1]}
        out[f"{kappa:.0e}"] = res
        del a, b, s
        torch.cuda.empty_cache()
    del work, u
    return out


def run_lu_ir_legs(args, dev):
    """The LU/IR comparison at every requested order; errors are reported in
    place so that the batched line still prints."""
    kappas = [float(k) for k in args.lu_kappas.split(",") if k]
    legs = {"timing": "device events, inputs resident; workspaces reserved; cold = first call, "
                      "warm = second call of each mode", "orders": {}}
    for n in [int(v) for v in str(args.lu_n).split(",") if v and int(v) > 0]:
        try:
            legs["orders"][str(n)] = run_lu_ir(n, kappas, dev)
        except Exception as exc:
            legs["orders"][str(n)] = {"error": f"{type(exc).__name__}: {exc}"}
    if args.chol_n > 0:
        try:
            legs["cholesky"] = {"n": args.chol_n,
                                "results": run_chol_ir(args.chol_n, kappas, dev)}
        except Exception as exc:
            legs["cholesky"] = {"n": args.chol_n, "error": f"{type(exc).__name__}: {exc}"}
    return legs


def run_ours(args):
    import torch
    import torch.distributed as dist
    import numax_b200 as nb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    dtype = torch.float64 if args.dtype == "f64" else torch.float32
    esize = 8 if args.dtype == "f64" else 4

    ns, data_seed = shard(rank, args.count, world)
    A, B = make_batch_torch(ns, NRHS, dtype, dev, data_seed)
    L = torch.empty_like(A)
    X = torch.empty_like(B)
    info = torch.empty(len(ns), dtype=torch.int32, device=dev)
    plan = nb.CholeskySolveBatch(ns, nrhs=NRHS, dtype=dtype, device=dev)
    launches_per_step = len(set(min(3, (int(n) - 1) // 32) for n in np.unique(ns)))

    stream = torch.cuda.current_stream(dev)
    # Untimed: the autotuner picks each size bucket's CTA shape on this batch,
    # then the warm-up steps (the first one captures the step's CUDA graph).
    schedule = plan.autotune(A, B, X, info, L, reps=2)
    for _ in range(max(args.warmup, 3)):
        plan.run(A, B, X, info, L, graph=True)
    torch.cuda.synchronize(dev)
    bad = int((info != 0).sum().item())
    if bad:
        raise RuntimeError(f"{bad} matrices reported non-positive pivots")

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # ---- device-timed: inputs resident in HBM (A, L ~ 4.7 GB each >> L2) ----
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    barrier()
    with ClockSampler(local) as clocks:
        t_start = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for s in range(args.steps):
            ev[s][0].record(stream)
            plan.run(A, B, X, info, L, graph=True)
            ev[s][1].record(stream)
        t_end.record(stream)
        barrier()
    total_s = max_over_ranks(t_start.elapsed_time(t_end) / 1e3, world, dev)
    launch_s = float(np.mean([a.elapsed_time(b) for a, b in ev])) / 1e3
    value = job_value(world, len(ns), args.steps, total_s)

    # ---- the dominant kernel alone: the n in (96, 128] bucket -------------
    # (about half of the step), as a plan over the same sizes with its own
    # seeded data and its autotuned shape, timed per launch.
    ns_big = ns[ns > 96]
    Ab, Bb = make_batch_torch(ns_big, NRHS, dtype, dev, SEED + 77 + 1000 * rank)
    Lb, Xb = torch.empty_like(Ab), torch.empty_like(Bb)
    ib = torch.empty(len(ns_big), dtype=torch.int32, device=dev)
    plan_big = nb.CholeskySolveBatch(ns_big, nrhs=NRHS, dtype=dtype, device=dev)
    big_shape = plan_big.autotune(Ab, Bb, Xb, ib, Lb, reps=2)[0]["threads"]
    for _ in range(3):
        plan_big.run(Ab, Bb, Xb, ib, Lb)
    barrier()
    evb = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    for s in range(args.steps):
        evb[s][0].record(stream)
        plan_big.run(Ab, Bb, Xb, ib, Lb)
        evb[s][1].record(stream)
    barrier()
    big_s = max_over_ranks(float(np.mean([a.elapsed_time(b) for a, b in evb])) / 1e3, world, dev)
    del Ab, Bb, Lb, Xb, ib, plan_big

    # ---- end to end through the public API: pinned host in, host out --------
    hA = A.cpu().pin_memory()
    hB = B.cpu().pin_memory()
    hX = torch.empty(X.shape, dtype=dtype).pin_memory()
    hI = torch.empty(info.shape, dtype=torch.int32).pin_memory()
    dA = torch.empty_like(A)
    dB = torch.empty_like(B)
    e2e_steps = max(2, min(args.steps, 5))

    def e2e_step():
        dA.copy_(hA, non_blocking=True)
        dB.copy_(hB, non_blocking=True)
        plan(dA, dB, X, info, L)  # synchronous public call
        hX.copy_(X, non_blocking=True)
        hI.copy_(info, non_blocking=True)
        stream.synchronize()

    e2e_step()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    barrier()
    e2e_s = max_over_ranks(e0.elapsed_time(e1) / 1e3, world, dev)
    e2e_value = job_value(world, len(ns), e2e_steps, e2e_s)
    h2d = (hA.numel() + hB.numel()) * esize
    d2h = hX.numel() * esize + hI.numel() * 4
    np.testing.assert_array_equal(hI.numpy(), 0)

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    abytes = algorithmic_bytes(ns, NRHS, esize)
    achieved = abytes / launch_s / 1e9
    big_bytes = algorithmic_bytes(ns_big, NRHS, esize)
    big_achieved = big_bytes / big_s / 1e9
    traffic = read_traffic()

    gemm_peaks = {}
    if world == 1 and (args.eigh_count > 0 or args.dense):
        try:
            gemm_peaks = measure_gemm_peaks(dev)
        except Exception as exc:
            gemm_peaks = {"error": f"{type(exc).__name__}: {exc}"}

    eigh = None
    if world == 1 and args.eigh_count > 0:
        try:
            eigh = run_eigh(args.eigh_count, dev)
            eigh["hbm_frac"] = eigh["hbm_gbs"] / float(peaks.get("hbm_gbs", 6650.0))
            if "fp32_gemm_tflops" in gemm_peaks:
                eigh["fp32_frac_of_measured_sgemm"] = (eigh["flop_rate_tflops"] /
                                                       gemm_peaks["fp32_gemm_tflops"])
        except Exception as exc:
            eigh = {"error": f"{type(exc).__name__}: {exc}"}

    dense = None
    if world == 1 and args.dense:
        try:
            dense = run_dense(dev)
            for leg, key in (("lu_f64", "fp64_gemm_tflops"), ("cholesky_f64", "fp64_gemm_tflops")):
                if key in gemm_peaks:
                    for rec in dense[leg].values():
                        rec["frac_of_measured_gemm"] = rec["tflops"] / gemm_peaks[key]
            if "fp32_gemm_tflops" in gemm_peaks:
                dense["qr_f32"]["frac_of_measured_gemm"] = (dense["qr_f32"]["tflops"] /
                                                            gemm_peaks["fp32_gemm_tflops"])
        except Exception as exc:
            dense = {"error": f"{type(exc).__name__}: {exc}"}

    npy = None
    if world == 1 and args.npy_gib > 0:
        try:
            npy = run_npy(dev, A, args.npy_gib)
        except Exception as exc:
            npy = {"error": f"{type(exc).__name__}: {exc}"}

    lu_ir = None
    if world == 1 and args.lu_n:
        lu_ir = run_lu_ir_legs(args, dev)

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        from oracle import build as obuild
        obuild.build()
        rate, threads, sample = cpu_baseline_sample(ns, SEED)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": total_s / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": arith_dtype(schedule, args.dtype), "io_dtype": args.dtype,
        "data": "synthetic (seeded torch generator, A=GG^T/n+nI, B~N(0,1))",
        "config": {"workload": "batched uneven Cholesky + cho_solve", "count_per_gpu": len(ns),
                   "n_range": [NMIN, NMAX], "nrhs": NRHS, "parallelism": f"shard{world}",
                   "l2": "inputs larger than L2 (A and L %.1f GB each)" % (A.numel() * esize / 1e9),
                   "schedule": schedule, "launch": "CUDA graph of the plan (autotuned shapes)"},
        "roofline": {"bound": "hbm", "achieved": big_achieved, "peak": peak, "unit": "GB/s",
                     "frac": big_achieved / peak, "traffic": traffic,
                     "kernel": kernel_name(big_shape, args.dtype) + " (n in 97..128)",
                     "peak_source": peak_src + " (hbm_gbs, MEASURED_PEAKS.json)",
                     "algorithmic_bytes_per_launch": big_bytes, "matrices_per_launch": int(len(ns_big)),
                     "launch_ms": big_s * 1e3,
                     "fp64_tflops": algorithmic_flops(ns_big, NRHS) / big_s / 1e12,
                     "whole_step": {"achieved": achieved, "frac": achieved / peak,
                                    "algorithmic_bytes": abytes, "ms": launch_s * 1e3,
                                    "fp64_tflops": algorithmic_flops(ns, NRHS) / launch_s / 1e12}},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks.summary(),
        "cpu_baseline": cpu,
        "measured_gemm_peaks": gemm_peaks,
        "eigh": eigh,
        "dense": dense,
        "lu_ir": lu_ir,
        "npy": npy,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_npy(dev, A, gib=1.0, reps=3):
    """The .npy seam: save a `gib` GiB slice of the batch from HBM to a
    file and load it back into HBM (nmx_npy_save / nmx_npy_load, pinned
    staging, chunked reads overlapping the copies), against the numax-style
    path of a whole-file host read followed by one copy to the device
    (numpy.load, then torch .to(device)).  Wall-clock per synchronous call,
    best of `reps`; the file sits in the page cache (tmpfs when /dev/shm
    exists), so this is the host pipeline's rate, not a disk's.  The loaded
    bytes are compared with the source."""
    import shutil
    import tempfile
    import time
    import torch
    from numax_b200.io import numpy as npx
    esize = A.element_size()
    n = min(int(gib * (1 << 30)) // esize, A.numel())
    src = A[:n]
    base = "/dev/shm" if os.path.isdir("/dev/shm") else None
    tmp = tempfile.mkdtemp(prefix="nmx_npy_", dir=base)
    path = os.path.join(tmp, "slice.npy")
    try:
        def best(fn):
            ts = []
            for _ in range(reps):
                torch.cuda.synchronize(dev)
                t0 = time.perf_counter()
                out = fn()
                torch.cuda.synchronize(dev)
                ts.append(time.perf_counter() - t0)
            return min(ts), out
        t_save, _ = best(lambda: npx.save(src, path))
        t_load, got = best(lambda: npx.load(path, src.dtype, n, device=dev))
        same = bool(torch.equal(got.view(torch.uint8), src.view(torch.uint8)))
        del got
        t_ref, ref = best(lambda: torch.from_numpy(np.load(path)).to(dev))
        del ref
        nbytes = n * esize
        return {"bytes": nbytes, "file_system": "tmpfs (/dev/shm)" if base else "tmp",
                "save_gbs": nbytes / t_save / 1e9, "load_gbs": nbytes / t_load / 1e9,
                "numpy_load_then_copy_gbs": nbytes / t_ref / 1e9,
                "load_speedup": t_ref / t_load, "bit_exact": same}
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def run_big_bucket(args):
    """The n in 97..128 bucket of this rank's shard alone, the plan's default
    schedule (no autotuning), `warmup` untimed and `steps` timed launches; one
    JSON line with the mean launch time.  Used to profile the dominant kernel."""
    import torch
    import numax_b200 as nb
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    torch.cuda.set_device(dev)
    dtype = torch.float64 if args.dtype == "f64" else torch.float32
    ns, seed = shard(0, args.count, 1)
    ns_big = ns[ns > 96]
    A, B = make_batch_torch(ns_big, NRHS, dtype, dev, seed + 77)
    L, X = torch.empty_like(A), torch.empty_like(B)
    info = torch.empty(len(ns_big), dtype=torch.int32, device=dev)
    plan = nb.CholeskySolveBatch(ns_big, nrhs=NRHS, dtype=dtype, device=dev)
    for _ in range(max(args.warmup, 1)):
        plan.run(A, B, X, info, L)
    stream = torch.cuda.current_stream(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    torch.cuda.synchronize(dev)
    for e0, e1 in ev:
        e0.record(stream)
        plan.run(A, B, X, info, L)
        e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = float(np.mean([a.elapsed_time(b) for a, b in ev]))
    esize = 8 if args.dtype == "f64" else 4
    byt = algorithmic_bytes(ns_big, NRHS, esize)
    print(json.dumps({"bucket": "n in 97..128", "matrices": int(len(ns_big)),
                      "schedule": plan.schedule(), "launch_ms": ms,
                      "algorithmic_bytes_per_launch": byt, "achieved_gbs": byt / ms / 1e6,
                      "info_nonzero": int((info != 0).sum())}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--dtype", choices=["f64", "f32"], default="f64")
    ap.add_argument("--count", type=int, default=COUNT)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--lu-n", default="16384,32768",
                    help="comma-separated orders of the FP64-LU vs low-precision IR comparison "
                         "(0 skips it)")
    ap.add_argument("--lu-kappas", default="1e2,1e5,1e8",
                    help="comma-separated condition numbers for the comparison")
    ap.add_argument("--chol-n", type=int, default=16384,
                    help="order of the FP64-Cholesky vs mixed-precision Cholesky IR leg "
                         "(0 skips it)")
    ap.add_argument("--only-lu", action="store_true", help="run only the LU/IR comparison")
    ap.add_argument("--only-dense", action="store_true",
                    help="run only the dense LU/Cholesky/QR leg")
    ap.add_argument("--no-dense", dest="dense", action="store_false",
                    help="skip the dense LU/Cholesky/QR leg")
    ap.add_argument("--eigh-count", type=int, default=65536,
                    help="matrices in the batched Jacobi eigh leg (0 skips it)")
    ap.add_argument("--only-qr", action="store_true",
                    help="run only the FP32 QR leg (geqrf + orgqr of 262144 x 256), for profiling")
    ap.add_argument("--npy-gib", type=float, default=1.0,
                    help="GiB of the .npy save/load leg (0 skips it)")
    ap.add_argument("--only-npy", action="store_true",
                    help="run only the .npy save/load leg")
    ap.add_argument("--only-eigh", type=int, default=0,
                    help="run only the dense FP64 eigh / eigvalsh leg at this order, for profiling")
    ap.add_argument("--only-big", action="store_true",
                    help="run only the n in 97..128 bucket of the batch (the dominant kernel), "
                         "default schedule, for profiling")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.only_big:
        return run_big_bucket(args)
    if args.only_qr:
        import torch
        dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
        torch.cuda.set_device(dev)
        print(json.dumps({"dense": run_dense(dev, orders=(), eigh_n=0)}), flush=True)
        return 0
    if args.only_npy:
        import torch
        dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
        torch.cuda.set_device(dev)
        ns, seed = shard(0, args.count, 1)
        A, _ = make_batch_torch(ns, NRHS, torch.float64, dev, seed)
        print(json.dumps({"npy": run_npy(dev, A, args.npy_gib)}), flush=True)
        return 0
    if args.only_eigh:
        import torch
        dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
        torch.cuda.set_device(dev)
        gen = torch.Generator(device=dev)
        gen.manual_seed(SEED + 41)
        print(json.dumps({"eigh_f64": run_eigh_dense(dev, args.only_eigh, gen)}), flush=True)
        return 0
    if args.only_dense:
        import torch
        dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
        torch.cuda.set_device(dev)
        print(json.dumps({"dense": run_dense(dev)}), flush=True)
        return 0
    if args.only_lu:
        import torch
        dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
        torch.cuda.set_device(dev)
        print(json.dumps({"lu_ir": run_lu_ir_legs(args, dev)}), flush=True)
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
