"""Batched uneven-size factorizations over ragged batches on one B200.

The numax spelling of a batch of small Cholesky solves is
`map_blocks[step=solve_step, gpu=True](problems, out)` with the Array-tier
`cholesky` + `cholesky_solve` inside `step`
(numax/core/functional.mojo:691-834; examples/advanced/batched_solve.mojo:
75-104): one fixed, compile-time n <= 64 per launch, one problem per GPU
thread.  Here a batch holds matrices of different orders (1..128) in a
ragged row-major layout and runs as one plan:

    plan = CholeskySolveBatch(ns, nrhs=4, dtype=torch.float64)
    L_in_A, X, info = plan(A, B)          # A, B: flat CUDA tensors

Ragged layout: matrix i occupies A[a_off[i] : a_off[i] + n_i*n_i] row-major,
a_off = exclusive prefix sum of n_i^2; its right-hand sides occupy
B[b_off[i] : b_off[i] + n_i*nrhs] row-major (n_i x nrhs), b_off the prefix
sum of n_i*nrhs.  `ragged_offsets` computes both.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib

_DT = {torch.float64: (_lib.NMX_F64, "f64"), torch.float32: (_lib.NMX_F32, "f32")}


def tile_shape(warps: int) -> int:
    """CTA shape code of the 8 x 8 DMMA tile kernel with `warps` (1, 2, 4 or
    8) warps per matrix, as the schedule reports it."""
    if warps not in (1, 2, 4, 8):
        raise ValueError("warps must be 1, 2, 4 or 8")
    return 1000 + 32 * warps


def ragged_offsets(ns, cols=None) -> np.ndarray:
    """Element offsets of a ragged batch: matrix i is n_i x (cols or n_i)."""
    ns = np.asarray(ns, dtype=np.int64)
    sizes = ns * (ns if cols is None else cols)
    off = np.zeros(len(ns), dtype=np.int64)
    if len(ns) > 1:
        off[1:] = np.cumsum(sizes)[:-1]
    return off


def partition(ns, ndev: int, nrhs: int = 4):
    """Split a ragged batch over `ndev` devices by predicted cost (longest
    processing time first; host only, nmx_batched_partition).  Returns
    (dev_of, cost_per_dev): the device of each matrix and each device's
    total predicted cost."""
    ns = np.ascontiguousarray(ns, dtype=np.int32)
    dev_of = np.empty(len(ns), dtype=np.int32)
    cost = np.empty(ndev, dtype=np.float64)
    _lib.call("nmx_batched_partition", len(ns), ns.ctypes.data, int(nrhs), int(ndev),
              dev_of.ctypes.data, cost.ctypes.data)
    return dev_of, cost


def _resolve_device(device) -> torch.device:
    if device is None:
        return torch.device("cuda", torch.cuda.current_device())
    device = torch.device(device)
    if device.type != "cuda":
        raise ValueError(f"numax_b200 runs on CUDA devices only, not {device}")
    if device.index is None:
        device = torch.device("cuda", torch.cuda.current_device())
    return device


def _stream_ptr(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _check_tensor(name, t, dtype, numel, device):
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if t.device != device:
        raise ValueError(f"{name} is on {t.device}, expected {device}")
    if t.dtype != dtype:
        raise TypeError(f"{name} has dtype {t.dtype}, expected {dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if t.numel() < numel:
        raise ValueError(f"{name} has {t.numel()} elements, the batch needs {numel}")


class CholeskySolveBatch:
    """A reusable plan for `cholesky` + `cholesky_solve` over a ragged batch.

    Per matrix the arithmetic follows numax's Array tier
    (numax/linalg/_array/cholesky.mojo:26-92): only the lower triangle of A_i
    is read, the diagonal is floored by guard_nonzero(d, 1e-30) before the
    square root (so a negative pivot yields NaN rather than raising), and the
    solves divide by guard_nonzero(l_ii, 1e-30).  On top of numax, `info[i]`
    reports the first pivot d <= 0 (1-based; 0 = positive definite), the
    rule of numax's potrf_diag (numax/linalg/panel.mojo:216-286).
    """

    def __init__(self, ns, nrhs: int = 4, dtype=torch.float64, device=None):
        if dtype not in _DT:
            raise TypeError("dtype must be torch.float32 or torch.float64")
        self.device = _resolve_device(device)
        self.dtype = dtype
        self.nrhs = int(nrhs)
        self.ns = np.ascontiguousarray(ns, dtype=np.int32)
        self.count = int(self.ns.size)
        self._ctx = _lib.context(self.device.index)
        h = C.c_void_p()
        code, self._suffix = _DT[dtype]
        _lib.call("nmx_potrf_potrs_batched_plan", self._ctx, code, self.count,
                  self.ns.ctypes.data if self.count else None, self.nrhs, C.byref(h))
        self._plan = h.value
        a, b = C.c_int64(), C.c_int64()
        _lib.call("nmx_batched_plan_sizes", self._plan, C.byref(a), C.byref(b))
        self.a_elems, self.b_elems = a.value, b.value

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan:
            try:
                _lib.load().nmx_batched_plan_destroy(plan)
            except Exception:
                pass
            self._plan = None

    def _operands(self, A, B, X, info, L):
        _check_tensor("A", A, self.dtype, self.a_elems, self.device)
        if L is None:
            L = A
        _check_tensor("L", L, self.dtype, self.a_elems, self.device)
        if self.nrhs:
            _check_tensor("B", B, self.dtype, self.b_elems, self.device)
            if X is None:
                X = torch.empty(self.b_elems, dtype=self.dtype, device=self.device)
            _check_tensor("X", X, self.dtype, self.b_elems, self.device)
        if info is None:
            info = torch.empty(self.count, dtype=torch.int32, device=self.device)
        _check_tensor("info", info, torch.int32, self.count, self.device)
        return L, X, info

    def _ptrs(self, A, B, X, info, L):
        return (A.data_ptr(), L.data_ptr(), B.data_ptr() if self.nrhs else None,
                X.data_ptr() if self.nrhs else None, info.data_ptr())

    def run(self, A: torch.Tensor, B: torch.Tensor | None, X: torch.Tensor | None = None,
            info: torch.Tensor | None = None, L: torch.Tensor | None = None, graph: bool = False):
        """Enqueue on the current stream.  The factors' lower triangles go to
        L (default: A itself, in place; the upper triangles are not written).
        graph=True replays a CUDA graph of the plan's launches (captured the
        first time these buffers are seen).  Returns (L, X, info) without
        synchronizing."""
        L, X, info = self._operands(A, B, X, info, L)
        fn = f"nmx_potrf_potrs_batched_{'graph_' if graph else ''}{self._suffix}"
        _lib.call(fn, self._ctx, self._plan, *self._ptrs(A, B, X, info, L),
                  _stream_ptr(self.device))
        return L, X, info

    def autotune(self, A, B, X=None, info=None, L=None, reps: int = 3):
        """Time every CTA shape that covers each size bucket on these
        buffers and keep the fastest (synchronizes; the outputs hold a valid
        result afterwards).  Returns the schedule."""
        L, X, info = self._operands(A, B, X, info, L)
        _lib.call("nmx_batched_plan_autotune", self._ctx, self._plan, *self._ptrs(A, B, X, info, L),
                  int(reps), _stream_ptr(self.device))
        return self.schedule()

    def force_shape(self, threads: int, bucket: int = -1):
        """Fix the CTA shape of one size bucket (or all, bucket = -1): 64, 96,
        128 or 192 threads (packed-triangle kernel) or tile_shape(w) =
        1000 + 32 w for w = 1, 2, 4, 8 warps per matrix (the kernel on 8 x 8
        DMMA tiles, FP64 arithmetic).  Returns the schedule."""
        _lib.call("nmx_batched_plan_set_shape", self._ctx, self._plan, int(bucket), int(threads))
        return self.schedule()

    def schedule(self):
        """Per size bucket (largest n first): n_max, threads per CTA, CTAs."""
        nmax, thr, ctas = (C.c_int32 * 8)(), (C.c_int32 * 8)(), (C.c_int32 * 8)()
        nb = C.c_int32()
        _lib.call("nmx_batched_plan_schedule", self._plan, nmax, thr, ctas, 8, C.byref(nb))
        return [{"n_max": nmax[i], "threads": thr[i], "ctas": ctas[i]} for i in range(nb.value)]

    def __call__(self, A, B, X=None, info=None, L=None):
        """Synchronous, like numax: factor (in place unless L is given),
        solve, synchronize, return (L, X, info)."""
        out = self.run(A, B, X, info, L)
        torch.cuda.current_stream(self.device).synchronize()
        return out


def cholesky_solve_batched(ns, A, B, nrhs: int = 4):
    """One-shot form: plan, run, synchronize.  Returns (A with L, X, info)."""
    plan = CholeskySolveBatch(ns, nrhs=nrhs, dtype=A.dtype, device=A.device)
    return plan(A, B)


class EighBatch:
    """A reusable plan for the symmetric eigensolver over a ragged batch
    (float32 data, n_i in 1..64).

    numax's Array-tier `eigh[T, n, sweeps=12]`
    (numax/linalg/_array/eigen.mojo:316-392) runs 12 fixed cyclic Jacobi
    sweeps per matrix inside one GPU thread.  This runs parallel-order Jacobi
    with float64 rotation angles and a float64 off-diagonal stopping test
    (sweeps stop once off(A) <= tol * ||A||_F, at most `max_sweeps`).
    Eigenvalues are the final diagonal; with sort=False they come in the
    solver's diagonal order (numax's convention: unsorted), with sort=True
    ascending and V's columns permuted to match.
    """

    def __init__(self, ns, device=None):
        self.device = _resolve_device(device)
        self.ns = np.ascontiguousarray(ns, dtype=np.int32)
        self.count = int(self.ns.size)
        self._ctx = _lib.context(self.device.index)
        h = C.c_void_p()
        _lib.call("nmx_syevj_batched_plan", self._ctx, self.count,
                  self.ns.ctypes.data if self.count else None, C.byref(h))
        self._plan = h.value
        a, w = C.c_int64(), C.c_int64()
        _lib.call("nmx_syevj_plan_sizes", self._plan, C.byref(a), C.byref(w))
        self.a_elems, self.w_elems = a.value, w.value

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan:
            try:
                _lib.load().nmx_syevj_plan_destroy(plan)
            except Exception:
                pass
            self._plan = None

    def _outputs(self, A, W, V, sweeps):
        _check_tensor("A", A, torch.float32, self.a_elems, self.device)
        if W is None:
            W = torch.empty(self.w_elems, dtype=torch.float32, device=self.device)
        if V is None:
            V = torch.empty(self.a_elems, dtype=torch.float32, device=self.device)
        if sweeps is None:
            sweeps = torch.empty(self.count, dtype=torch.int32, device=self.device)
        _check_tensor("W", W, torch.float32, self.w_elems, self.device)
        _check_tensor("V", V, torch.float32, self.a_elems, self.device)
        _check_tensor("sweeps", sweeps, torch.int32, self.count, self.device)
        return W, V, sweeps

    def run(self, A, W=None, V=None, sweeps=None, tol: float = 1e-7, max_sweeps: int = 20,
            sort: bool = False, graph: bool = False):
        """Enqueue on the current stream; returns (W, V, sweeps).  graph=True
        replays a CUDA graph of the plan's launches (captured the first time
        these buffers and arguments are seen)."""
        W, V, sweeps = self._outputs(A, W, V, sweeps)
        fn = "nmx_syevj_batched_graph_f32" if graph else "nmx_syevj_batched_f32"
        _lib.call(fn, self._ctx, self._plan, A.data_ptr(), W.data_ptr(), V.data_ptr(),
                  sweeps.data_ptr(), float(tol), int(max_sweeps), int(bool(sort)),
                  _stream_ptr(self.device))
        return W, V, sweeps

    def autotune(self, A, W=None, V=None, sweeps=None, tol: float = 1e-7, max_sweeps: int = 20,
                 sort: bool = False, reps: int = 2):
        """Time every (threads, group) shape per size bucket on these buffers
        and keep the fastest (synchronizes; the outputs hold the kept
        schedule's result).  Returns the schedule."""
        W, V, sweeps = self._outputs(A, W, V, sweeps)
        _lib.call("nmx_syevj_plan_autotune", self._ctx, self._plan, A.data_ptr(), W.data_ptr(),
                  V.data_ptr(), sweeps.data_ptr(), float(tol), int(max_sweeps), int(bool(sort)),
                  int(reps), _stream_ptr(self.device))
        return self.schedule()

    def schedule(self):
        """Per size bucket: n_max, threads per CTA, threads per matrix, CTAs."""
        nmax, thr, grp, ctas = ((C.c_int32 * 8)() for _ in range(4))
        nb = C.c_int32()
        _lib.call("nmx_syevj_plan_schedule", self._plan, nmax, thr, grp, ctas, 8, C.byref(nb))
        return [{"n_max": nmax[i], "threads": thr[i], "group": grp[i], "ctas": ctas[i]}
                for i in range(nb.value)]

    def __call__(self, A, W=None, V=None, sweeps=None, tol: float = 1e-7, max_sweeps: int = 20,
                 sort: bool = False):
        out = self.run(A, W, V, sweeps, tol, max_sweeps, sort)
        torch.cuda.current_stream(self.device).synchronize()
        return out


def eigh_batched(ns, A, tol: float = 1e-7, max_sweeps: int = 20, sort: bool = False):
    """One-shot form of EighBatch: returns (W, V, sweeps)."""
    return EighBatch(ns, device=A.device)(A, tol=tol, max_sweeps=max_sweeps, sort=sort)
