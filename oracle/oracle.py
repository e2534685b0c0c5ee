"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Wraps oracle/liboracle.so (a C restatement of numax.linalg's algorithms,
numax 0.3.0) with numpy in and numpy out.  Only the tests, the smoke check
and the benchmark's CPU-baseline leg import this module; the library under
test never does.

Conventions follow numax: row-major matrices, 0-based LAPACK-style pivots
(`pivots[j]` = the row interchanged with row j), 1-based `info`.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build as _build

_LIB = None

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        path = _build.LIB
        if not os.path.exists(path):
            _build.build()
        _LIB = C.CDLL(path)
        for suf, ct in (("f64", np.float64), ("f32", np.float32)):
            fp = np.ctypeslib.ndpointer(dtype=ct, flags="C_CONTIGUOUS")
            vp = C.c_void_p
            sig = {
                "orc_array_cholesky": (None, [C.c_int, fp, fp]),
                "orc_array_cholesky_solve": (None, [C.c_int, fp, fp, fp, fp]),
                "orc_jacobi_eigh": (None, [C.c_int, C.c_int, fp, fp, fp, fp]),
                "orc_getrf_panel": (None, [fp, C.c_int64, C.c_int, C.c_int, C.c_int, _i32p, _i32p]),
                "orc_getrf2": (None, [fp, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p]),
                "orc_lu_factor": (C.c_int, [fp, C.c_int64, C.c_int, C.c_int, C.c_int, _i32p, _i32p]),
                "orc_lu_solve": (None, [fp, C.c_int64, _i32p, fp, C.c_int64, C.c_int, C.c_int, C.c_int]),
                "orc_potrf_diag": (None, [fp, C.c_int64, C.c_int, C.c_int, _i32p]),
                "orc_cholesky": (None, [fp, C.c_int64, C.c_int, C.c_int, C.c_int, _i32p]),
                "orc_cholesky_solve": (None, [fp, C.c_int64, fp, C.c_int64, C.c_int, C.c_int, C.c_int]),
                "orc_trsv": (None, [fp, C.c_int64, fp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
                "orc_trsm": (None, [fp, C.c_int64, fp, C.c_int64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
                "orc_qr_factor": (None, [fp, C.c_int64, C.c_int, C.c_int, C.c_int, fp, fp]),
                "orc_qr_q": (None, [fp, C.c_int64, C.c_int, C.c_int, C.c_int, fp, fp, C.c_int64, fp]),
                "orc_batched_cholesky_solve": (None, [C.c_int64, _i32p, _i64p, fp, vp, _i64p, fp, fp, C.c_int, C.c_int]),
                "orc_eigh": (C.c_int, [C.c_int, fp, C.c_int, fp, vp, fp]),
                "orc_batched_jacobi_eigh": (None, [C.c_int64, _i32p, _i64p, fp, _i64p, fp, fp, C.c_int, C.c_int]),
            }
            for name, (res, args) in sig.items():
                f = getattr(_LIB, f"{name}_{suf}")
                f.restype = res
                f.argtypes = args
        _LIB.orc_max_threads.restype = C.c_int
    return _LIB


def _suffix(dtype) -> str:
    dt = np.dtype(dtype)
    if dt == np.float64:
        return "f64"
    if dt == np.float32:
        return "f32"
    raise TypeError(f"oracle supports float32/float64, not {dt}")


def _fn(name: str, dtype):
    return getattr(lib(), f"{name}_{_suffix(dtype)}")


def max_threads() -> int:
    return lib().orc_max_threads()


# ---- Array tier (numax/linalg/_array) -------------------------------------

def array_cholesky(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a)
    n = a.shape[0]
    out = np.empty_like(a)
    _fn("orc_array_cholesky", a.dtype)(n, a, out)
    return out


def array_cholesky_solve(lower: np.ndarray, b: np.ndarray) -> np.ndarray:
    lower = np.ascontiguousarray(lower)
    b = np.ascontiguousarray(b, dtype=lower.dtype)
    n = lower.shape[0]
    x = np.empty(n, dtype=lower.dtype)
    tmp = np.empty(n, dtype=lower.dtype)
    _fn("orc_array_cholesky_solve", lower.dtype)(n, lower, b, x, tmp)
    return x


def jacobi_eigh(a: np.ndarray, sweeps: int = 12):
    """(values unsorted, vectors as columns) -- numax's Array-tier eigh."""
    a = np.ascontiguousarray(a)
    n = a.shape[0]
    w = np.empty(n, dtype=a.dtype)
    v = np.empty_like(a)
    work = np.empty_like(a)
    _fn("orc_jacobi_eigh", a.dtype)(n, sweeps, a, w, v, work)
    return w, v


# ---- Tensor tier ------------------------------------------------------------

def eigh(a: np.ndarray, vectors: bool = True):
    """(values ascending, vectors as columns or None) -- numax's Tensor-tier
    eigh / eigvalsh at block = 1 (sytrd, implicit QL, insertion sort, Q Z).
    Only the lower triangle of `a` is read."""
    a = np.ascontiguousarray(a)
    n = a.shape[0]
    w = np.empty(n, dtype=a.dtype)
    z = np.empty((n, n), dtype=a.dtype) if vectors else None
    work = np.empty(2 * n * n + 4 * n + 1, dtype=a.dtype)
    rc = _fn("orc_eigh", a.dtype)(n, a, n, w, z.ctypes.data if vectors else None, work)
    if rc:
        raise ValueError(f"eigvalsh: eigenvalue {rc - 1} did not converge in 60 sweeps -- the "
                         "matrix holds a NaN or an infinity")
    return w, z


def getrf_panel(a: np.ndarray, k: int, nb: int):
    """In place on a copy; returns (a, pivots, info)."""
    a = np.array(a, order="C")
    n = a.shape[0]
    piv = np.zeros(n, dtype=np.int32)
    info = np.zeros(1, dtype=np.int32)
    _fn("orc_getrf_panel", a.dtype)(a, n, n, k, nb, piv, info)
    return a, piv, int(info[0])


def getrf2(a: np.ndarray, k: int, nb: int, base: int):
    a = np.array(a, order="C")
    n = a.shape[0]
    piv = np.zeros(n, dtype=np.int32)
    info = np.zeros(1, dtype=np.int32)
    _fn("orc_getrf2", a.dtype)(a, n, n, k, nb, base, piv, info)
    return a, piv, int(info[0])


def lu_factor(a: np.ndarray, block: int = 32, base: int = 16):
    """numax lu_factor: returns (packed L\\U, pivots int32, sign, info)."""
    a = np.array(a, order="C")
    n = a.shape[0]
    piv = np.zeros(n, dtype=np.int32)
    info = np.zeros(1, dtype=np.int32)
    sign = _fn("orc_lu_factor", a.dtype)(a, n, n, block, base, piv, info)
    return a, piv, int(sign), int(info[0])


def lu_solve(lu: np.ndarray, piv: np.ndarray, b: np.ndarray, block: int = 32) -> np.ndarray:
    lu = np.ascontiguousarray(lu)
    x = np.array(b, dtype=lu.dtype, order="C")
    n = lu.shape[0]
    rhs = 1 if x.ndim == 1 else x.shape[1]
    ldb = 1 if x.ndim == 1 else rhs
    _fn("orc_lu_solve", lu.dtype)(lu, n, np.ascontiguousarray(piv, dtype=np.int32), x, ldb, n, rhs, block)
    return x


def plu(lu: np.ndarray, piv: np.ndarray):
    """(P, L, U) with A = P @ L @ U from the packed factor and the pivots,
    numax's `lu` (numax/linalg/lu.mojo:849-975)."""
    n = lu.shape[0]
    perm = np.arange(n)
    for j in range(n):
        p = int(piv[j])
        if p != j:
            perm[[j, p]] = perm[[p, j]]
    # rows of P^T A are A[perm]; so P = I[:, perm] ... A = P L U with P[perm[i], i] = 1
    P = np.zeros((n, n), dtype=lu.dtype)
    P[perm, np.arange(n)] = 1
    L = np.tril(lu, -1) + np.eye(n, dtype=lu.dtype)
    U = np.triu(lu)
    return P, L, U


def det(lu: np.ndarray, sign: int):
    return sign * np.prod(np.diag(lu))


def cholesky(a: np.ndarray, block: int = 64, tile: int = 128):
    """numax cholesky (tensor tier) on a copy: returns (L with zero upper, info)."""
    a = np.array(a, order="C")
    n = a.shape[0]
    info = np.zeros(1, dtype=np.int32)
    _fn("orc_cholesky", a.dtype)(a, n, n, block, tile, info)
    return a, int(info[0])


def potrf_diag(a: np.ndarray, k: int, nb: int):
    a = np.array(a, order="C")
    info = np.zeros(1, dtype=np.int32)
    _fn("orc_potrf_diag", a.dtype)(a, a.shape[0], k, nb, info)
    return a, int(info[0])


def cholesky_solve(lower: np.ndarray, b: np.ndarray, block: int = 16) -> np.ndarray:
    lower = np.ascontiguousarray(lower)
    x = np.array(b, dtype=lower.dtype, order="C")
    n = lower.shape[0]
    rhs = 1 if x.ndim == 1 else x.shape[1]
    ldb = 1 if x.ndim == 1 else rhs
    _fn("orc_cholesky_solve", lower.dtype)(lower, n, x, ldb, n, rhs, block)
    return x


def solve_triangular(a: np.ndarray, b: np.ndarray, upper: bool, unit: bool = False,
                     trans: bool = False, block: int = 16) -> np.ndarray:
    a = np.ascontiguousarray(a)
    x = np.array(b, dtype=a.dtype, order="C")
    n = a.shape[0]
    if x.ndim == 1:
        _fn("orc_trsv", a.dtype)(a, n, x, n, block, int(upper), int(unit), int(trans))
    else:
        _fn("orc_trsm", a.dtype)(a, n, x, x.shape[1], n, x.shape[1], block, int(upper), int(unit), int(trans))
    return x


def qr_factor(a: np.ndarray, block: int = 16):
    """numax qr_factor: returns (packed R + reflectors, taus)."""
    a = np.array(a, order="C")
    m, n = a.shape
    tau = np.zeros(n, dtype=a.dtype)
    scratch = np.zeros(block * block + 2 * block * max(n, 1), dtype=a.dtype)
    _fn("orc_qr_factor", a.dtype)(a, n, m, n, block, tau, scratch)
    return a, tau


def qr_r(factored: np.ndarray) -> np.ndarray:
    n = factored.shape[1]
    return np.triu(factored[:n, :n])


def qr_q(factored: np.ndarray, tau: np.ndarray, block: int = 16) -> np.ndarray:
    factored = np.ascontiguousarray(factored)
    m, n = factored.shape
    q = np.zeros((m, n), dtype=factored.dtype)
    scratch = np.zeros(block * block + 2 * block * max(n, 1), dtype=factored.dtype)
    _fn("orc_qr_q", factored.dtype)(factored, n, m, n, block, np.ascontiguousarray(tau), q, n, scratch)
    return q


# ---- batched (ragged) drivers ----------------------------------------------

def ragged_offsets(ns: np.ndarray, cols=None) -> np.ndarray:
    """Element offsets of a ragged batch: matrix i is n_i x (cols or n_i)."""
    ns = np.asarray(ns, dtype=np.int64)
    sizes = ns * (ns if cols is None else cols)
    off = np.zeros(len(ns), dtype=np.int64)
    if len(ns) > 1:
        off[1:] = np.cumsum(sizes)[:-1]
    return off


def batched_cholesky_solve(ns, A, B, nrhs: int, want_l: bool = True, threads: int = 0):
    """numax map_blocks(cholesky + cholesky_solve) over a ragged batch.
    Returns (L, X); L holds the factor's lower triangle (upper left as zero)."""
    ns = np.ascontiguousarray(ns, dtype=np.int32)
    a_off = ragged_offsets(ns)
    b_off = ragged_offsets(ns, nrhs)
    A = np.ascontiguousarray(A)
    B = np.ascontiguousarray(B, dtype=A.dtype)
    X = np.zeros_like(B)
    L = np.zeros_like(A) if want_l else None
    _fn("orc_batched_cholesky_solve", A.dtype)(
        len(ns), ns, a_off, A, None if L is None else L.ctypes.data, b_off, B, X, nrhs, threads)
    return L, X


def batched_jacobi_eigh(ns, A, sweeps: int = 12, threads: int = 0):
    ns = np.ascontiguousarray(ns, dtype=np.int32)
    a_off = ragged_offsets(ns)
    w_off = ragged_offsets(ns, 1)
    A = np.ascontiguousarray(A)
    W = np.zeros(int(ns.astype(np.int64).sum()), dtype=A.dtype)
    V = np.zeros_like(A)
    _fn("orc_batched_jacobi_eigh", A.dtype)(len(ns), ns, a_off, A, w_off, W, V, sweeps, threads)
    return W, V
