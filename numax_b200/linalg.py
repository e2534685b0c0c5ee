"""numax.linalg's dense entry points over CUDA tensors, on libnmxla.so.

Mirrors numax's Tensor-tier call surface (numax/linalg/__init__.mojo:323-426):

    lu_factor(a) -> LU            numax/linalg/lu.mojo:454-701
    LU.solve(b), LU.det(), LU.slogdet()   numax/linalg/lu.mojo:181-451
    lu(a) -> (P, L, U), LU.plu()  numax/linalg/lu.mojo:877-975
    inverse(a)                    numax/linalg/basic.mojo:149-192
    qr_factor(a) -> QR, QR.r(), QR.q(), QR.apply_q_transpose(b), QR.solve(b), lstsq(a, b)
                                  numax/linalg/qr.mojo:330-746
    solve(a, b)                   numax/linalg/basic.mojo:55-146
    cholesky(a)                   numax/linalg/cholesky.mojo:233-468
    cholesky_solve(lower, b)      numax/linalg/cholesky.mojo:471-580
    solve_triangular(a, b, ...)   numax/linalg/triangular.mojo:228-425
    eigh(a) -> Eigh, eigvalsh(a)  numax/linalg/eigen.mojo:1220-1341, 1449+

Operands are torch tensors on a CUDA device standing in for numax's
`Tensor` over a `DeviceBuffer`: row-major, float64 or float32, 2-D with unit
column stride (a leading dimension is allowed), vectors 1-D.  Like numax,
inputs are borrowed and copied into the result's own storage, every call
synchronizes before returning, and the raised messages are numax's.
"""
from __future__ import annotations


import torch

from . import _lib
from .batched import _resolve_device

_SUF = {torch.float64: "f64", torch.float32: "f32"}


def _check_matrix(name, a, square=True):
    if not isinstance(a, torch.Tensor):
        raise TypeError(f"{name} must be a torch.Tensor")
    if a.device.type != "cuda":
        raise ValueError(f"{name} must be on a CUDA device (numax_b200 has no CPU path)")
    if a.dtype not in _SUF:
        raise TypeError(f"{name}: dtype {a.dtype} is not float32/float64")
    if a.dim() != 2:
        raise ValueError(f"{name} must be 2-D")
    if square and a.shape[0] != a.shape[1]:
        raise ValueError(f"{name} must be square, got {tuple(a.shape)}")


def _dense_copy(a):
    """A contiguous copy (numax copies its input into its own workspace)."""
    return a.contiguous().clone()


def _stream(dev):
    return torch.cuda.current_stream(dev).cuda_stream


def _ctx(dev):
    return _lib.context(dev.index)


def _as_rhs(b, n, dtype, device):
    if not isinstance(b, torch.Tensor) or b.device != device or b.dtype != dtype:
        raise TypeError("b must be a tensor with the matrix's dtype on its device")
    if b.shape[0] != n or b.dim() not in (1, 2):
        raise ValueError(f"b must have {n} rows")
    x = b.reshape(n, -1).contiguous().clone()
    return x


class LU:
    """A blocked LU with partial pivoting (numax's `LU`, numax/linalg/lu.mojo:75-451).

    `factored` holds L below the diagonal (unit diagonal implicit) and U on
    and above it; `pivots[j]` is the row column j interchanged with
    (0-based, LAPACK's ipiv convention); `sign` is the swap parity.
    """

    def __init__(self, factored, pivots, sign, info):
        self.factored = factored
        self.pivots = pivots
        self.sign = sign
        self.info = info
        self.n = factored.shape[0]

    def solve(self, b):
        """x with A x = b (vector or matrix b), reusing the factorization."""
        a = self.factored
        x = _as_rhs(b, self.n, a.dtype, a.device)
        if self.n:
            _lib.call(f"nmx_getrs_{_SUF[a.dtype]}", _ctx(a.device), self.n, x.shape[1], a.data_ptr(),
                      a.stride(0), self.pivots.data_ptr(), x.data_ptr(), x.shape[1], _stream(a.device))
        torch.cuda.current_stream(a.device).synchronize()
        return x.reshape(b.shape)

    def _slogdet3(self):
        a = self.factored
        out = torch.zeros(3, dtype=a.dtype, device=a.device)
        _lib.call(f"nmx_lu_slogdet_{_SUF[a.dtype]}", _ctx(a.device), self.n, a.data_ptr(),
                  max(1, a.stride(0)), self.pivots.data_ptr(), out.data_ptr(), _stream(a.device))
        return out.cpu().tolist()  # synchronizes

    def det(self):
        """det(A) = sign * prod(diag(U)) (numax/linalg/lu.mojo:382-403), on the device."""
        return self._slogdet3()[2]

    def slogdet(self):
        """(sign, ln|det|), (0, -inf) when singular (numax/linalg/lu.mojo:405-451)."""
        s, lg, _ = self._slogdet3()
        return float(s), float(lg)

    def plu(self):
        """(P, L, U) with A = P L U (numax's lu, numax/linalg/lu.mojo:877-975)."""
        a = self.factored
        P, L, U = (torch.empty_like(a) for _ in range(3))
        if self.n:
            _lib.call(f"nmx_lu_unpack_{_SUF[a.dtype]}", _ctx(a.device), self.n, a.data_ptr(),
                      a.stride(0), self.pivots.data_ptr(), P.data_ptr(), P.stride(0),
                      L.data_ptr(), L.stride(0), U.data_ptr(), U.stride(0), _stream(a.device))
        torch.cuda.current_stream(a.device).synchronize()
        return P, L, U


def lu_factor(a) -> LU:
    """Factor a (n x n) into P L U with partial pivoting, on a's device.

    Rank deficiency is not an error (numax/linalg/lu.mojo:96-98): an exactly
    zero pivot column leaves `info` = its 1-based index and the solves then
    produce non-finite values."""
    _check_matrix("a", a)
    dev = _resolve_device(a.device)
    n = a.shape[0]
    f = _dense_copy(a)
    piv = torch.zeros(n, dtype=torch.int32, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.call(f"nmx_getrf_{_SUF[a.dtype]}", _ctx(dev), n, f.data_ptr(), f.stride(0) if n else 1,
              piv.data_ptr(), info.data_ptr(), _stream(dev))
    host = piv.cpu()
    torch.cuda.current_stream(dev).synchronize()
    sign = 1
    if n:
        swaps = int((host != torch.arange(n, dtype=torch.int32)).sum().item())
        sign = -1 if swaps % 2 else 1
    return LU(f, piv, sign, int(info.item()))


def solve(a, b):
    """x with a x = b (numax/linalg/basic.mojo:55-146)."""
    return lu_factor(a).solve(b)


def lu(a):
    """(P, L, U) with a = P L U (numax/linalg/lu.mojo:877-975)."""
    return lu_factor(a).plu()


def inverse(a):
    """a^-1 by one LU and one solve against the identity
    (numax/linalg/basic.mojo:149-192); a singular a gives non-finite
    entries, not an error."""
    _check_matrix("a", a)
    dev = _resolve_device(a.device)
    n = a.shape[0]
    x = torch.empty((n, n), dtype=a.dtype, device=dev)
    piv = torch.zeros(max(n, 1), dtype=torch.int32, device=dev)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    if n:
        A = a.contiguous()
        _lib.call(f"nmx_inverse_{_SUF[a.dtype]}", _ctx(dev), n, A.data_ptr(), A.stride(0),
                  x.data_ptr(), x.stride(0), piv.data_ptr(), info.data_ptr(), _stream(dev))
    torch.cuda.current_stream(dev).synchronize()
    return x


def det(a):
    return lu_factor(a).det()


def slogdet(a):
    return lu_factor(a).slogdet()


def cholesky(a):
    """The lower-triangular L with L L^T = a, upper triangle zero
    (numax/linalg/cholesky.mojo:233-396).  Reads only a's lower triangle.

    Raises numax's error when a is not positive definite: the factorization
    runs to the end with the failing pivots floored, then reports the first."""
    _check_matrix("a", a)
    dev = _resolve_device(a.device)
    n = a.shape[0]
    l = _dense_copy(a)
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.call(f"nmx_potrf_{_SUF[a.dtype]}", _ctx(dev), n, l.data_ptr(), l.stride(0) if n else 1,
              info.data_ptr(), _stream(dev))
    flag = int(info.item())
    if flag != 0:
        raise ValueError("cholesky: matrix is not positive definite (non-positive pivot at index "
                         f"{flag - 1})")
    return l


def cholesky_solve(lower, b):
    """x with (L L^T) x = b from cholesky's L (numax/linalg/cholesky.mojo:471-580)."""
    _check_matrix("lower", lower)
    n = lower.shape[0]
    x = _as_rhs(b, n, lower.dtype, lower.device)
    L = lower.contiguous()
    if n:
        _lib.call(f"nmx_potrs_{_SUF[lower.dtype]}", _ctx(lower.device), n, x.shape[1], L.data_ptr(),
                  L.stride(0), x.data_ptr(), x.shape[1], _stream(lower.device))
    torch.cuda.current_stream(lower.device).synchronize()
    return x.reshape(b.shape)


class QR:
    """A blocked Householder QR (numax's `QR`, numax/linalg/qr.mojo:330-612):
    `factored` in LAPACK's packed form plus `taus`."""

    def __init__(self, factored, taus):
        self.factored = factored
        self.taus = taus
        self.m, self.n = factored.shape

    def r(self):
        """The n x n upper-triangular R (numax/linalg/qr.mojo:371-403)."""
        return torch.triu(self.factored[: self.n, : self.n]).contiguous()

    def q(self):
        """The thin m x n Q with orthonormal columns (numax/linalg/qr.mojo:405-468)."""
        f = self.factored
        q = torch.empty((self.m, self.n), dtype=f.dtype, device=f.device)
        if self.n:
            _lib.call(f"nmx_orgqr_{_SUF[f.dtype]}", _ctx(f.device), self.m, self.n, f.data_ptr(),
                      f.stride(0), self.taus.data_ptr(), q.data_ptr(), q.stride(0), _stream(f.device))
        torch.cuda.current_stream(f.device).synchronize()
        return q

    def apply_q_transpose(self, b):
        """Q^T b against the full Q, without forming it (m x k result; its
        leading n rows are the thin product) -- numax/linalg/qr.mojo:470-530."""
        f = self.factored
        x = _as_rhs(b, self.m, f.dtype, f.device)
        if self.n and x.shape[1]:
            _lib.call(f"nmx_ormqr_{_SUF[f.dtype]}", _ctx(f.device), self.m, self.n, f.data_ptr(),
                      f.stride(0), self.taus.data_ptr(), x.data_ptr(), x.stride(0), x.shape[1],
                      _stream(f.device))
        torch.cuda.current_stream(f.device).synchronize()
        return x.reshape(b.shape)

    def solve(self, b):
        """The least-squares x minimizing ||A x - b|| for a vector b
        (numax/linalg/qr.mojo:532-612): Q^T b, then R's back substitution."""
        f = self.factored
        if b.dim() != 1:
            raise ValueError("QR.solve takes a vector b")
        bb = _as_rhs(b, self.m, f.dtype, f.device).reshape(self.m)
        x = torch.empty(self.n, dtype=f.dtype, device=f.device)
        work = torch.empty(self.m, dtype=f.dtype, device=f.device)
        if self.n:
            _lib.call(f"nmx_qr_solve_{_SUF[f.dtype]}", _ctx(f.device), self.m, self.n,
                      f.data_ptr(), f.stride(0), self.taus.data_ptr(), bb.data_ptr(),
                      x.data_ptr(), work.data_ptr(), _stream(f.device))
        torch.cuda.current_stream(f.device).synchronize()
        return x


def lstsq(a, b):
    """The least-squares solution of a x ~= b (m >= n) through qr_factor and
    QR.solve (numax's lstsq over the Tensor tier, numax/linalg/qr.mojo:746)."""
    return qr_factor(a).solve(b)


def qr_factor(a) -> QR:
    """Householder QR of an m x n matrix with m >= n (numax/linalg/qr.mojo:615-743)."""
    _check_matrix("a", a, square=False)
    m, n = a.shape
    if m < n:
        raise ValueError(f"qr_factor needs m >= n, got {m} x {n}")
    dev = _resolve_device(a.device)
    f = _dense_copy(a)
    tau = torch.zeros(n, dtype=a.dtype, device=dev)
    if n:
        _lib.call(f"nmx_geqrf_{_SUF[a.dtype]}", _ctx(dev), m, n, f.data_ptr(), f.stride(0),
                  tau.data_ptr(), _stream(dev))
    torch.cuda.current_stream(dev).synchronize()
    return QR(f, tau)


_IR_MODES = {name: code for code, name in _lib.IR_PRECISION_NAMES.items()}


def solve_ir(a, b, precision: str = "bf16", gmres: bool | str = "auto", tol: float = 1e-14,
             max_iter: int = 50, escalate: bool = False, spd: bool = False):
    """x with a x = b for float64 a, b: low-precision LU (BF16/FP16 tensor-core
    trailing updates, BF16 splits with ~16 ("bf16x3") or 24 ("bf16x6") bits,
    FP32, or FP64) refined in FP64 to backward error <= tol, with GMRES-IR
    when `gmres` is True (or "auto": when plain refinement stalls); with
    `escalate`, a precision whose refinement cannot converge is replaced by
    the next more accurate one.  x is the iterate with the smallest backward
    error.  With `spd` (a symmetric positive definite, both triangles
    holding it) the factors are Cholesky's instead of LU's.

    Returns (x, stats) with stats a dict: iterations, gmres_iterations,
    converged, info, used_gmres, final_precision (name), backward_error,
    factor_ms, refine_ms."""
    _check_matrix("a", a)
    if a.dtype != torch.float64:
        raise TypeError("solve_ir needs float64 a and b")
    dev = _resolve_device(a.device)
    n = a.shape[0]
    A = a.contiguous()
    bb = _as_rhs(b, n, torch.float64, a.device).reshape(n)
    x = torch.empty(n, dtype=torch.float64, device=dev)
    mode = _IR_MODES[precision]
    if gmres is True:
        mode |= _lib.NMX_IR_GMRES
    elif gmres == "auto":
        mode |= _lib.NMX_IR_AUTO
    if escalate:
        mode |= _lib.NMX_IR_ESCALATE
    st = _lib.IrStats()
    import ctypes as _C
    _lib.call("nmx_posv_ir_f64" if spd else "nmx_gesv_ir_f64", _ctx(dev), n, A.data_ptr(),
              A.stride(0), bb.data_ptr(),
              x.data_ptr(), mode, float(tol), int(max_iter), _C.byref(st), _stream(dev))
    stats = {f: getattr(st, f) for f, _ in _lib.IrStats._fields_}
    stats["final_precision"] = _lib.IR_PRECISION_NAMES.get(st.final_precision, "?")
    return x.reshape(b.shape), stats


class Eigh:
    """eigh's result (numax's `Eigh`, numax/linalg/eigen.mojo:1220-1246):
    `values` ascending, `vectors` orthonormal with `vectors[:, j]` the
    eigenvector of `values[j]`."""

    def __init__(self, values, vectors):
        self.values = values
        self.vectors = vectors

    def __iter__(self):
        return iter((self.values, self.vectors))


def _syevd(name, a, vectors):
    _check_matrix(name, a, square=False)
    n, m = a.shape
    if m != n:
        raise ValueError(f"{name}: the matrix must be square, got {n} x {m}")
    if n < 1:
        raise ValueError(f"{name}: the matrix is empty")
    if a.stride(1) != 1:
        a = a.contiguous()
    dev = a.device
    w = torch.empty(n, dtype=a.dtype, device=dev)
    v = torch.empty(n, n, dtype=a.dtype, device=dev) if vectors else None
    info = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.call(f"nmx_syevd_{_SUF[a.dtype]}", _ctx(dev), n, a.data_ptr(), a.stride(0), w.data_ptr(),
              v.data_ptr() if vectors else None, n, info.data_ptr(), _stream(dev))
    if int(info.item()):
        raise ValueError(f"{name}: an eigenvalue did not converge -- the matrix holds a NaN or "
                         "an infinity")
    return w, v


def eigh(a) -> Eigh:
    """Eigenvalues (ascending) and orthonormal eigenvectors (columns) of the
    symmetric `a`, reading only its lower triangle (numax's Tensor-tier eigh,
    numax/linalg/eigen.mojo:1268-1341): tridiagonalization, divide and
    conquer and the back-transform all on the device (nmx_syevd_*)."""
    w, v = _syevd("eigh", a, True)
    return Eigh(w, v)


def eigvalsh(a):
    """The eigenvalues of the symmetric `a`, ascending, lower triangle read
    (numax's eigvalsh): tridiagonalization and bisection on the device."""
    return _syevd("eigvalsh", a, False)[0]
