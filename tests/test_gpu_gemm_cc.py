"""The dense factorizations' own GEMM (FP64 on DMMA, FP32 on the CUDA cores)
through the C ABI, against a plain PyTorch FP64 product of the same op:
C = alpha op(A) op(B) + beta C, row-major with leading dimensions, every
transpose combination, the lower-triangle (SYRK) mode, beta = 0 never
reading C, ragged sizes around the tile edges.

Tolerances: FP64 1e-13 normwise relative; FP32 2e-6 normwise relative
(FP32 accumulation over k <= 1000 against an FP64 reference)."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1, 1), (7, 13, 5), (64, 64, 16), (129, 257, 33), (300, 70, 1000), (1000, 1000, 256),
          (33, 2000, 17), (5000, 16, 200)]


def _call(dtype, ta, tb, m, n, k, alpha, A, B, beta, Cm, lower):
    from numax_b200 import _lib
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    fn = lib.nmx_gemm_f64 if dtype == torch.float64 else lib.nmx_gemm_f32
    rc = fn(ctx, int(ta), int(tb), m, n, k, alpha, C.c_void_p(A.data_ptr()), A.stride(0),
            C.c_void_p(B.data_ptr()), B.stride(0), beta, C.c_void_p(Cm.data_ptr()), Cm.stride(0),
            int(lower), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, _lib.last_error()


def _operands(dtype, ta, tb, m, n, k, seed, pad=3):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    # Strided operands: each lives in a wider buffer (ld = cols + pad).
    ar, ac = (k, m) if ta else (m, k)
    br, bc = (n, k) if tb else (k, n)
    A = torch.randn((ar, ac + pad), generator=g, dtype=torch.float64, device="cuda")[:, :ac]
    B = torch.randn((br, bc + pad), generator=g, dtype=torch.float64, device="cuda")[:, :bc]
    Cm = torch.randn((m, n + pad), generator=g, dtype=torch.float64, device="cuda")[:, :n]
    return A.to(dtype), B.to(dtype), Cm.to(dtype)


def _rel(got, want):
    return float((got - want).norm() / max(float(want.norm()), 1e-300))


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("ta,tb", [(False, False), (False, True), (True, False), (True, True)])
@pytest.mark.parametrize("m,n,k", SHAPES)
def test_gemm_matches_fp64_reference(dtype, ta, tb, m, n, k):
    A, B, Cm = _operands(dtype, ta, tb, m, n, k, seed=m * 31 + n * 7 + k)
    opA = A.double().T if ta else A.double()
    opB = B.double().T if tb else B.double()
    alpha, beta = -1.0, 1.0
    want = alpha * (opA @ opB) + beta * Cm.double()
    out = Cm.clone()
    _call(dtype, ta, tb, m, n, k, alpha, A, B, beta, out, False)
    torch.cuda.synchronize()
    tol = 1e-13 if dtype == torch.float64 else 2e-6
    assert _rel(out.double(), want) <= tol


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_gemm_beta_zero_never_reads_c_and_scales(dtype):
    m, n, k = 200, 150, 40
    A, B, _ = _operands(dtype, False, False, m, n, k, seed=5)
    out = torch.full((m, n), float("nan"), dtype=dtype, device="cuda")
    _call(dtype, False, False, m, n, k, 2.5, A, B, 0.0, out, False)
    torch.cuda.synchronize()
    want = 2.5 * (A.double() @ B.double())
    tol = 1e-13 if dtype == torch.float64 else 2e-6
    assert _rel(out.double(), want) <= tol
    # k = 0: C = beta C.
    c0 = torch.randn((m, n), dtype=dtype, device="cuda")
    out = c0.clone()
    _call(dtype, False, False, m, n, 0, 1.0, A, B, 0.5, out, False)
    torch.cuda.synchronize()
    assert torch.equal(out, 0.5 * c0)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("n,k", [(1, 3), (100, 64), (300, 256), (1100, 128)])
def test_gemm_lower_triangle_syrk(dtype, n, k):
    """C -= A A^T on the lower triangle only; the strict upper triangle is left
    bit-for-bit untouched."""
    A, _, Cm = _operands(dtype, False, True, n, n, k, seed=n + k)
    out = Cm.clone()
    _call(dtype, False, True, n, n, k, -1.0, A, A, 1.0, out, True)
    torch.cuda.synchronize()
    want = Cm.double() - A.double() @ A.double().T
    lo = torch.tril(torch.ones(n, n, dtype=torch.bool, device="cuda"))
    tol = 1e-13 if dtype == torch.float64 else 2e-6
    assert _rel(out.double()[lo], want[lo]) <= tol
    assert torch.equal(out[~lo], Cm[~lo])


def test_gemm_rejects_bad_arguments():
    from numax_b200 import _lib
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    assert lib.nmx_gemm_f64(None, 0, 0, 1, 1, 1, 1.0, None, 1, None, 1, 0.0, None, 1, 0, None) == -1
    assert lib.nmx_gemm_f64(ctx, 0, 0, 4, 4, 4, 1.0, None, 3, None, 4, 0.0, None, 4, 0, None) == -9
    assert lib.nmx_gemm_f32(ctx, 0, 0, 4, 4, 4, 1.0, None, 4, None, 4, 0.0, None, 3, 0, None) == -14
