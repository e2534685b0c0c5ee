"""The tensor-core trailing update (tcgen05, BF16/FP16 inputs, FP32
accumulate) against an FP64 product of the same rounded inputs: normwise
relative error within 1e-5 (FP32 accumulation), on ragged shapes and
strided operands."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (300, 200, 96), (1000, 513, 257), (37, 64, 16)])
def test_gemm_sub_tc(prec, m, n, k):
    from numax_b200 import _lib
    g = torch.Generator(device="cuda")
    g.manual_seed(m * 31 + n * 7 + k)
    lda, ldb, ldc = k + 5, n + 3, (n + 7) // 8 * 8 + 8
    A = torch.randn((m, lda), generator=g, device="cuda", dtype=torch.float32)
    B = torch.randn((k, ldb), generator=g, device="cuda", dtype=torch.float32)
    C = torch.randn((m, ldc), generator=g, device="cuda", dtype=torch.float32)
    dt = torch.bfloat16 if prec == 1 else torch.float16
    want = C[:, :n].double() - A[:, :k].to(dt).double() @ B[:, :n].to(dt).double()
    rc = _lib.load().nmx_gemm_sub_f32(_lib.context(0), m, n, k, A.data_ptr(), lda, B.data_ptr(),
                                       ldb, C.data_ptr(), ldc, prec,
                                       torch.cuda.current_stream().cuda_stream)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    err = float((C[:, :n].double() - want).norm() / want.norm())
    assert err <= 1e-5, err


@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (1000, 513, 257), (37, 64, 16)])
def test_gemm_sub_bf16x3_reaches_fp32_level(m, n, k):
    """Precision 3 (BF16 hi/lo splits, hi*hi + hi*lo + lo*hi) against the
    FP64 product of the unrounded FP32 operands: the dropped lo*lo term and
    the FP32 accumulation leave about 1e-5 relative at most, where one BF16
    rounding of the operands alone costs ~3e-3."""
    from numax_b200 import _lib
    g = torch.Generator(device="cuda")
    g.manual_seed(m * 13 + n * 5 + k)
    lda, ldb, ldc = k + 3, n + 1, (n + 7) // 8 * 8
    A = torch.randn((m, lda), generator=g, device="cuda", dtype=torch.float32)
    B = torch.randn((k, ldb), generator=g, device="cuda", dtype=torch.float32)
    C = torch.randn((m, ldc), generator=g, device="cuda", dtype=torch.float32)
    prod = A[:, :k].double() @ B[:, :n].double()
    want = C[:, :n].double() - prod
    rc = _lib.load().nmx_gemm_sub_f32(_lib.context(0), m, n, k, A.data_ptr(), lda, B.data_ptr(),
                                       ldb, C.data_ptr(), ldc, 3,
                                       torch.cuda.current_stream().cuda_stream)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    err = float((C[:, :n].double() - want).norm() / prod.norm())
    assert err <= 2e-5, err
    one = float(((A[:, :k].bfloat16().double() @ B[:, :n].bfloat16().double()) - prod).norm()
                / prod.norm())
    assert err < one / 20, (err, one)


@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (1000, 513, 257), (37, 64, 16)])
def test_gemm_sub_bf16x6_reaches_fp32_accumulation(m, n, k):
    """Precision 4 (BF16 hi/mid/lo splits, six products) against the FP64
    product of the FP32 operands: what is left is the tensor cores' FP32
    accumulation (a few 1e-6 relative over 6 K terms), below BF16X3's error
    from its dropped lo*lo term."""
    from numax_b200 import _lib
    g = torch.Generator(device="cuda")
    g.manual_seed(m * 17 + n * 3 + k)
    lda, ldb, ldc = k + 3, n + 1, (n + 7) // 8 * 8
    A = torch.randn((m, lda), generator=g, device="cuda", dtype=torch.float32)
    B = torch.randn((k, ldb), generator=g, device="cuda", dtype=torch.float32)
    C = torch.randn((m, ldc), generator=g, device="cuda", dtype=torch.float32)
    prod = A[:, :k].double() @ B[:, :n].double()
    want = C[:, :n].double() - prod
    rc = _lib.load().nmx_gemm_sub_f32(_lib.context(0), m, n, k, A.data_ptr(), lda, B.data_ptr(),
                                       ldb, C.data_ptr(), ldc, 4,
                                       torch.cuda.current_stream().cuda_stream)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    err = float((C[:, :n].double() - want).norm() / prod.norm())
    assert err <= 6e-6, err
    # The same update with BF16X3 operands is less accurate.
    C3 = C.clone()
    C3[:, :n] = (want + prod).float()
    rc = _lib.load().nmx_gemm_sub_f32(_lib.context(0), m, n, k, A.data_ptr(), lda, B.data_ptr(),
                                       ldb, C3.data_ptr(), ldc, 3,
                                       torch.cuda.current_stream().cuda_stream)
    assert rc == 0, _lib.last_error()
    torch.cuda.synchronize()
    err3 = float((C3[:, :n].double() - want).norm() / prod.norm())
    assert err < err3, (err, err3)
