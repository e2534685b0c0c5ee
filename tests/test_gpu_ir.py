"""Mixed-precision LU with iterative refinement (no numax counterpart): the
solution must reach FP64-level normwise backward error (<= 1e-14) and agree
with the FP64 LU solve (the oracle here is LAPACK's FP64 solve) to within
the conditioning, for A = U diag(s) V^T with Haar U, V and geometric s."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def haar(n, rng):
    q, r = np.linalg.qr(rng.standard_normal((n, n)))
    return q * np.sign(np.diag(r))


def make_system(n, kappa, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    u, v = haar(n, rng), haar(n, rng)
    s = np.geomspace(1.0, 1.0 / kappa, n)
    a = (u * s) @ v.T
    x = rng.standard_normal(n)
    return a, a @ x, x


def berr(a, x, b):
    return np.abs(b - a @ x).max() / (np.abs(a).sum(1).max() * np.abs(x).max() + np.abs(b).max())


# Converging cases: 16-bit factors with plain/auto refinement at kappa 1e2,
# FP16 factors with GMRES-IR at 1e5, FP32 factors through 1e8, split-BF16
# (bf16x3) updates through 1e5.  Single-BF16 factors at kappa >= 1e5 are
# reported by the benchmark, not asserted here.
@pytest.mark.parametrize("precision,gmres,kappa", [
    ("bf16", "auto", 1e2), ("fp16", "auto", 1e2), ("fp16", True, 1e5),
    ("fp32", "auto", 1e5), ("fp32", True, 1e8), ("bf16x3", "auto", 1e2), ("bf16x3", "auto", 1e5),
])
def test_ir_reaches_fp64_backward_error(precision, gmres, kappa):
    from numax_b200 import linalg
    n = 1000
    a, b, xt = make_system(n, kappa, seed=int(np.log10(kappa)))
    x, st = linalg.solve_ir(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(),
                            precision=precision, gmres=gmres, tol=1e-14, max_iter=60)
    x = x.cpu().numpy()
    assert st["converged"] == 1, st
    assert berr(a, x, b) <= 1e-14, (berr(a, x, b), st)
    xr = np.linalg.solve(a, b)
    fe = np.abs(x - xr).max() / np.abs(xr).max()
    assert fe <= kappa * 1e-13, fe


def test_ir_rejects_bad_arguments():
    from numax_b200 import _lib
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    assert lib.nmx_gesv_ir_f64(ctx, 0, None, 1, None, None, 1, 1e-14, 10, None, None) == -2
    a = torch.eye(4, dtype=torch.float64, device="cuda")
    assert lib.nmx_gesv_ir_f64(ctx, 4, a.data_ptr(), 4, a.data_ptr(), a.data_ptr(), 9, 1e-14, 10,
                               None, None) == -7
