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
# updates (bf16x3 through 1e5, bf16x6 through 1e8), and single-BF16 factors
# at 1e8 when escalation may move to more accurate factors.
@pytest.mark.parametrize("precision,gmres,kappa,escalate", [
    ("bf16", "auto", 1e2, False), ("fp16", "auto", 1e2, False), ("fp16", True, 1e5, False),
    ("fp32", "auto", 1e5, False), ("fp32", True, 1e8, False), ("bf16x3", "auto", 1e2, False),
    ("bf16x3", "auto", 1e5, False), ("bf16x6", "auto", 1e5, False), ("bf16x6", True, 1e8, False),
    ("bf16", False, 1e8, True), ("fp64", False, 1e8, False),
])
def test_ir_reaches_fp64_backward_error(precision, gmres, kappa, escalate):
    from numax_b200 import linalg
    n = 1000
    a, b, xt = make_system(n, kappa, seed=int(np.log10(kappa)))
    x, st = linalg.solve_ir(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(),
                            precision=precision, gmres=gmres, tol=1e-14, max_iter=60,
                            escalate=escalate)
    x = x.cpu().numpy()
    assert st["converged"] == 1, st
    assert berr(a, x, b) <= 1e-14, (berr(a, x, b), st)
    xr = np.linalg.solve(a, b)
    fe = np.abs(x - xr).max() / np.abs(xr).max()
    assert fe <= kappa * 1e-13, fe
    if not escalate:
        assert st["final_precision"] == precision


def _haar_gpu(n, gen):
    g = torch.randn((n, n), generator=gen, dtype=torch.float64, device="cuda")
    q, r = torch.linalg.qr(g)
    return q * torch.sign(torch.diagonal(r))[None, :]


@pytest.fixture(scope="module")
def system_8192():
    """A = U diag(s) V^T at n = 8192 (Haar U, V on the GPU), per kappa."""
    n = 8192
    gen = torch.Generator(device="cuda")
    gen.manual_seed(8192)
    u, v = _haar_gpu(n, gen), _haar_gpu(n, gen)
    xt = torch.randn(n, generator=gen, dtype=torch.float64, device="cuda")
    cache = {}

    def get(kappa):
        if kappa not in cache:
            s = torch.logspace(0.0, -np.log10(kappa), n, dtype=torch.float64, device="cuda")
            a = (u * s[None, :]) @ v.T
            cache.clear()
            cache[kappa] = (a, a @ xt)
        return cache[kappa]
    return get


def _berr_gpu(a, x, b):
    r = b - a @ x
    return float(r.abs().max() / (a.abs().sum(1).max() * x.abs().max() + b.abs().max()))


# The BASELINE conditioning range at n = 8192: every case must end at FP64
# backward error; with escalation the solver may move to more accurate
# factors, and reports which it finished with.
@pytest.mark.parametrize("kappa,precision,gmres,escalate", [
    (1e2, "bf16x3", "auto", False), (1e2, "fp16", "auto", False), (1e2, "bf16", "auto", True),
    (1e5, "bf16x6", "auto", False), (1e5, "bf16x3", "auto", True),
    (1e8, "bf16x6", "auto", True), (1e8, "fp16", "auto", True),
])
def test_ir_8192_across_conditioning(system_8192, kappa, precision, gmres, escalate):
    from numax_b200 import linalg
    a, b = system_8192(kappa)
    x, st = linalg.solve_ir(a, b, precision=precision, gmres=gmres, tol=1e-14, max_iter=80,
                            escalate=escalate)
    assert st["converged"] == 1, st
    be = _berr_gpu(a, x, b)
    assert be <= 1e-14, (be, st)
    # Against the FP64 LU solve of the same system (cuSOLVER, for data only).
    xr = torch.linalg.solve(a, b)
    fe = float((x - xr).abs().max() / xr.abs().max())
    assert fe <= kappa * 1e-12, (fe, st)


def test_ir_returns_its_best_iterate():
    """Single-BF16 factors at kappa 1e8 without escalation cannot converge:
    the solver stops and returns the iterate whose backward error it reports
    (never a later, worse one)."""
    from numax_b200 import linalg
    n = 1000
    a, b, _ = make_system(n, 1e8, seed=8)
    x, st = linalg.solve_ir(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(),
                            precision="bf16", gmres=False, tol=1e-14, max_iter=12)
    x = x.cpu().numpy()
    assert st["converged"] == 0
    assert np.all(np.isfinite(x))
    got = berr(a, x, b)
    assert got <= 1.0001 * st["backward_error"] + 1e-300, (got, st)
    # It is no worse than x = 0 (backward error 1).
    assert got < 1.0


def test_ir_rejects_bad_arguments():
    from numax_b200 import _lib
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    assert lib.nmx_gesv_ir_f64(ctx, 0, None, 1, None, None, 1, 1e-14, 10, None, None) == -2
    a = torch.eye(4, dtype=torch.float64, device="cuda")
    assert lib.nmx_gesv_ir_f64(ctx, 4, a.data_ptr(), 4, a.data_ptr(), a.data_ptr(), 9, 1e-14, 10,
                               None, None) == -7
    assert lib.nmx_gesv_ir_reserve(ctx, 0, 1) == -2
    assert lib.nmx_gesv_ir_reserve(ctx, 64, 0) == -3
    assert lib.nmx_gesv_ir_reserve(ctx, 64, 1 | 0x40) == 0


def make_spd(n, kappa, seed):
    """A = U diag(s) U^T (Haar U, s geometric 1 .. 1/kappa): symmetric positive
    definite with condition number kappa."""
    rng = np.random.Generator(np.random.PCG64(seed))
    u = haar(n, rng)
    s = np.geomspace(1.0, 1.0 / kappa, n)
    a = (u * s) @ u.T
    a = (a + a.T) / 2
    x = rng.standard_normal(n)
    return a, a @ x


@pytest.mark.parametrize("precision,gmres,kappa,escalate", [
    ("bf16x3", "auto", 1e2, False), ("fp16", "auto", 1e2, False), ("bf16", "auto", 1e2, True),
    ("bf16x6", "auto", 1e5, False), ("fp32", "auto", 1e5, False), ("bf16x6", True, 1e8, False),
    ("bf16", False, 1e8, True), ("fp64", False, 1e8, False),
])
def test_spd_ir_reaches_fp64_backward_error(precision, gmres, kappa, escalate):
    """Cholesky factors (tensor-core SYRK / triangular-solve products) with
    FP64 refinement: FP64 backward error, forward error within the
    conditioning, against LAPACK's FP64 solve."""
    from numax_b200 import linalg
    n = 1000
    a, b = make_spd(n, kappa, seed=7 + int(np.log10(kappa)))
    x, st = linalg.solve_ir(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(),
                            precision=precision, gmres=gmres, tol=1e-14, max_iter=60,
                            escalate=escalate, spd=True)
    x = x.cpu().numpy()
    assert st["converged"] == 1, st
    assert berr(a, x, b) <= 1e-14, (berr(a, x, b), st)
    xr = np.linalg.solve(a, b)
    assert np.abs(x - xr).max() / np.abs(xr).max() <= kappa * 1e-13
    if not escalate:
        assert st["final_precision"] == precision


@pytest.mark.parametrize("kappa,precision,escalate", [
    (1e2, "bf16x3", False), (1e2, "fp16", False), (1e5, "bf16x6", False), (1e8, "bf16x6", True),
])
def test_spd_ir_8192(kappa, precision, escalate):
    """The SPD solve at n = 8192 (U diag(s) U^T, U Haar on the GPU)."""
    from numax_b200 import linalg
    n = 8192
    gen = torch.Generator(device="cuda")
    gen.manual_seed(4096 + int(np.log10(kappa)))
    u = _haar_gpu(n, gen)
    s = torch.logspace(0.0, -np.log10(kappa), n, dtype=torch.float64, device="cuda")
    a = (u * s[None, :]) @ u.T
    a = (a + a.T) / 2
    del u
    xt = torch.randn(n, generator=gen, dtype=torch.float64, device="cuda")
    b = a @ xt
    x, st = linalg.solve_ir(a, b, precision=precision, gmres="auto", tol=1e-14, max_iter=80,
                            escalate=escalate, spd=True)
    assert st["converged"] == 1, st
    assert _berr_gpu(a, x, b) <= 1e-14, st
    xr = torch.linalg.solve(a, b)
    assert float((x - xr).abs().max() / xr.abs().max()) <= kappa * 1e-12, st


def test_spd_ir_gram_matrix_and_not_spd():
    """The BASELINE SPD family G G^T / n + I solves at BF16X3; a matrix that
    is not positive definite does not converge and reports so (it never
    returns a blown-up x)."""
    from numax_b200 import linalg
    n = 2000
    rng = np.random.Generator(np.random.PCG64(2000))
    g = rng.standard_normal((n, n))
    a = g @ g.T / n + np.eye(n)
    b = rng.standard_normal(n)
    x, st = linalg.solve_ir(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(),
                            precision="bf16x3", tol=1e-14, spd=True)
    assert st["converged"] == 1 and berr(a, x.cpu().numpy(), b) <= 1e-14, st
    a2 = a - 3.0 * np.eye(n)  # indefinite
    x2, st2 = linalg.solve_ir(torch.from_numpy(a2).cuda(), torch.from_numpy(b).cuda(),
                              precision="bf16x3", tol=1e-14, spd=True, max_iter=10)
    assert st2["converged"] == 0
    assert np.all(np.isfinite(x2.cpu().numpy())) or st2["backward_error"] != st2["backward_error"]
