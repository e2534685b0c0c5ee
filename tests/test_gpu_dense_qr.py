"""Householder QR on the GPU vs the oracle (numax's qr_factor / QR.q
restated) and LAPACK's packed form.  float32 within 1e-5 normwise (the
tall-skinny config is float32), float64 within 1e-12."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def rel(a, b):
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d else 1.0))


@pytest.mark.parametrize("m,n", [(1, 1), (17, 5), (70, 40), (300, 33), (1000, 64)])
def test_qr_matches_oracle_f64(oracle, m, n):
    from numax_b200 import linalg
    rng = np.random.Generator(np.random.PCG64(m * 7 + n))
    a = rng.standard_normal((m, n))
    f = linalg.qr_factor(torch.from_numpy(a).cuda())
    want, tau = oracle.qr_factor(a, block=16)
    assert rel(f.factored.cpu().numpy(), want) <= 1e-12
    assert rel(f.taus.cpu().numpy(), tau) <= 1e-12
    q = f.q().cpu().numpy()
    assert rel(q, oracle.qr_q(want, tau, block=16)) <= 1e-12
    r = f.r().cpu().numpy()
    assert np.abs(q @ r - a).max() <= 1e-12 * np.abs(a).max() * m
    assert np.abs(q.T @ q - np.eye(n)).max() <= 1e-12 * m


def test_qr_tall_skinny_f32_vs_lapack():
    import scipy.linalg as sl
    from numax_b200 import linalg
    m, n = 65536, 96
    rng = np.random.Generator(np.random.PCG64(1))
    a = rng.standard_normal((m, n)).astype(np.float32)
    f = linalg.qr_factor(torch.from_numpy(a).cuda())
    (packed, tau), _ = sl.qr(a.astype(np.float64), mode="raw")
    assert rel(f.factored.cpu().numpy().astype(np.float64), np.ascontiguousarray(packed)) <= 1e-5
    assert rel(f.taus.cpu().numpy().astype(np.float64), tau) <= 1e-5
    q = f.q().cpu().numpy().astype(np.float64)
    assert np.abs(q.T @ q - np.eye(n)).max() <= 1e-5


def test_qr_zero_column_keeps_tau_zero(oracle):
    from numax_b200 import linalg
    a = np.zeros((8, 3))
    a[:, 1] = np.arange(8.0)
    a[0, 2] = 5.0
    f = linalg.qr_factor(torch.from_numpy(a).cuda())
    want, tau = oracle.qr_factor(a, block=16)
    np.testing.assert_allclose(f.taus.cpu().numpy(), tau, atol=1e-15)
    assert rel(f.factored.cpu().numpy(), want) <= 1e-12


def test_qr_config_262144x256_f32_vs_lapack():
    """The BASELINE tall-skinny QR (262144 x 256, float32 Gaussian) against
    LAPACK's packed geqrf of the same data in float64: R/V and tau within
    1e-5 normwise, the thin Q orthogonal to 1e-5."""
    import scipy.linalg as sl
    from numax_b200 import linalg
    m, n = 262144, 256
    rng = np.random.Generator(np.random.PCG64(262144))
    a = rng.standard_normal((m, n)).astype(np.float32)
    f = linalg.qr_factor(torch.from_numpy(a).cuda())
    (packed, tau), _ = sl.qr(a.astype(np.float64), mode="raw")
    assert rel(f.factored.cpu().numpy().astype(np.float64), np.ascontiguousarray(packed)) <= 1e-5
    assert rel(f.taus.cpu().numpy().astype(np.float64), tau) <= 1e-5
    q = f.q().double()
    eye = torch.eye(n, dtype=torch.float64, device="cuda")
    assert float((q.T @ q - eye).abs().max()) <= 1e-5


@pytest.mark.parametrize("dtype,m,n,k", [(np.float64, 300, 33, 5), (np.float64, 2000, 100, 17),
                                         (np.float32, 4096, 64, 3), (np.float64, 40, 40, 1)])
def test_qr_apply_q_transpose_and_lstsq(dtype, m, n, k):
    """numax's QR.apply_q_transpose (Q^T B against the full Q, Q never formed)
    against LAPACK's full Q, and QR.solve / lstsq against numpy's
    least-squares solution."""
    import scipy.linalg as sl
    from numax_b200 import linalg
    rng = np.random.Generator(np.random.PCG64(m + 3 * n + k))
    a = rng.standard_normal((m, n)).astype(dtype)
    B = rng.standard_normal((m, k)).astype(dtype)
    f = linalg.qr_factor(torch.from_numpy(a).cuda())
    got = f.apply_q_transpose(torch.from_numpy(B).cuda()).cpu().numpy().astype(np.float64)
    qf, _ = sl.qr(a.astype(np.float64), mode="full")
    # Same reflectors (LAPACK's sign convention), so the full Q agrees.
    want = qf.T @ B.astype(np.float64)
    tol = 1e-12 if dtype == np.float64 else 2e-5
    assert rel(got, want) <= tol
    b = rng.standard_normal(m).astype(dtype)
    x = linalg.lstsq(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()).cpu().numpy()
    xr = np.linalg.lstsq(a.astype(np.float64), b.astype(np.float64), rcond=None)[0]
    assert rel(x.astype(np.float64), xr) <= (1e-11 if dtype == np.float64 else 1e-4)
