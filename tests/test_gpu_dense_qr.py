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
