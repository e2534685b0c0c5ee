"""Pins the CPU oracle (the checker for every GPU test) against numax's own
golden values and against LAPACK on seeded inputs.  CPU only."""
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def nx():
    return np.load(os.path.join(GOLD, "numax_fixtures.npz"))


@pytest.fixture(scope="module")
def lp():
    return np.load(os.path.join(GOLD, "lapack_fixtures.npz"))


def test_lu_matches_numax_scipy_golden(oracle, nx):
    # tests/linalg/test_lu_plu.mojo:44-109: SciPy's P, L, U at 1e-14.
    for block in (1, 2, 3, 4, 32):
        lu, piv, sign, info = oracle.lu_factor(nx["lu_a"], block=block, base=16)
        p, l, u = oracle.plu(lu, piv)
        np.testing.assert_allclose(p, nx["lu_p"], atol=1e-14)
        np.testing.assert_allclose(l, nx["lu_l"], atol=1e-14)
        np.testing.assert_allclose(u, nx["lu_u"], atol=1e-14)
        assert info == 0
        # tests/linalg/test_lu_plu.mojo:112-120: a 4-cycle, det(P) = -1.
        assert sign == -1
        np.testing.assert_allclose(oracle.det(lu, sign), np.linalg.det(nx["lu_a"]), atol=1e-12)


def test_exchange_matrix(oracle, nx):
    # tests/linalg/test_tensor_linalg.mojo:816-832
    lu, piv, sign, info = oracle.lu_factor(nx["exchange"], block=2)
    assert abs(oracle.det(lu, sign) - (-1.0)) < 1e-12
    x = oracle.lu_solve(lu, piv, nx["exchange_b"], block=2)
    np.testing.assert_allclose(x, nx["exchange_x"], atol=1e-12)


def test_panel_picks_largest_pivot(oracle, nx):
    # tests/linalg/test_panel.mojo:258-275
    _, piv, info = oracle.getrf_panel(nx["panel3"], 0, 1)
    assert piv[0] == 2 and info == 0


def test_getrf2_pivots_bit_equal_across_base(oracle):
    # tests/linalg/test_panel.mojo:366-460: n=12, nb=7 (prime), base 1..5.
    n = 12
    a = np.array([[((i * 7 + j * 3) % 11 + 1.0 + (n if i == j else 0)) * (1.0 + 0.25 * i)
                   for j in range(n)] for i in range(n)])
    want, want_p, _ = oracle.getrf2(a, 0, 7, 7)
    for base in (1, 2, 3, 4, 5):
        got, got_p, _ = oracle.getrf2(a, 0, 7, base)
        np.testing.assert_array_equal(got_p, want_p)
        np.testing.assert_allclose(got, want, atol=1e-10)


@pytest.mark.parametrize("n", [17, 64])
def test_lu_matches_lapack(oracle, lp, n):
    a = lp[f"lu{n}_a"]
    for block, base in ((32, 16), (16, 16), (5, 2)):
        lu, piv, sign, info = oracle.lu_factor(a, block=block, base=base)
        np.testing.assert_array_equal(piv, lp[f"lu{n}_piv"])
        assert np.linalg.norm(lu - lp[f"lu{n}_lu"]) <= 1e-12 * np.linalg.norm(lp[f"lu{n}_lu"])


def test_lu_solve_residual_and_block_invariance(oracle):
    # tests/linalg/test_tensor_linalg.mojo:744-896: residual <= 1e-12, block 1/2/4.
    rng = np.random.Generator(np.random.PCG64(7))
    n = 37
    a = rng.standard_normal((n, n))
    b = rng.standard_normal(n)
    bm = rng.standard_normal((n, 5))
    xs = []
    for block in (1, 2, 4, 32):
        lu, piv, _, _ = oracle.lu_factor(a, block=block)
        x = oracle.lu_solve(lu, piv, b, block=block)
        assert np.abs(a @ x - b).max() <= 1e-12 * np.abs(b).max() * n
        xm = oracle.lu_solve(lu, piv, bm, block=block)
        assert np.abs(a @ xm - bm).max() <= 1e-12 * np.abs(bm).max() * n
        xs.append(x)
    for x in xs[1:]:
        np.testing.assert_allclose(x, xs[0], rtol=1e-10, atol=1e-12)


def test_cholesky_matches_lapack_and_block_tile_invariance(oracle, lp):
    a = lp["chol40_a"]
    for block, tile in ((64, 128), (32, 40), (1, 3), (5, 7), (16, 16)):
        l, info = oracle.cholesky(a, block=block, tile=tile)
        assert info == 0
        assert np.allclose(np.triu(l, 1), 0)
        assert np.linalg.norm(l - lp["chol40_l"]) <= 1e-12 * np.linalg.norm(lp["chol40_l"])


def test_cholesky_reads_only_lower(oracle, nx):
    # tests/linalg/test_tensor_linalg.mojo:562-659: garbage above the diagonal is ignored.
    a = nx["spd5"].copy()
    want, _ = oracle.cholesky(a, block=2)
    a[np.triu_indices(5, 1)] = 1e6
    got, _ = oracle.cholesky(a, block=2)
    np.testing.assert_allclose(got, want, atol=0)


def test_cholesky_failure_index(oracle, nx):
    # tests/linalg/test_tensor_linalg.mojo:681-741: "index 3" (info 4) at block=2.
    _, info = oracle.cholesky(nx["later_block"], block=2)
    assert info - 1 == 3
    _, info = oracle.cholesky(nx["not_spd_2x2"], block=2)
    assert info > 0


def test_cholesky_solve(oracle, lp):
    a = lp["chol40_a"]
    l, _ = oracle.cholesky(a)
    rng = np.random.Generator(np.random.PCG64(3))
    b = rng.standard_normal(40)
    bm = rng.standard_normal((40, 16))
    x = oracle.cholesky_solve(l, b)
    xm = oracle.cholesky_solve(l, bm)
    np.testing.assert_allclose(a @ x, b, atol=1e-12)
    np.testing.assert_allclose(a @ xm, bm, atol=1e-12)
    np.testing.assert_allclose(xm[:, 0], oracle.cholesky_solve(l, bm[:, 0].copy()), atol=1e-13)


def test_qr_matches_lapack_packed_form(oracle, lp):
    a = lp["qr70_a"]
    for block in (16, 7, 40):
        f, tau = oracle.qr_factor(a, block=block)
        np.testing.assert_allclose(tau, lp["qr70_tau"], atol=1e-13)
        assert np.linalg.norm(f - lp["qr70_packed"]) <= 1e-12 * np.linalg.norm(f)
        q = oracle.qr_q(f, tau, block=block)
        r = oracle.qr_r(f)
        np.testing.assert_allclose(q @ r, a, atol=1e-12)
        np.testing.assert_allclose(q.T @ q, np.eye(40), atol=1e-13)


def test_array_cholesky_and_solve(oracle, nx):
    a = nx["spd5"]
    l = oracle.array_cholesky(a)
    np.testing.assert_allclose(l, np.linalg.cholesky(a), atol=1e-14)
    b = np.arange(5.0)
    x = oracle.array_cholesky_solve(l, b)
    np.testing.assert_allclose(a @ x, b, atol=1e-12)
    # Array tier floors an exactly-zero pivot and gives NaN for a negative one.
    z = oracle.array_cholesky(np.zeros((2, 2)))
    assert z[0, 0] == pytest.approx(1e-15)
    assert np.isnan(oracle.array_cholesky(nx["not_spd_2x2"])[1, 1])


def test_jacobi_eigh_invariants(oracle, nx, lp):
    # tests/linalg/test_linalg.mojo:576-645
    a = nx["spd3"]
    w, v = oracle.jacobi_eigh(a)
    assert abs(w.sum() - np.trace(a)) < 1e-12
    np.testing.assert_allclose(a @ v, v * w, atol=1e-12)
    np.testing.assert_allclose(v.T @ v, np.eye(3), atol=1e-12)
    assert (w > 0).all()
    w, _ = oracle.jacobi_eigh(np.diag([3.0, -1.0, 7.0]))
    assert sorted(w) == pytest.approx([-1.0, 3.0, 7.0], abs=1e-12)
    w, _ = oracle.jacobi_eigh(np.eye(3))
    np.testing.assert_allclose(w, 1.0, atol=1e-14)
    for key in ("eig24", "well24"):
        w, _ = oracle.jacobi_eigh(lp[f"{key}_a"])
        np.testing.assert_allclose(np.sort(w), lp[f"{key}_w"], atol=1e-10)


def test_batched_oracle_matches_per_matrix(oracle):
    rng = np.random.Generator(np.random.PCG64(11))
    ns = rng.integers(1, 129, size=40).astype(np.int32)
    mats = []
    for n in ns:
        g = rng.standard_normal((n, n))
        mats.append((g @ g.T / n + n * np.eye(n)).ravel())
    A = np.concatenate(mats)
    B = rng.standard_normal(int(ns.astype(np.int64).sum() * 4))
    L, X = oracle.batched_cholesky_solve(ns, A, B, 4)
    ao, bo = oracle.ragged_offsets(ns), oracle.ragged_offsets(ns, 4)
    for i, n in enumerate(ns):
        a = A[ao[i]:ao[i] + n * n].reshape(n, n)
        x = X[bo[i]:bo[i] + 4 * n].reshape(n, 4)
        b = B[bo[i]:bo[i] + 4 * n].reshape(n, 4)
        np.testing.assert_allclose(a @ x, b, atol=1e-10)
        np.testing.assert_allclose(np.tril(L[ao[i]:ao[i] + n * n].reshape(n, n)),
                                   np.linalg.cholesky(a), rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("n", [1, 2, 3, 10, 64, 150])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_eigh_matches_lapack(oracle, n, dtype):
    """numax's Tensor-tier eigh restated (sytrd, implicit QL, sort, Q Z)
    against LAPACK's syevd: values ascending, vectors orthonormal and
    satisfying A v = lambda v; only the lower triangle is read."""
    rng = np.random.Generator(np.random.PCG64(n))
    g = rng.standard_normal((n, n))
    a = ((g + g.T) / 2).astype(dtype)
    noisy = np.tril(a) + np.triu(rng.standard_normal((n, n)).astype(dtype), 1)
    w, v = oracle.eigh(noisy)
    want = np.linalg.eigvalsh(a.astype(np.float64))
    tol = 1e-13 if dtype == np.float64 else 2e-6
    scale = max(1.0, np.abs(want).max())
    assert np.abs(w - want).max() / scale < tol
    v64 = v.astype(np.float64)
    assert np.abs(a.astype(np.float64) @ v64 - v64 * w).max() / scale < 20 * tol
    assert np.abs(v64.T @ v64 - np.eye(n)).max() < 20 * tol
    w2, none = oracle.eigh(noisy, vectors=False)
    assert none is None and np.array_equal(w, w2)


def test_oracle_eigh_reports_nan():
    a = np.eye(4)
    a[2, 1] = np.nan
    with pytest.raises(ValueError, match="did not converge"):
        from oracle import oracle as O
        O.eigh(a)
