"""Dense LU with partial pivoting and the LU solve on the GPU vs the oracle
(numax's lu_factor / LU.solve restated on the CPU) and LAPACK.

Bars (north star): pivots bit-exact; float64 factors and solutions within
1e-12 normwise relative; float32 within 1e-5."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d else 1.0))


def gpu_lu(a):
    from numax_b200 import linalg
    return linalg.lu_factor(torch.from_numpy(np.ascontiguousarray(a)).cuda())


def test_lu_numax_golden_plu():
    nx = np.load(os.path.join(GOLD, "numax_fixtures.npz"))
    from oracle import oracle as O
    f = gpu_lu(nx["lu_a"])
    p, l, u = O.plu(f.factored.cpu().numpy(), f.pivots.cpu().numpy())
    np.testing.assert_allclose(p, nx["lu_p"], atol=1e-14)
    np.testing.assert_allclose(l, nx["lu_l"], atol=1e-14)
    np.testing.assert_allclose(u, nx["lu_u"], atol=1e-14)
    assert f.sign == -1
    assert abs(f.det() - np.linalg.det(nx["lu_a"])) < 1e-12


def test_lu_exchange_matrix_and_pivot_row():
    nx = np.load(os.path.join(GOLD, "numax_fixtures.npz"))
    f = gpu_lu(nx["exchange"])
    assert abs(f.det() + 1.0) < 1e-12
    x = f.solve(torch.from_numpy(nx["exchange_b"]).cuda()).cpu().numpy()
    np.testing.assert_allclose(x, nx["exchange_x"], atol=1e-12)
    f = gpu_lu(nx["panel3"])
    assert int(f.pivots[0]) == 2


@pytest.mark.parametrize("n", [1, 2, 5, 31, 32, 33, 64, 65, 100, 257, 700])
def test_lu_matches_oracle_f64(oracle, n):
    rng = np.random.Generator(np.random.PCG64(1000 + n))
    a = rng.standard_normal((n, n))
    f = gpu_lu(a)
    lu, piv, sign, info = oracle.lu_factor(a, block=16, base=16)
    np.testing.assert_array_equal(f.pivots.cpu().numpy(), piv)
    assert f.sign == sign and f.info == info == 0
    assert rel(f.factored.cpu().numpy(), lu) <= 1e-12
    b = rng.standard_normal(n)
    bm = rng.standard_normal((n, 16))
    x = f.solve(torch.from_numpy(b).cuda()).cpu().numpy()
    xm = f.solve(torch.from_numpy(bm).cuda()).cpu().numpy()
    assert rel(x, oracle.lu_solve(lu, piv, b, block=16)) <= 1e-12
    assert rel(xm, oracle.lu_solve(lu, piv, bm, block=16)) <= 1e-12


def test_lu_matches_lapack_large():
    import scipy.linalg as sl
    n = 2048
    rng = np.random.Generator(np.random.PCG64(77))
    a = rng.standard_normal((n, n))
    f = gpu_lu(a)
    lu, piv = sl.lu_factor(a)
    np.testing.assert_array_equal(f.pivots.cpu().numpy(), piv)
    assert rel(f.factored.cpu().numpy(), lu) <= 1e-12
    b = rng.standard_normal((n, 16))
    x = f.solve(torch.from_numpy(b).cuda()).cpu().numpy()
    assert rel(x, sl.lu_solve((lu, piv), b)) <= 1e-12


@pytest.mark.parametrize("n", [7, 96, 300])
def test_lu_matches_oracle_f32(oracle, n):
    # Factors and pivots on a Gaussian matrix; solutions compared on a
    # well-conditioned one (a float32 solution's forward error scales with
    # cond(A) * 6e-8, so 1e-5 is only meaningful for cond(A) ~ 1), and by
    # normwise backward error on the Gaussian one.
    rng = np.random.Generator(np.random.PCG64(n))
    a = rng.standard_normal((n, n)).astype(np.float32)
    f = gpu_lu(a)
    lu, piv, sign, info = oracle.lu_factor(a, block=16, base=16)
    np.testing.assert_array_equal(f.pivots.cpu().numpy(), piv)
    assert rel(f.factored.cpu().numpy(), lu) <= 1e-5
    b = rng.standard_normal((n, 3)).astype(np.float32)
    x = f.solve(torch.from_numpy(b).cuda()).cpu().numpy().astype(np.float64)
    a64 = a.astype(np.float64)
    berr = np.abs(a64 @ x - b).max() / (np.abs(a64).sum(1).max() * np.abs(x).max() + np.abs(b).max())
    assert berr <= 1e-5
    w = (rng.standard_normal((n, n)) / np.sqrt(n) + 2 * np.eye(n)).astype(np.float32)
    g = gpu_lu(w)
    lw, pw, _, _ = oracle.lu_factor(w, block=16, base=16)
    xw = g.solve(torch.from_numpy(b).cuda()).cpu().numpy()
    assert rel(xw, oracle.lu_solve(lw, pw, b, block=16)) <= 1e-5


def test_lu_singular_reports_info_and_gives_nonfinite(oracle):
    a = np.random.Generator(np.random.PCG64(3)).standard_normal((6, 6))
    a[:, 2] = 0.0
    f = gpu_lu(a)
    _, piv, _, info = oracle.lu_factor(a, block=16)
    assert f.info == info == 3
    np.testing.assert_array_equal(f.pivots.cpu().numpy(), piv)
    x = f.solve(torch.ones(6, dtype=torch.float64, device="cuda")).cpu().numpy()
    assert not np.isfinite(x).all()


def test_lu_leading_dimension_and_argument_errors():
    from numax_b200 import _lib, linalg
    n = 40
    rng = np.random.Generator(np.random.PCG64(5))
    big = torch.from_numpy(rng.standard_normal((n, n + 9))).cuda()
    g = linalg.lu_factor(big[:, :n].contiguous())
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    piv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    # The C ABI factors the strided block in place (lda = n + 9).
    rc = lib.nmx_getrf_f64(ctx, n, big.data_ptr(), n + 9, piv.data_ptr(), info.data_ptr(),
                           torch.cuda.current_stream().cuda_stream)
    assert rc == 0
    torch.cuda.synchronize()
    np.testing.assert_array_equal(piv.cpu().numpy(), g.pivots.cpu().numpy())
    assert rel(big[:, :n].cpu().numpy(), g.factored.cpu().numpy()) <= 1e-12
    # The columns past the leading dimension's n are never touched.
    np.testing.assert_array_equal(big[:, n:].cpu().numpy(),
                                  np.random.Generator(np.random.PCG64(5)).standard_normal((n, n + 9))[:, n:])
    assert lib.nmx_getrf_f64(ctx, 4, None, 4, None, None, None) == -3
    assert lib.nmx_getrf_f64(ctx, 4, big.data_ptr(), 3, None, None, None) == -4


@pytest.mark.parametrize("cluster", [0, 2, -1])
def test_lu_leaf_paths_match_lapack(cluster):
    """The panel leaf runs as a thread-block cluster exchanging candidates
    through distributed shared memory, or as a cooperative grid exchanging
    through global memory ("lu.cluster" = 0).  A 2-CTA cluster holds only
    part of a 4000-row panel, which narrows the leaves to 8 and 16 columns
    near the top and leaves the tallest panels to the cooperative kernel, so
    every leaf form runs here; all must give LAPACK's pivots."""
    import scipy.linalg as sl
    from numax_b200 import _lib, linalg
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    n = 4000
    rng = np.random.Generator(np.random.PCG64(4000))
    a = rng.standard_normal((n, n))
    lib.nmx_tune_set(ctx, b"lu.cluster", cluster)
    try:
        f = linalg.lu_factor(torch.from_numpy(a).cuda())
    finally:
        lib.nmx_tune_set(ctx, b"lu.cluster", -1)
    lu, piv = sl.lu_factor(a)
    np.testing.assert_array_equal(f.pivots.cpu().numpy(), piv)
    assert f.info == 0
    assert rel(f.factored.cpu().numpy(), lu) <= 1e-12


# The look-ahead LU (panels on two streams, leaves' interchanges deferred as
# row-move lists): numax's pivots exactly, the factors to rounding.
@pytest.mark.parametrize("n,nb", [(700, 64), (1500, 256), (2100, 512)])
def test_lu_lookahead_matches_lapack(n, nb):
    import scipy.linalg as sl
    from numax_b200 import _lib
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    rng = np.random.Generator(np.random.PCG64(4000 + n))
    a = rng.standard_normal((n, n))
    lib.nmx_tune_set(ctx, b"lu.lookahead", nb)
    try:
        f = gpu_lu(a)
    finally:
        lib.nmx_tune_set(ctx, b"lu.lookahead", -1)
    lu, piv = sl.lu_factor(a)
    np.testing.assert_array_equal(f.pivots.cpu().numpy(), piv)
    assert rel(f.factored.cpu().numpy(), lu) <= 1e-12
    b = rng.standard_normal((n, 4))
    x = f.solve(torch.from_numpy(b).cuda()).cpu().numpy()
    berr = np.abs(b - a @ x).max() / (np.abs(a).sum(1).max() * np.abs(x).max())
    assert berr <= 1e-14, berr


def test_lu_config_order_8192_lookahead_matches_lapack():
    """The FP64 LU at a BASELINE order (8192: the default look-ahead path with
    cluster leaves): pivots bit-exact against LAPACK's, factors within 1e-12
    normwise.  The 16-right-hand-side solve is backward stable (normwise
    backward error <= 1e-14) and agrees with LAPACK's solve to the forward
    error its conditioning allows: two backward-stable solves differ by about
    kappa(A) u, which for a Gaussian matrix of this order is above 1e-12
    (kappa from LAPACK's own estimate, dgecon)."""
    import scipy.linalg as sl
    n = 8192
    rng = np.random.Generator(np.random.PCG64(8192))
    a = rng.standard_normal((n, n))
    f = gpu_lu(a)
    lu, piv = sl.lu_factor(a)
    got = f.pivots.cpu().numpy()
    first = np.flatnonzero(got != piv)
    assert first.size == 0, f"pivots differ first at column {first[0]}"
    assert rel(f.factored.cpu().numpy(), lu) <= 1e-12
    b = rng.standard_normal((n, 16))
    x = f.solve(torch.from_numpy(b).cuda()).cpu().numpy()
    berr = np.abs(b - a @ x).max() / (np.abs(a).sum(1).max() * np.abs(x).max() + np.abs(b).max())
    assert berr <= 1e-14, berr
    rcond, _ = sl.lapack.dgecon(lu, np.abs(a).sum(0).max(), norm="1")
    kappa = 1.0 / rcond
    assert rel(x, sl.lu_solve((lu, piv), b)) <= max(1e-12, 16 * np.finfo(float).eps * kappa)


@pytest.mark.parametrize("n", [1, 3, 33, 200, 1000])
def test_lu_det_slogdet_plu_on_device(oracle, n):
    """LU.det / LU.slogdet / lu -> (P, L, U) from the device entry points
    against the oracle's restatement of numax's (pivot parity x diagonal,
    sum of logs, interchanges replayed on the identity) and numpy."""
    from numax_b200 import linalg
    rng = np.random.Generator(np.random.PCG64(7000 + n))
    a = rng.standard_normal((n, n))
    f = gpu_lu(a)
    lu, piv, sign, info = oracle.lu_factor(a, block=16, base=16)
    s, lg = f.slogdet()
    ws, wl = np.linalg.slogdet(a)
    assert s == ws and abs(lg - wl) <= 1e-12 * max(1.0, abs(wl))
    if n <= 200:
        d = f.det()
        assert abs(d - oracle.det(lu, sign)) <= 1e-12 * abs(oracle.det(lu, sign))
    P, L, U = (t.cpu().numpy() for t in linalg.lu(torch.from_numpy(a).cuda()))
    p, l, u = oracle.plu(lu, piv)
    np.testing.assert_array_equal(P, p)
    assert rel(L, l) <= 1e-12 and rel(U, u) <= 1e-12
    assert np.abs(P @ L @ U - a).max() <= 1e-12 * np.abs(a).max() * n


def test_lu_det_slogdet_singular_and_golden():
    """A singular matrix gives (0, -inf) and det 0 (numax's convention); the
    exchange matrix's determinant is -1 (numax's fixture)."""
    from numax_b200 import linalg
    a = np.array([[1.0, 2.0, 3.0], [2.0, 4.0, 6.0], [1.0, 0.0, 1.0]])
    f = gpu_lu(a)
    assert f.slogdet() == (0.0, -np.inf)
    assert f.det() == 0.0
    nx = np.load(os.path.join(GOLD, "numax_fixtures.npz"))
    assert abs(linalg.det(torch.from_numpy(nx["exchange"]).cuda()) + 1.0) < 1e-12


@pytest.mark.parametrize("dtype,n", [(np.float64, 1), (np.float64, 5), (np.float64, 64),
                                     (np.float64, 257), (np.float64, 1500), (np.float32, 300)])
def test_inverse_matches_numpy(dtype, n):
    """numax's inverse (one LU, one solve against the identity): A A^-1 = I
    and agreement with numpy's inverse within the conditioning."""
    from numax_b200 import linalg
    rng = np.random.Generator(np.random.PCG64(8000 + n))
    a = (rng.standard_normal((n, n)) + n ** 0.5 * np.eye(n)).astype(dtype)
    x = linalg.inverse(torch.from_numpy(a).cuda()).cpu().numpy().astype(np.float64)
    a64 = a.astype(np.float64)
    tol = 1e-12 if dtype == np.float64 else 1e-4
    assert np.abs(a64 @ x - np.eye(n)).max() <= tol * n
    assert rel(x, np.linalg.inv(a64)) <= tol * 10


def test_inverse_singular_is_non_finite():
    from numax_b200 import linalg
    a = np.array([[1.0, 2.0], [2.0, 4.0]])
    x = linalg.inverse(torch.from_numpy(a).cuda()).cpu().numpy()
    assert not np.all(np.isfinite(x))
