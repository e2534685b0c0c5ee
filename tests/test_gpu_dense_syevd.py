"""Symmetric eigendecomposition of one matrix on the device (nmx_syevd_*)
against the oracle's restatement of numax's Tensor-tier eigh (sytrd +
implicit QL + sort + Q Z, itself pinned to LAPACK in test_oracle.py).

Tolerances: eigenvalues normwise relative to max |lambda| 1e-12 (FP64) /
1e-5 (FP32); eigenvectors through size-independent properties -- the
residual ||A V - V diag(w)|| / ||A||, orthogonality |V^T V - I| -- and, for
eigenvalues separated from their neighbours, |<v_j, v_j(oracle)>| = 1 (the
sign of an eigenvector is arbitrary)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = {np.float64: 1e-12, np.float32: 1e-5}


def sym(n, seed, dtype=np.float64):
    rng = np.random.Generator(np.random.PCG64(seed))
    g = rng.standard_normal((n, n))
    return ((g + g.T) / 2).astype(dtype)


def with_garbage_upper(a, seed):
    """Only the lower triangle is read: fill the strict upper with noise."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.tril(a) + np.triu(rng.standard_normal(a.shape).astype(a.dtype) * 1e3, 1)


def run(a, vectors=True):
    from numax_b200 import linalg as L
    t = torch.from_numpy(a.copy()).cuda()
    if vectors:
        r = L.eigh(t)
        return r.values.cpu().numpy(), r.vectors.cpu().numpy()
    return L.eigvalsh(t).cpu().numpy(), None


def check(a, w, v, want_w, want_v, tol):
    a64 = np.tril(a).astype(np.float64)
    a64 = a64 + np.tril(a64, -1).T
    scale = max(np.abs(want_w).max(), 1e-300)
    assert np.all(np.diff(w) >= 0)
    assert np.abs(w.astype(np.float64) - want_w).max() / scale < tol
    if v is None:
        return
    v64 = v.astype(np.float64)
    n = a.shape[0]
    anorm = max(np.linalg.norm(a64, 2), 1e-300)
    assert np.linalg.norm(a64 @ v64 - v64 * w.astype(np.float64), 2) / anorm < tol * max(1, n) ** 0.5
    assert np.abs(v64.T @ v64 - np.eye(n)).max() < tol * max(1, n) ** 0.5
    if want_v is not None and n > 1:
        gaps = np.minimum(np.r_[np.inf, np.diff(want_w)], np.r_[np.diff(want_w), np.inf])
        sep = gaps > 1e-3 * scale
        dots = np.abs(np.sum(v64 * want_v.astype(np.float64), axis=0))
        assert np.all(np.abs(dots[sep] - 1) < 1e3 * tol)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [1, 2, 3, 5, 17, 32, 33, 64, 65, 100, 129, 257, 600])
def test_eigh_matches_oracle(oracle, dtype, n):
    a = with_garbage_upper(sym(n, seed=n, dtype=dtype), seed=n + 1)
    w, v = run(a)
    want_w, want_v = oracle.eigh(a)
    check(a, w, v, want_w.astype(np.float64), want_v, TOL[dtype])


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [1, 2, 7, 64, 300])
def test_eigvalsh_matches_oracle(oracle, dtype, n):
    a = with_garbage_upper(sym(n, seed=3 * n, dtype=dtype), seed=5)
    w, _ = run(a, vectors=False)
    want_w, _ = oracle.eigh(a, vectors=False)
    check(a, w, None, want_w.astype(np.float64), None, TOL[dtype])


def _special(name, n):
    rng = np.random.Generator(np.random.PCG64(11))
    q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    if name == "diagonal":
        return np.diag(rng.standard_normal(n))
    if name == "identity":
        return np.eye(n)
    if name == "zero":
        return np.zeros((n, n))
    if name == "two_clusters":
        return (q * np.repeat([1.0, 2.0], [n // 2, n - n // 2])) @ q.T
    if name == "tridiagonal_toeplitz":
        return 2 * np.eye(n) - np.eye(n, k=1) - np.eye(n, k=-1)
    if name == "graded":
        s = 10.0 ** (-np.arange(n) / (n / 12))
        return (q * s) @ q.T
    if name == "rank_one":
        x = rng.standard_normal(n)
        return np.outer(x, x)
    if name == "huge":
        return 1e150 * sym(n, 2)
    if name == "tiny":
        return 1e-150 * sym(n, 2)
    raise ValueError(name)


@pytest.mark.parametrize("name", ["diagonal", "identity", "zero", "two_clusters",
                                  "tridiagonal_toeplitz", "graded", "rank_one", "huge", "tiny"])
def test_eigh_structured(oracle, name):
    n = 160
    a = _special(name, n)
    w, v = run(a)
    want_w, want_v = oracle.eigh(a)
    check(a, w, v, want_w, want_v, 1e-12)


def test_eigh_large_properties():
    # n = 2048: the divide and conquer's top merges go through the GEMM.
    n = 2048
    a = sym(n, seed=21)
    w, v = run(a)
    want = np.linalg.eigvalsh(a)
    check(a, w, v, want, None, 1e-12)


def test_eigh_two_staging_chunks():
    # n = 4500 > 4096 columns: v is staged in two chunks per column; checked
    # on the device (residual, orthogonality) and against the values-only
    # path and cuSOLVER's eigenvalues.
    from numax_b200 import linalg as L
    n = 4500
    g = torch.randn(n, n, dtype=torch.float64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(3))
    a = (g + g.T) / 2
    r = L.eigh(a)
    w = L.eigvalsh(a)
    ref = torch.linalg.eigvalsh(a)
    scale = ref.abs().max()
    assert float((r.values - ref).abs().max() / scale) < 1e-12
    assert float((w - ref).abs().max() / scale) < 1e-12
    V = r.vectors
    res = torch.linalg.matrix_norm(a @ V - V * r.values, 2) / torch.linalg.matrix_norm(a, 2)
    assert float(res) < 1e-12 * n ** 0.5
    eye = torch.eye(n, dtype=torch.float64, device="cuda")
    assert float((V.T @ V - eye).abs().max()) < 1e-12 * n ** 0.5


def test_eigh_rejects_nonfinite_and_bad_shapes():
    from numax_b200 import linalg as L
    a = sym(50, 1)
    a[30, 10] = np.nan
    with pytest.raises(ValueError, match="NaN or an infinity"):
        L.eigh(torch.from_numpy(a).cuda())
    a[30, 10] = np.inf
    with pytest.raises(ValueError, match="NaN or an infinity"):
        L.eigvalsh(torch.from_numpy(a).cuda())
    # A NaN above the diagonal is never read.
    b = sym(50, 1)
    b[10, 30] = np.nan
    w, _ = run(b, vectors=False)
    assert np.isfinite(w).all()
    with pytest.raises(ValueError, match="must be square"):
        L.eigh(torch.zeros(3, 4, dtype=torch.float64, device="cuda"))
    with pytest.raises(ValueError, match="empty"):
        L.eigh(torch.zeros(0, 0, dtype=torch.float64, device="cuda"))


def test_eigh_strided_input_is_not_modified():
    import ctypes as C
    from numax_b200 import _lib
    n, lda = 70, 96
    a = sym(n, 4)
    big = torch.zeros(n, lda, dtype=torch.float64, device="cuda")
    big[:, :n] = torch.from_numpy(a).cuda()
    before = big.clone()
    w = torch.empty(n, dtype=torch.float64, device="cuda")
    v = torch.empty(n, n + 5, dtype=torch.float64, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("nmx_syevd_f64", _lib.context(0), n, big.data_ptr(), lda, w.data_ptr(),
              v.data_ptr(), n + 5, info.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert torch.equal(big, before)
    assert int(info.item()) == 0
    vv = v[:, :n].cpu().numpy()
    assert np.abs(a @ vv - vv * w.cpu().numpy()).max() < 1e-12 * np.abs(a).sum(1).max()
