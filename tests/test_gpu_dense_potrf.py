"""Dense Cholesky + cholesky_solve on the GPU vs the oracle (numax's blocked
cholesky / cholesky_solve restated) and LAPACK.  float64 within 1e-12
normwise relative, float32 within 1e-5; numax's failure message and index."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d else 1.0))


def spd(n, seed, dtype=np.float64):
    rng = np.random.Generator(np.random.PCG64(seed))
    g = rng.standard_normal((n, n))
    return (g @ g.T / n + np.eye(n)).astype(dtype)


@pytest.mark.parametrize("n", [1, 2, 5, 31, 32, 33, 64, 96, 257, 600])
def test_cholesky_matches_oracle_f64(oracle, n):
    from numax_b200 import linalg
    a = spd(n, 40 + n)
    L = linalg.cholesky(torch.from_numpy(a).cuda()).cpu().numpy()
    want, info = oracle.cholesky(a, block=32, tile=n)
    assert info == 0
    assert rel(L, want) <= 1e-12
    assert np.all(np.triu(L, 1) == 0)
    rng = np.random.Generator(np.random.PCG64(n))
    b = rng.standard_normal(n)
    bm = rng.standard_normal((n, 16))
    dl = torch.from_numpy(L).cuda()
    x = linalg.cholesky_solve(dl, torch.from_numpy(b).cuda()).cpu().numpy()
    xm = linalg.cholesky_solve(dl, torch.from_numpy(bm).cuda()).cpu().numpy()
    assert rel(x, oracle.cholesky_solve(want, b)) <= 1e-12
    assert rel(xm, oracle.cholesky_solve(want, bm)) <= 1e-12


def test_cholesky_large_vs_lapack():
    from numax_b200 import linalg
    n = 3000
    a = spd(n, 7)
    L = linalg.cholesky(torch.from_numpy(a).cuda()).cpu().numpy()
    assert rel(L, np.linalg.cholesky(a)) <= 1e-12


@pytest.mark.parametrize("n", [9, 100])
def test_cholesky_f32(oracle, n):
    from numax_b200 import linalg
    a = spd(n, n, np.float32)
    L = linalg.cholesky(torch.from_numpy(a).cuda()).cpu().numpy()
    want, _ = oracle.cholesky(a, block=32, tile=n)
    assert rel(L, want) <= 1e-5


def test_cholesky_reads_only_lower_and_reports_numax_errors():
    from numax_b200 import linalg
    nx = np.load(os.path.join(GOLD, "numax_fixtures.npz"))
    a = nx["spd5"].copy()
    want = linalg.cholesky(torch.from_numpy(a).cuda()).cpu().numpy()
    a[np.triu_indices(5, 1)] = np.nan
    got = linalg.cholesky(torch.from_numpy(a).cuda()).cpu().numpy()
    np.testing.assert_array_equal(got, want)
    # tests/linalg/test_tensor_linalg.mojo:681-741
    with pytest.raises(ValueError, match="not positive definite"):
        linalg.cholesky(torch.from_numpy(nx["not_spd_2x2"]).cuda())
    with pytest.raises(ValueError, match="index 3"):
        linalg.cholesky(torch.from_numpy(nx["later_block"]).cuda())


def test_cholesky_config_order_8192_matches_lapack():
    """FP64 Cholesky at a BASELINE order (SPD G G^T / n + I, n = 8192) against
    LAPACK's factor, and the 16-right-hand-side cholesky_solve, within 1e-12."""
    import scipy.linalg as sl
    from numax_b200 import linalg
    n = 8192
    a = spd(n, 8192)
    L = linalg.cholesky(torch.from_numpy(a).cuda())
    want = np.linalg.cholesky(a)
    assert rel(L.cpu().numpy(), want) <= 1e-12
    rng = np.random.Generator(np.random.PCG64(3))
    bm = rng.standard_normal((n, 16))
    x = linalg.cholesky_solve(L, torch.from_numpy(bm).cuda()).cpu().numpy()
    assert rel(x, sl.cho_solve((want, True), bm)) <= 1e-12


def test_info_readback_for_the_mojo_raise():
    """The path the Mojo binding takes for numax's raise: nmx_potrf_f64 then
    nmx_memcpy_to_host of the info word, which names numax's 0-based index
    (info - 1) of the first non-positive pivot; nmx_synchronize on the
    stream."""
    import ctypes as C
    from numax_b200 import _lib
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    nx = np.load(os.path.join(GOLD, "numax_fixtures.npz"))
    a = torch.from_numpy(np.ascontiguousarray(nx["later_block"])).cuda()
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    n = a.shape[0]
    assert lib.nmx_potrf_f64(ctx, n, C.c_void_p(a.data_ptr()), n, C.c_void_p(info.data_ptr()),
                             C.c_void_p(stream)) == 0
    host = C.c_int32(-1)
    assert lib.nmx_memcpy_to_host(ctx, C.byref(host), C.c_void_p(info.data_ptr()), 4,
                                  C.c_void_p(stream)) == 0
    assert host.value - 1 == 3  # numax's "non-positive pivot at index 3"
    assert lib.nmx_synchronize(ctx, C.c_void_p(stream)) == 0
