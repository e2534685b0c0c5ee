"""The allocation-free batched Cholesky + cho_solve entry point.

Some callers cannot allocate device memory -- a host runtime whose allocator
already owns the GPU, or code running inside another framework's memory
pool -- so nmx_potrf_potrs_batched_noalloc_f64 keeps its schedule in a fixed
device array built into the library.  This checks it through the C ABI
against the plan-based entry point on the same inputs, on two calls in a
row (the second with different sizes and values, so nothing left in the
shared array by the first call can leak into the second).  It is collected
last so that a stop at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _batch(ns, nrhs, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    mats, rhs = [], []
    for n in ns:
        g = rng.standard_normal((n, n))
        mats.append((g @ g.T / n + n * np.eye(n)).ravel())
        rhs.append(rng.standard_normal(n * nrhs))
    return np.concatenate(mats), np.concatenate(rhs)


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_noalloc_matches_plan_path_twice():
    import numax_b200 as nb
    from numax_b200 import _lib
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    stream = torch.cuda.current_stream().cuda_stream
    for call, seed in enumerate((21, 22)):
        rng = np.random.Generator(np.random.PCG64(seed))
        count = 300 if call == 0 else 517
        ns = np.ascontiguousarray(rng.integers(1, 129, size=count), dtype=np.int32)
        nrhs = 4 if call == 0 else 3
        A, B = _batch(ns, nrhs, seed + 100)
        dA = torch.from_numpy(A).cuda()
        dB = torch.from_numpy(B).cuda()
        # Reference: the plan-based entry point.
        plan = nb.CholeskySolveBatch(ns, nrhs=nrhs, dtype=torch.float64)
        refL, refX, refI = plan(dA, dB, L=torch.zeros_like(dA))
        # Allocation-free entry point, called through the C ABI.
        L = torch.zeros_like(dA)
        X = torch.full_like(dB, float("nan"))
        info = torch.full((count,), -7, dtype=torch.int32, device=dA.device)
        rc = lib.nmx_potrf_potrs_batched_noalloc_f64(
            ctx, count, ns.ctypes.data, nrhs, C.c_void_p(dA.data_ptr()), C.c_void_p(L.data_ptr()),
            C.c_void_p(dB.data_ptr()), C.c_void_p(X.data_ptr()), C.c_void_p(info.data_ptr()),
            C.c_void_p(stream))
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        assert _rel(X.cpu().numpy(), refX.cpu().numpy()) <= 1e-12
        ao = nb.ragged_offsets(ns)
        got, want = L.cpu().numpy(), refL.cpu().numpy()
        for i, n in enumerate(ns):
            g = np.tril(got[ao[i]:ao[i] + n * n].reshape(n, n))
            w = np.tril(want[ao[i]:ao[i] + n * n].reshape(n, n))
            assert _rel(g, w) <= 1e-12
        assert (info.cpu().numpy() == refI.cpu().numpy()).all()


def _noalloc_call(lib, ctx, ns, nrhs, dA, L, dB, X, info, stream):
    return lib.nmx_potrf_potrs_batched_noalloc_f64(
        ctx, len(ns), ns.ctypes.data, nrhs, C.c_void_p(dA.data_ptr()), C.c_void_p(L.data_ptr()),
        C.c_void_p(dB.data_ptr()), C.c_void_p(X.data_ptr()), C.c_void_p(info.data_ptr()),
        C.c_void_p(stream))


def test_noalloc_matches_oracle_at_the_limit_with_a_failing_matrix(oracle):
    """65,536 matrices (the limit), one of them not positive definite:
    factors and solutions against the oracle (numax's Array-tier Cholesky and
    cholesky_solve per matrix), `info` = 4 for the failing one (numax's
    later-block failure fixture), NaN exactly where the oracle has NaN."""
    from numax_b200 import _lib
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.Generator(np.random.PCG64(31))
    count, nrhs, bad_at = 65536, 2, 40000
    ns = np.ascontiguousarray(rng.integers(1, 25, size=count), dtype=np.int32)
    ns[bad_at] = 4
    A, B = _batch(ns, nrhs, 32)
    ao = np.zeros(count, dtype=np.int64)
    ao[1:] = np.cumsum(ns.astype(np.int64) ** 2)[:-1]
    A[ao[bad_at]:ao[bad_at] + 16] = [4.0, 1.0, 0.0, 0.0, 1.0, 4.0, 0.0, 0.0,
                                     0.0, 0.0, 1.0, 3.0, 0.0, 0.0, 3.0, 1.0]
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    L = torch.zeros_like(dA)
    X = torch.full_like(dB, float("nan"))
    info = torch.full((count,), -7, dtype=torch.int32, device=dA.device)
    assert _noalloc_call(lib, ctx, ns, nrhs, dA, L, dB, X, info, stream) == 0, _lib.last_error()
    torch.cuda.synchronize()
    want_info = np.zeros(count, dtype=np.int32)
    want_info[bad_at] = 4
    np.testing.assert_array_equal(info.cpu().numpy(), want_info)
    wantL, wantX = oracle.batched_cholesky_solve(ns, A, B, nrhs)
    gotL, gotX = L.cpu().numpy(), X.cpu().numpy()
    np.testing.assert_array_equal(np.isnan(gotX), np.isnan(wantX))
    ok = ~np.isnan(wantX)
    bo = np.zeros(count, dtype=np.int64)
    bo[1:] = np.cumsum(ns.astype(np.int64) * nrhs)[:-1]
    worst_l = worst_x = 0.0
    for i in range(0, count, 7):  # every 7th matrix, plus the failing one
        n = int(ns[i])
        if i == bad_at:
            continue
        g = np.tril(gotL[ao[i]:ao[i] + n * n].reshape(n, n))
        w = np.tril(wantL[ao[i]:ao[i] + n * n].reshape(n, n))
        worst_l = max(worst_l, _rel(g, w))
        worst_x = max(worst_x, _rel(gotX[bo[i]:bo[i] + n * nrhs], wantX[bo[i]:bo[i] + n * nrhs]))
    assert worst_l <= 1e-12, worst_l
    assert worst_x <= 1e-12, worst_x
    assert _rel(gotX[ok], wantX[ok]) <= 1e-12
    bad = np.tril(gotL[ao[bad_at]:ao[bad_at] + 16].reshape(4, 4))
    np.testing.assert_allclose(bad[:2, :2], np.tril(wantL[ao[bad_at]:ao[bad_at] + 16]
                                                     .reshape(4, 4))[:2, :2], rtol=1e-14)


def test_noalloc_refuses_a_capturing_stream():
    """The sizes are checked on the host at each call, so a call made while
    its stream is being captured is refused rather than recorded."""
    from numax_b200 import _lib
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    ns = np.array([3, 5], dtype=np.int32)
    A, B = _batch(ns, 1, 3)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    L, X = torch.zeros_like(dA), torch.zeros_like(dB)
    info = torch.zeros(2, dtype=torch.int32, device="cuda")
    # Set-up on this device happens on a first, uncaptured call.
    assert _noalloc_call(lib, ctx, ns, 1, dA, L, dB, X, info,
                         torch.cuda.current_stream().cuda_stream) == 0, _lib.last_error()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    with torch.cuda.graph(g, stream=side):
        rc = _noalloc_call(lib, ctx, ns, 1, dA, L, dB, X, info, side.cuda_stream)
    assert rc == -1002
    assert "captured" in _lib.last_error()


def test_noalloc_rejects_batches_over_the_limit():
    from numax_b200 import _lib
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    ns = np.full(65537, 4, dtype=np.int32)
    rc = lib.nmx_potrf_potrs_batched_noalloc_f64(ctx, len(ns), ns.ctypes.data, 1, None, None,
                                                 None, None, None, None)
    assert rc == -2
    assert "65536" in _lib.last_error()
