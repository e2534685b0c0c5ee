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


def test_noalloc_rejects_batches_over_the_limit():
    from numax_b200 import _lib
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    ns = np.full(65537, 4, dtype=np.int32)
    rc = lib.nmx_potrf_potrs_batched_noalloc_f64(ctx, len(ns), ns.ctypes.data, 1, None, None,
                                                 None, None, None, None)
    assert rc == -2
    assert "65536" in _lib.last_error()
