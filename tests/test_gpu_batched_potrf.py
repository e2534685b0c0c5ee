"""Batched uneven Cholesky + cho_solve on the GPU vs the oracle (numax's
Array-tier cholesky/cholesky_solve run per matrix on the CPU).

Tolerances (north star): normwise relative 1e-12 for float64, 1e-5 for
float32, on L (lower triangle) and X per matrix."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = {np.float64: 1e-12, np.float32: 1e-5}


def make_batch(ns, nrhs, dtype, seed):
    """A_i = G G^T / n + n I with G iid N(0,1); B iid N(0,1) (PCG64)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    mats, rhs = [], []
    for n in ns:
        g = rng.standard_normal((n, n))
        mats.append((g @ g.T / n + n * np.eye(n)).astype(dtype).ravel())
        rhs.append(rng.standard_normal(n * nrhs).astype(dtype))
    return np.concatenate(mats), np.concatenate(rhs) if nrhs else np.zeros(0, dtype)


def run_gpu(ns, A, B, nrhs, alias=False):
    import numax_b200 as nb
    dt = torch.float64 if A.dtype == np.float64 else torch.float32
    dA = torch.from_numpy(A.copy()).cuda()
    dB = torch.from_numpy(B.copy()).cuda() if nrhs else None
    plan = nb.CholeskySolveBatch(ns, nrhs=nrhs, dtype=dt)
    X = dB if alias else None
    dA, dX, info = plan(dA, dB, X)
    return dA.cpu().numpy(), (dX.cpu().numpy() if nrhs else None), info.cpu().numpy()


def relerr(got, want):
    d = np.linalg.norm(want)
    return np.linalg.norm(got - want) / (d if d > 0 else 1.0)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_batched_potrf_potrs_matches_oracle(oracle, dtype):
    edge = [1, 2, 3, 7, 8, 15, 16, 17, 31, 32, 33, 47, 48, 63, 64, 65, 95, 96, 97, 127, 128]
    rng = np.random.Generator(np.random.PCG64(5))
    ns = np.array(edge + list(rng.integers(1, 129, size=300)), dtype=np.int32)
    rng.shuffle(ns)
    nrhs = 4
    A, B = make_batch(ns, nrhs, dtype, seed=9)
    gotA, gotX, info = run_gpu(ns, A, B, nrhs)
    wantL, wantX = oracle.batched_cholesky_solve(ns, A, B, nrhs)
    ao, bo = oracle.ragged_offsets(ns), oracle.ragged_offsets(ns, nrhs)
    tol = TOL[dtype]
    assert (info == 0).all()
    worst_l = worst_x = 0.0
    for i, n in enumerate(ns):
        gl = np.tril(gotA[ao[i]:ao[i] + n * n].reshape(n, n))
        wl = np.tril(wantL[ao[i]:ao[i] + n * n].reshape(n, n))
        # The upper triangle of A is left untouched.
        np.testing.assert_array_equal(np.triu(gotA[ao[i]:ao[i] + n * n].reshape(n, n), 1),
                                      np.triu(A[ao[i]:ao[i] + n * n].reshape(n, n), 1))
        worst_l = max(worst_l, relerr(gl, wl))
        worst_x = max(worst_x, relerr(gotX[bo[i]:bo[i] + n * nrhs], wantX[bo[i]:bo[i] + n * nrhs]))
    assert worst_l <= tol, worst_l
    assert worst_x <= tol, worst_x


@pytest.mark.parametrize("nrhs", [0, 1, 8])
def test_batched_rhs_counts_and_aliasing(oracle, nrhs):
    # 16 and 32 put 16 x 8 = 128 back-solve items on a 64-thread CTA.
    ns = np.array([5, 128, 33, 1, 64, 100, 16, 32, 31], dtype=np.int32)
    A, B = make_batch(ns, nrhs, np.float64, seed=nrhs)
    gotA, gotX, info = run_gpu(ns, A, B, nrhs, alias=nrhs > 0)
    wantL, wantX = oracle.batched_cholesky_solve(ns, A, B if nrhs else np.zeros(0), nrhs)
    ao = oracle.ragged_offsets(ns)
    for i, n in enumerate(ns):
        assert relerr(np.tril(gotA[ao[i]:ao[i] + n * n].reshape(n, n)),
                      np.tril(wantL[ao[i]:ao[i] + n * n].reshape(n, n))) <= 1e-12
    if nrhs:
        assert relerr(gotX, wantX) <= 1e-12


def test_batched_not_positive_definite_info_and_nan(oracle):
    # numax's later-block failure (tests/linalg/test_tensor_linalg.mojo:700-741):
    # positive definite leading 2x2, fails at index 3 -> info 4.
    bad = np.array([4.0, 1.0, 0.0, 0.0, 1.0, 4.0, 0.0, 0.0, 0.0, 0.0, 1.0, 3.0,
                    0.0, 0.0, 3.0, 1.0])
    good_ns = np.array([20, 70], dtype=np.int32)
    goodA, goodB = make_batch(good_ns, 2, np.float64, seed=1)
    ns = np.array([20, 4, 70], dtype=np.int32)
    A = np.concatenate([goodA[:400], bad, goodA[400:]])
    B = np.concatenate([goodB[:40], np.ones(8), goodB[40:]])
    gotA, gotX, info = run_gpu(ns, A, B, 2)
    assert list(info) == [0, 4, 0]
    wantL, wantX = oracle.batched_cholesky_solve(ns, A, B, 2)
    # Array-tier semantics: NaN exactly where the oracle has NaN.
    np.testing.assert_array_equal(np.isnan(gotX), np.isnan(wantX))
    L4 = gotA[400:416].reshape(4, 4)
    np.testing.assert_allclose(np.tril(L4)[:2, :2], np.tril(wantL[400:416].reshape(4, 4))[:2, :2],
                               rtol=1e-14)
    assert np.isnan(L4[3, 3])


def test_batched_reads_only_lower_triangle(oracle):
    ns = np.array([9, 40, 128], dtype=np.int32)
    A, B = make_batch(ns, 4, np.float64, seed=3)
    ao = oracle.ragged_offsets(ns)
    garbage = A.copy()
    for i, n in enumerate(ns):
        m = garbage[ao[i]:ao[i] + n * n].reshape(n, n)
        m[np.triu_indices(n, 1)] = np.nan
    gA, gX, _ = run_gpu(ns, A, B, 4)
    hA, hX, _ = run_gpu(ns, garbage, B, 4)
    np.testing.assert_array_equal(gX, hX)
    for i, n in enumerate(ns):
        np.testing.assert_array_equal(np.tril(gA[ao[i]:ao[i] + n * n].reshape(n, n)),
                                      np.tril(hA[ao[i]:ao[i] + n * n].reshape(n, n)))


def test_batched_rejects_bad_arguments():
    import numax_b200 as nb
    with pytest.raises(nb._lib.NmxError):
        nb.CholeskySolveBatch(np.array([129], dtype=np.int32), nrhs=4)
    with pytest.raises(nb._lib.NmxError):
        nb.CholeskySolveBatch(np.array([0], dtype=np.int32), nrhs=4)
    with pytest.raises(nb._lib.NmxError):
        nb.CholeskySolveBatch(np.array([4], dtype=np.int32), nrhs=9)
    plan = nb.CholeskySolveBatch(np.array([4, 5], dtype=np.int32), nrhs=1)
    with pytest.raises(ValueError):
        plan(torch.zeros(10, dtype=torch.float64, device="cuda"),
             torch.zeros(9, dtype=torch.float64, device="cuda"))


def test_batched_autotune_and_graph_replay(oracle):
    """The autotuner picks a covering CTA shape per size bucket and leaves
    valid outputs; a CUDA-graph replay of the plan gives bit-identical
    results to the direct launches, and re-captures for new buffers."""
    import numax_b200 as nb
    ns = np.array([5, 128, 33, 100, 64, 17, 96, 120, 8, 70], dtype=np.int32)
    nrhs = 4
    A, B = make_batch(ns, nrhs, np.float64, seed=21)
    wantL, wantX = oracle.batched_cholesky_solve(ns, A, B, nrhs)
    plan = nb.CholeskySolveBatch(ns, nrhs=nrhs, dtype=torch.float64)
    dA, dB = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    L = torch.empty_like(dA)
    X = torch.empty_like(dB)
    info = torch.empty(len(ns), dtype=torch.int32, device="cuda")
    sched = plan.autotune(dA, dB, X, info, L, reps=2)
    assert len(sched) == 4 and all(s["threads"] in (64, 96, 128, 192, 1032, 1064, 1128, 1256)
                                   and s["ctas"] >= 1 for s in sched)
    torch.cuda.synchronize()
    assert int(info.abs().sum()) == 0
    assert relerr(X.cpu().numpy(), wantX) <= 1e-12
    # Zero-filled L buffers: the plan writes only the lower triangles.
    L1, X1, _ = plan.run(dA, dB, torch.empty_like(dB), info, torch.zeros_like(dA))
    X1, L1 = X1.clone(), L1.clone()
    Lg, Xg = torch.zeros_like(dA), torch.empty_like(dB)
    for _ in range(2):  # capture, then replay
        plan.run(dA, dB, Xg, info, Lg, graph=True)
        torch.cuda.synchronize()
        assert torch.equal(Xg, X1) and torch.equal(Lg, L1)
    Xh = torch.empty_like(dB)  # new buffers: a new capture
    plan.run(dA, dB, Xh, info, Lg, graph=True)
    torch.cuda.synchronize()
    assert torch.equal(Xh, X1)


def test_batched_f32_full_config_vs_oracle_sample(oracle):
    """float32 at the BASELINE size: 100,000 SPD matrices, n ~ U[8, 128],
    4 right-hand sides, in one plan; every 50th matrix against the oracle
    (numax's Array-tier cholesky + cholesky_solve) within 1e-5."""
    import numax_b200 as nb
    rng = np.random.Generator(np.random.PCG64(100000))
    ns = rng.integers(8, 129, size=100_000).astype(np.int32)
    nrhs = 4
    sample = np.arange(0, len(ns), 50)
    # Data on the GPU (per size group), the sample copied back for the oracle.
    a_off = oracle.ragged_offsets(ns)
    b_off = oracle.ragged_offsets(ns, nrhs)
    total_a = int((ns.astype(np.int64) ** 2).sum())
    A = torch.empty(total_a, dtype=torch.float32, device="cuda")
    gen = torch.Generator(device="cuda")
    gen.manual_seed(7)
    ns_t = torch.from_numpy(ns).cuda()
    a_off_t = torch.from_numpy(a_off).cuda()
    for n in np.unique(ns):
        idx = torch.nonzero(ns_t == int(n)).flatten()
        g = torch.randn((idx.numel(), int(n), int(n)), generator=gen, dtype=torch.float64,
                        device="cuda")
        m = g @ g.transpose(1, 2) / n + n * torch.eye(int(n), dtype=torch.float64, device="cuda")
        pos = a_off_t[idx][:, None] + torch.arange(int(n) * int(n), device="cuda")[None, :]
        A[pos.flatten()] = m.reshape(-1).float()
    B = torch.randn(int(ns.astype(np.int64).sum()) * nrhs, generator=gen, dtype=torch.float32,
                    device="cuda")
    plan = nb.CholeskySolveBatch(ns, nrhs=nrhs, dtype=torch.float32)
    L, X, info = plan(A.clone(), B)
    assert int(info.abs().sum()) == 0
    hA, hB, hL, hX = A.cpu().numpy(), B.cpu().numpy(), L.cpu().numpy(), X.cpu().numpy()
    sub_ns = ns[sample]
    sa = np.concatenate([hA[a_off[i]:a_off[i] + ns[i] ** 2] for i in sample])
    sb = np.concatenate([hB[b_off[i]:b_off[i] + ns[i] * nrhs] for i in sample])
    wantL, wantX = oracle.batched_cholesky_solve(sub_ns, sa, sb, nrhs)
    so, sbo = oracle.ragged_offsets(sub_ns), oracle.ragged_offsets(sub_ns, nrhs)
    worst_l = worst_x = 0.0
    for j, i in enumerate(sample):
        n = int(ns[i])
        gl = np.tril(hL[a_off[i]:a_off[i] + n * n].reshape(n, n))
        wl = np.tril(wantL[so[j]:so[j] + n * n].reshape(n, n))
        worst_l = max(worst_l, relerr(gl, wl))
        worst_x = max(worst_x, relerr(hX[b_off[i]:b_off[i] + n * nrhs],
                                      wantX[sbo[j]:sbo[j] + n * nrhs]))
    assert worst_l <= 1e-5, worst_l
    assert worst_x <= 1e-5, worst_x


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("threads", [128, 192])
def test_batched_packed_shape_matches_oracle(oracle, threads, dtype):
    """The packed-triangle kernel forced on both element types (the plan's
    default is the tile kernel) against the oracle on ragged sizes that shape
    covers."""
    import numax_b200 as nb
    hi = 128 if threads == 192 else 96
    rng = np.random.Generator(np.random.PCG64(threads))
    ns = np.array([1, 8, 9, 16, 17, 33, 64, 65, hi] + list(rng.integers(1, hi + 1, size=150)),
                  dtype=np.int32)
    nrhs = 4
    A, B = make_batch(ns, nrhs, dtype, seed=threads)
    dt = torch.float64 if dtype == np.float64 else torch.float32
    plan = nb.CholeskySolveBatch(ns, nrhs=nrhs, dtype=dt)
    assert all(s["threads"] == threads for s in plan.force_shape(threads))
    gotA, gotX, info = plan(torch.from_numpy(A.copy()).cuda(), torch.from_numpy(B.copy()).cuda())
    wantL, wantX = oracle.batched_cholesky_solve(ns, A, B, nrhs)
    ao = oracle.ragged_offsets(ns)
    gotA, gotX = gotA.cpu().numpy(), gotX.cpu().numpy()
    assert (info.cpu().numpy() == 0).all()
    for i, n in enumerate(ns):
        blk = gotA[ao[i]:ao[i] + n * n].reshape(n, n)
        assert relerr(np.tril(blk), np.tril(wantL[ao[i]:ao[i] + n * n].reshape(n, n))) <= TOL[dtype]
    assert relerr(gotX, wantX) <= TOL[dtype]


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_batched_default_shapes(dt):
    """The plan's default schedule for both element types: the tile kernel,
    1 warp per matrix up to n = 64, 2 up to 96, 4 up to 128."""
    import numax_b200 as nb
    ns = np.array([20, 50, 90, 120], dtype=np.int32)
    sched = nb.CholeskySolveBatch(ns, nrhs=4, dtype=dt).schedule()
    assert [(s["n_max"], s["threads"]) for s in sched] == [(120, 1128), (90, 1064), (50, 1032),
                                                          (20, 1032)]


@pytest.mark.parametrize("warps", [1, 2, 4, 8])
def test_batched_tile_shape_f32_matches_oracle(oracle, warps):
    """The tile kernel on an FP32 batch (widened to FP64 on load, rounded on
    store) against the oracle's FP32 algorithm: ragged sizes around every tile
    edge, 0 and 4 right-hand sides, within FP32 tolerance."""
    import numax_b200 as nb
    shape = nb.batched.tile_shape(warps)
    edge = [1, 2, 7, 8, 9, 15, 16, 17, 31, 32, 33, 63, 64, 65, 95, 96, 97, 120, 127, 128]
    rng = np.random.Generator(np.random.PCG64(512 + warps))
    for nrhs in (0, 4):
        ns = np.array(edge + list(rng.integers(1, 129, size=100)), dtype=np.int32)
        rng.shuffle(ns)
        A, B = make_batch(ns, nrhs, np.float32, seed=nrhs + 70)
        plan = nb.CholeskySolveBatch(ns, nrhs=nrhs, dtype=torch.float32)
        assert all(s["threads"] == shape for s in plan.force_shape(shape))
        dA = torch.from_numpy(A.copy()).cuda()
        dB = torch.from_numpy(B.copy()).cuda() if nrhs else None
        gotA, gotX, info = plan(dA, dB)
        gotA, info = gotA.cpu().numpy(), info.cpu().numpy()
        wantL, wantX = oracle.batched_cholesky_solve(ns, A, B if nrhs else np.zeros(0, np.float32), nrhs)
        ao, bo = oracle.ragged_offsets(ns), oracle.ragged_offsets(ns, nrhs)
        assert (info == 0).all()
        for i, n in enumerate(ns):
            blk = gotA[ao[i]:ao[i] + n * n].reshape(n, n)
            assert relerr(np.tril(blk), np.tril(wantL[ao[i]:ao[i] + n * n].reshape(n, n))) <= 1e-5
            np.testing.assert_array_equal(np.triu(blk, 1),
                                          np.triu(A[ao[i]:ao[i] + n * n].reshape(n, n), 1))
        if nrhs:
            gotX = gotX.cpu().numpy()
            for i, n in enumerate(ns):
                assert relerr(gotX[bo[i]:bo[i] + n * nrhs], wantX[bo[i]:bo[i] + n * nrhs]) <= 1e-5


@pytest.mark.parametrize("warps", [1, 2, 4, 8])
def test_batched_tile_shape_matches_oracle(oracle, warps):
    """The 8 x 8 DMMA tile kernel (FP64) with 1, 2, 4 and 8 warps per matrix,
    forced on every bucket through the schedule override, against the oracle
    on ragged sizes around every tile edge, several right-hand-side counts,
    and numax's later-block failure (info = 4, NaN where the oracle has NaN)."""
    import numax_b200 as nb
    shape = nb.batched.tile_shape(warps)
    dtype = np.float64
    edge = [1, 2, 7, 8, 9, 15, 16, 17, 31, 32, 33, 63, 64, 65, 95, 96, 97, 120, 127, 128]
    rng = np.random.Generator(np.random.PCG64(256 + warps))
    for nrhs in (0, 1, 4, 8):
        ns = np.array(edge + list(rng.integers(1, 129, size=120)), dtype=np.int32)
        rng.shuffle(ns)
        A, B = make_batch(ns, nrhs, dtype, seed=nrhs + 40)
        plan = nb.CholeskySolveBatch(ns, nrhs=nrhs, dtype=torch.float64)
        assert all(s["threads"] == shape for s in plan.force_shape(shape))
        dA = torch.from_numpy(A.copy()).cuda()
        dB = torch.from_numpy(B.copy()).cuda() if nrhs else None
        gotA, gotX, info = plan(dA, dB)
        gotA, info = gotA.cpu().numpy(), info.cpu().numpy()
        wantL, wantX = oracle.batched_cholesky_solve(ns, A, B if nrhs else np.zeros(0), nrhs)
        ao, bo = oracle.ragged_offsets(ns), oracle.ragged_offsets(ns, nrhs)
        assert (info == 0).all()
        for i, n in enumerate(ns):
            blk = gotA[ao[i]:ao[i] + n * n].reshape(n, n)
            assert relerr(np.tril(blk), np.tril(wantL[ao[i]:ao[i] + n * n].reshape(n, n))) <= 1e-12
            np.testing.assert_array_equal(np.triu(blk, 1),
                                          np.triu(A[ao[i]:ao[i] + n * n].reshape(n, n), 1))
        if nrhs:
            gotX = gotX.cpu().numpy()
            for i, n in enumerate(ns):
                assert relerr(gotX[bo[i]:bo[i] + n * nrhs], wantX[bo[i]:bo[i] + n * nrhs]) <= 1e-12
    # numax's later-block failure through the tile kernel.
    bad = np.array([4.0, 1.0, 0.0, 0.0, 1.0, 4.0, 0.0, 0.0, 0.0, 0.0, 1.0, 3.0,
                    0.0, 0.0, 3.0, 1.0])
    good_ns = np.array([20, 70], dtype=np.int32)
    goodA, goodB = make_batch(good_ns, 2, np.float64, seed=1)
    ns = np.array([20, 4, 70], dtype=np.int32)
    A = np.concatenate([goodA[:400], bad, goodA[400:]])
    B = np.concatenate([goodB[:40], np.ones(8), goodB[40:]])
    plan = nb.CholeskySolveBatch(ns, nrhs=2, dtype=torch.float64)
    plan.force_shape(shape)
    gotA, gotX, info = plan(torch.from_numpy(A.copy()).cuda(), torch.from_numpy(B.copy()).cuda())
    assert list(info.cpu().numpy()) == [0, 4, 0]
    wantL, wantX = oracle.batched_cholesky_solve(ns, A, B, 2)
    np.testing.assert_array_equal(np.isnan(gotX.cpu().numpy()), np.isnan(wantX))
