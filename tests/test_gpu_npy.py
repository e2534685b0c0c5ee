""".npy interchange with device memory: files written from HBM are
byte-identical to numpy.save's, files numpy wrote load into HBM bit-exactly,
and a (count, n, n) stack saved by numpy feeds the batched Cholesky +
cho_solve directly (its A layout), checked against the oracle."""
import io

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def np_bytes(a):
    b = io.BytesIO()
    np.save(b, a)
    return b.getvalue()


@pytest.fixture
def npx():
    from numax_b200.io import numpy as npx
    return npx


def test_device_round_trip_multichunk(npx, tmp_path):
    # 96 MiB of float64: twelve 8 MiB chunks across the worker threads.
    rng = np.random.Generator(np.random.PCG64(1))
    a = rng.standard_normal((3, 2048, 2048))
    d = torch.from_numpy(a).cuda()
    p = tmp_path / "a.npy"
    npx.save(d, p)
    assert p.read_bytes() == np_bytes(a)
    back = npx.load(p, torch.float64, 3, 2048, 2048, device="cuda")
    assert back.is_cuda
    assert torch.equal(back.view(torch.int64).cpu(), d.view(torch.int64).cpu())


@pytest.mark.parametrize("np_dt,t_dt", [(np.float32, torch.float32), (np.int32, torch.int32),
                                        (np.bool_, torch.bool), (np.float16, torch.float16),
                                        (np.uint8, torch.uint8)])
@pytest.mark.parametrize("shape", [(5,), (0,), (), (3, 7, 2)])
def test_device_types_and_shapes(npx, tmp_path, np_dt, t_dt, shape):
    rng = np.random.Generator(np.random.PCG64(7))
    a = (rng.standard_normal(shape) * 50).astype(np_dt)
    p = tmp_path / "t.npy"
    np.save(p, a)
    got = npx.load_dyn(p, t_dt, len(shape), device="cuda")
    assert got.is_cuda and tuple(got.shape) == shape
    assert got.cpu().numpy().tobytes() == a.tobytes()
    q = tmp_path / "u.npy"
    npx.save(got, q)
    assert q.read_bytes() == np_bytes(a)


def test_device_load_rejects_before_copying(npx, tmp_path):
    from numax_b200.io import NpyError
    p = tmp_path / "f.npy"
    np.save(p, np.zeros((4, 4), np.float32))
    with pytest.raises(NpyError, match="dtype mismatch"):
        npx.load(p, torch.float64, 4, 4, device="cuda")
    with pytest.raises(NpyError, match="shape mismatch"):
        npx.load(p, torch.float32, 4, 5, device="cuda")
    np.save(p, np.asfortranarray(np.zeros((4, 4), np.float32)))
    with pytest.raises(NpyError, match="Fortran-ordered"):
        npx.load(p, torch.float32, 4, 4, device="cuda")


def _spd_stack(count, n, nrhs, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    g = rng.standard_normal((count, n, n))
    a = g @ g.transpose(0, 2, 1) / n + n * np.eye(n)
    return a, rng.standard_normal((count, n, nrhs))


def test_numpy_stack_feeds_the_batched_cholesky(npx, tmp_path, oracle):
    import numax_b200 as nb
    count, n, nrhs = 300, 48, 4
    a, b = _spd_stack(count, n, nrhs, seed=3)
    pa, pb = tmp_path / "A.npy", tmp_path / "B.npy"
    np.save(pa, a)
    np.save(pb, b)
    dA = npx.load(pa, torch.float64, count, n, n, device="cuda")
    dB = npx.load(pb, torch.float64, count, n, nrhs, device="cuda")
    ns = np.full(count, n, np.int32)
    plan = nb.CholeskySolveBatch(ns, nrhs=nrhs, dtype=torch.float64)
    L, X, info = plan(dA.reshape(-1), dB.reshape(-1))
    torch.cuda.synchronize()
    wantL, wantX = oracle.batched_cholesky_solve(ns, a.ravel(), b.ravel(), nrhs)
    assert (info.cpu().numpy() == 0).all()
    gl = np.tril(L.cpu().numpy().reshape(count, n, n))
    wl = np.tril(wantL.reshape(count, n, n))
    assert np.linalg.norm(gl - wl) / np.linalg.norm(wl) < 1e-12
    gx = X.cpu().numpy()
    assert np.linalg.norm(gx - wantX) / np.linalg.norm(wantX) < 1e-12
    # The factors go back out as numpy reads them.
    pl = tmp_path / "L.npy"
    npx.save(L.reshape(count, n, n), pl)
    assert np.load(pl).tobytes() == L.cpu().numpy().tobytes()


def test_ragged_batch_from_a_flat_file(npx, tmp_path, oracle):
    import numax_b200 as nb
    rng = np.random.Generator(np.random.PCG64(5))
    ns = rng.integers(1, 129, 200).astype(np.int32)
    mats, rhs = [], []
    for n in ns:
        g = rng.standard_normal((n, n))
        mats.append((g @ g.T / n + n * np.eye(n)).ravel())
        rhs.append(rng.standard_normal(n * 4))
    A, B = np.concatenate(mats), np.concatenate(rhs)
    np.save(tmp_path / "A.npy", A)
    np.save(tmp_path / "ns.npy", ns)
    dA = npx.load_dyn(tmp_path / "A.npy", torch.float64, 1, device="cuda")
    sizes = npx.load_dyn(tmp_path / "ns.npy", torch.int32, 1).numpy()
    assert (sizes == ns).all()
    plan = nb.CholeskySolveBatch(sizes, nrhs=4, dtype=torch.float64)
    L, X, info = plan(dA, torch.from_numpy(B).cuda())
    torch.cuda.synchronize()
    wantL, wantX = oracle.batched_cholesky_solve(ns, A, B, 4)
    assert (info.cpu().numpy() == 0).all()
    gx = X.cpu().numpy()
    assert np.linalg.norm(gx - wantX) / np.linalg.norm(wantX) < 1e-12
