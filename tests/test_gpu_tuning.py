"""Per-context tuning knobs (the autotuner's hook): round trip, rejection of
unknown keys and bad values, and results that do not depend on them -- the
LU's pivots and factors for every leaf width, the IR solution for every
tensor-core threshold."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

KEYS = [b"lu.leaf_ctas", b"lu.cluster", b"lu.leaf_w", b"ir.trsv_ctas", b"ir.tc_min",
        b"lu.tournament", b"lu.lookahead", b"lu.panel_sms"]


def test_tune_keys_round_trip_and_errors():
    import ctypes as C
    from numax_b200 import _lib
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    v = C.c_int64()
    for key in KEYS:
        assert lib.nmx_tune_get(ctx, key, C.byref(v)) == 0
        old = v.value
        assert lib.nmx_tune_set(ctx, key, 48) == 0
        assert lib.nmx_tune_get(ctx, key, C.byref(v)) == 0 and v.value == 48
        assert lib.nmx_tune_set(ctx, key, old) == 0
    assert lib.nmx_tune_set(ctx, b"no.such.key", 1) == -2
    assert lib.nmx_tune_set(ctx, b"lu.cluster", -5) == -3


@pytest.mark.parametrize("leaf_w", [8, 16, 48, 64])
def test_lu_leaf_width_does_not_change_results(leaf_w):
    import scipy.linalg as sl
    from numax_b200 import _lib, linalg
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    n = 1500
    a = np.random.Generator(np.random.PCG64(7 + leaf_w)).standard_normal((n, n))
    lib.nmx_tune_set(ctx, b"lu.leaf_w", leaf_w)
    try:
        f = linalg.lu_factor(torch.from_numpy(a).cuda())
    finally:
        lib.nmx_tune_set(ctx, b"lu.leaf_w", 0)
    lu, piv = sl.lu_factor(a)
    np.testing.assert_array_equal(f.pivots.cpu().numpy(), piv)
    assert np.linalg.norm(f.factored.cpu().numpy() - lu) / np.linalg.norm(lu) <= 1e-12


@pytest.mark.parametrize("tc_min", [0, 64, 100000])
def test_ir_tensor_core_threshold(tc_min):
    from numax_b200 import _lib, linalg
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    n = 1200
    rng = np.random.Generator(np.random.PCG64(11))
    a = rng.standard_normal((n, n)) / np.sqrt(n) + 2 * np.eye(n)
    b = rng.standard_normal(n)
    lib.nmx_tune_set(ctx, b"ir.tc_min", tc_min)
    try:
        x, st = linalg.solve_ir(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda(),
                                precision="bf16x3", tol=1e-14)
    finally:
        lib.nmx_tune_set(ctx, b"ir.tc_min", -1)
    x = x.cpu().numpy()
    assert st["converged"] == 1, st
    berr = np.abs(b - a @ x).max() / (np.abs(a).sum(1).max() * np.abs(x).max() + np.abs(b).max())
    assert berr <= 1e-14
