"""Host-side helpers of the batched plan and of bench.py's JSON line, on the
CPU: the tile kernel's CTA-shape codes, the arithmetic type a schedule runs
in, the kernel a shape selects, and the algorithmic byte and flop counts."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def test_tile_shape_codes():
    from numax_b200.batched import tile_shape
    assert [tile_shape(w) for w in (1, 2, 4, 8)] == [1032, 1064, 1128, 1256]
    for bad in (0, 3, 16):
        with pytest.raises(ValueError):
            tile_shape(bad)


def test_arithmetic_type_of_a_schedule():
    import bench
    tile = [{"threads": 1128}, {"threads": 1032}]
    packed = [{"threads": 192}, {"threads": 64}]
    assert bench.arith_dtype(tile, "f64") == "f64"
    assert bench.arith_dtype(tile, "f32") == "f64"      # the tile kernel computes in FP64
    assert bench.arith_dtype(packed, "f32") == "f32"
    assert bench.arith_dtype(packed, "f64") == "f64"
    assert bench.arith_dtype(tile + packed, "f32") == "f32+f64"


def test_kernel_names_follow_the_shape_code():
    import bench
    assert bench.kernel_name(1128, "f64").startswith("potrf_tile_batched_kernel<4>")
    assert bench.kernel_name(1032, "f32").startswith("potrf_tile_batched_kernel<1>")
    assert bench.kernel_name(192, "f64") == "potrf_potrs_batched_kernel<double, 192>"
    assert bench.kernel_name(96, "f32") == "potrf_potrs_batched_kernel<float, 96>"


def test_algorithmic_bytes_and_flops():
    import bench
    ns = np.array([1, 8, 128], dtype=np.int64)
    nrhs = 4
    # lower(A) read + lower(L) written + B read + X written, per matrix, plus 4-byte info.
    want = sum(8 * (n * (n + 1) // 2 * 2 + 2 * nrhs * n) for n in ns) + 4 * len(ns)
    assert bench.algorithmic_bytes(ns, nrhs, 8) == want
    assert bench.algorithmic_flops(ns, nrhs) == pytest.approx(
        float(sum(n ** 3 / 3 + 2 * nrhs * n ** 2 for n in ns)))


def test_syevd_and_npy_argument_checks_need_no_device():
    """Argument errors come back as -(index) before any CUDA call."""
    import ctypes as C
    from numax_b200 import _lib
    lib = _lib.load()
    info = C.c_int32()
    # ctx NULL is argument 1; n < 0 is argument 2 (checked after ctx).
    assert lib.nmx_syevd_f64(None, 4, None, 4, None, None, 4, C.byref(info), None) == -1
    assert lib.nmx_syevd_f32(None, 4, None, 4, None, None, 4, C.byref(info), None) == -1
    fake_ctx = C.c_void_p(1)
    assert lib.nmx_syevd_f64(fake_ctx, -1, None, 4, None, None, 4, C.byref(info), None) == -2
    assert lib.nmx_syevd_f64(fake_ctx, 4, None, 4, None, None, 4, C.byref(info), None) == -3
    buf = (C.c_double * 16)()
    assert lib.nmx_syevd_f64(fake_ctx, 4, buf, 3, buf, None, 4, C.byref(info), None) == -4
    assert lib.nmx_syevd_f64(fake_ctx, 4, buf, 4, buf, buf, 2, C.byref(info), None) == -7
    assert lib.nmx_syevd_f64(fake_ctx, 4, buf, 4, buf, None, 4, None, None) == -8
    shape = (C.c_int64 * 2)(2, 2)
    assert lib.nmx_npy_load(None, None, 0, 2, shape, None, 0, None) == -2
    assert lib.nmx_npy_load(None, b"x.npy", 99, 2, shape, None, 0, None) == -3
    assert lib.nmx_npy_load(None, b"x.npy", 0, 65, shape, None, 0, None) == -4
    assert lib.nmx_npy_save(None, b"x.npy", 1, 1, (C.c_int64 * 1)(-3), None, None) == -5
    assert lib.nmx_npy_header(None, None, None, None, 0, None) == -1
