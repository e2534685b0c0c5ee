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
