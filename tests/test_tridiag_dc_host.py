"""The eigh kernels' divide-and-conquer arithmetic (tridiag_dc.cuh:
deflation, secular roots, Loewner z-hat, merged ranks) compiled for the host
and run merge by merge in the kernels' order (tests/host/tridiag_dc_host.cu),
checked against LAPACK on random and structured tridiagonals.  CPU only:
nvcc compiles the header's __host__ __device__ functions for the host."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def dc(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    out = str(tmp_path_factory.mktemp("dc") / "libdc_host.so")
    subprocess.run([nvcc, "-O2", "-x", "cu", "-shared", "-Xcompiler", "-fPIC",
                    "-Wno-deprecated-gpu-targets", "-I", os.path.join(ROOT, "numax_b200", "csrc"),
                    os.path.join(ROOT, "tests", "host", "tridiag_dc_host.cu"), "-o", out],
                   check=True)
    lib = C.CDLL(out)
    lib.dc_host_solve.restype = C.c_int
    return lib


def solve(lib, d, e):
    n = len(d)
    d = np.ascontiguousarray(d, dtype=np.float64)
    e = np.ascontiguousarray(np.concatenate([e[:n - 1], [0.0]]), dtype=np.float64)
    w = np.zeros(n)
    z = np.zeros((n, n))
    it = C.c_int()
    rc = lib.dc_host_solve(n, d.ctypes.data_as(C.c_void_p), e.ctypes.data_as(C.c_void_p),
                           w.ctypes.data_as(C.c_void_p), z.ctypes.data_as(C.c_void_p), C.byref(it))
    assert rc == 0
    return w, z, it.value


def cases():
    rng = np.random.Generator(np.random.PCG64(0))
    for n in (1, 2, 3, 5, 8, 17, 64, 100, 257, 600):
        yield f"random{n}", rng.standard_normal(n), rng.standard_normal(n)
    n = 400
    yield "zero_offdiag", rng.standard_normal(n), np.zeros(n)
    yield "identity", np.ones(n), np.zeros(n)
    yield "two_values_tiny_e", np.repeat([1.0, 2.0], n // 2), 1e-18 * rng.standard_normal(n)
    yield "toeplitz", 2.0 * np.ones(n), -np.ones(n)
    yield "wilkinson", np.abs(np.arange(-(n // 2), n - n // 2)).astype(float), np.ones(n)
    yield "graded", 10.0 ** (-np.arange(n) / 40), 0.5 * 10.0 ** (-np.arange(n) / 40)
    yield "zero_diag", np.zeros(n), np.ones(n)
    yield "huge", 1e200 * rng.standard_normal(n), 1e200 * rng.standard_normal(n)
    yield "tiny", 1e-200 * rng.standard_normal(n), 1e-200 * rng.standard_normal(n)


@pytest.mark.parametrize("name,d,e", list(cases()), ids=[c[0] for c in cases()])
def test_divide_and_conquer_matches_lapack(dc, name, d, e):
    n = len(d)
    T = np.diag(d) + np.diag(e[:n - 1], 1) + np.diag(e[:n - 1], -1)
    w, z, it = solve(dc, d, e)
    want = np.linalg.eigvalsh(T)
    scale = max(np.abs(want).max(), np.finfo(float).tiny)
    assert np.all(np.diff(w) >= 0)
    assert np.abs(w - want).max() / scale < 1e-13
    assert np.abs(z.T @ z - np.eye(n)).max() < 1e-13
    assert np.abs(T @ z - z * w).max() / scale < 1e-13
    assert it <= 60  # the one-pole rational steps converge in a handful


@pytest.mark.parametrize("name,d,e", [c for c in cases() if c[0] not in ("huge", "tiny")],
                         ids=[c[0] for c in cases() if c[0] not in ("huge", "tiny")])
def test_sturm_multisection_matches_lapack(dc, name, d, e):
    """The values-only path's multisection (sturm_kth): every eigenvalue to
    a few ulps of max |lambda| (the kernel runs it on the scaled matrix, so
    the extreme-scale cases are the scaling's business, not the count's)."""
    n = len(d)
    T = np.diag(d) + np.diag(e[:n - 1], 1) + np.diag(e[:n - 1], -1)
    dd = np.ascontiguousarray(d, dtype=np.float64)
    ee = np.ascontiguousarray(np.concatenate([e[:n - 1], [0.0]]), dtype=np.float64)
    w = np.zeros(n)
    dc.sturm_host_values(n, dd.ctypes.data_as(C.c_void_p), ee.ctypes.data_as(C.c_void_p),
                         w.ctypes.data_as(C.c_void_p))
    want = np.linalg.eigvalsh(T)
    scale = max(np.abs(want).max(), np.finfo(float).tiny)
    assert np.all(np.diff(w) >= 0)
    assert np.abs(w - want).max() / scale < 1e-13
