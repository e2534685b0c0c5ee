"""The C-ABI library builds, loads and exports every entry point its public
header declares.  CPU only: nothing here launches a kernel."""
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        names += re.findall(r"NMX_API[^;(]*?\b(nmx_\w+)\s*\(", open(h).read())
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from numax_b200 import build, _lib
    build.build()
    return _lib.load()


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "nmx_create" in names and len(names) >= 8


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from numax_b200 import _lib
    missing = [n for n in declared_symbols() if n not in _lib.SIGNATURES]
    assert not missing, missing


def test_argument_errors_need_no_device(lib):
    import ctypes as C
    from numax_b200 import _lib
    # A NULL output pointer is rejected before any CUDA call: -(argument index).
    assert lib.nmx_create(0, None) == -2
    assert "out is NULL" in _lib.last_error()
    assert lib.nmx_version() >= 100
    assert lib.nmx_batched_plan_sizes(None, None, None) == -1


def test_tuning_keys_documented(lib):
    """Every key nmx_tune_set accepts is documented in the public header, and
    only those; argument errors come back without a device."""
    src = open(os.path.join(ROOT, "numax_b200", "csrc", "context.cu")).read()
    accepted = set(re.findall(r'strcmp\(key, "([a-z_.]+)"\)', src))
    hdr = open(os.path.join(ROOT, "include", "nmx_la.h")).read()
    block = hdr[hdr.index("Per-context tuning knobs"):hdr.index("NMX_API int nmx_tune_set")]
    documented = set(re.findall(r'"([a-z_]+\.[a-z_]+)"', block))
    assert accepted and accepted == documented, (accepted, documented)
    assert lib.nmx_tune_set(None, b"lu.lookahead", 256) == -1


def test_mojo_shim_binds_only_declared_symbols(lib):
    """Every C symbol the Mojo binding (mojo/nmx_la.mojo) looks up is declared
    in the header and exported by the library, and the shim covers every
    family of entry points numax's gpu=True branches need."""
    src = open(os.path.join(ROOT, "mojo", "nmx_la.mojo")).read()
    used = set(re.findall(r'"(nmx_\w+)"', src))
    declared = set(declared_symbols())
    assert used <= declared, used - declared
    assert all(hasattr(lib, n) for n in used)
    for family in ("nmx_getrf_f64", "nmx_getrs_f64", "nmx_lu_slogdet_f64", "nmx_lu_unpack_f64",
                   "nmx_inverse_f64", "nmx_potrf_f64", "nmx_potrs_f64", "nmx_geqrf_f32",
                   "nmx_orgqr_f32", "nmx_ormqr_f32", "nmx_qr_solve_f32", "nmx_gesv_ir_f64",
                   "nmx_posv_ir_f64", "nmx_potrf_potrs_batched_plan",
                   "nmx_batched_plan_destroy", "nmx_syevj_batched_plan", "nmx_syevj_plan_destroy",
                   "nmx_synchronize", "nmx_memcpy_to_host"):
        assert family in used, family
    # numax's Cholesky raise text, reproduced verbatim.
    assert "cholesky: matrix is not positive definite (non-positive pivot at index " in src
