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
