"""numax.io's `.npy` interchange over torch tensors, on libnmxla.so.

Mirrors numax's `from numax.io import numpy` namespace
(numax/io/npy.mojo:262-453):

    numpy.save(a, path)                      npy.mojo:273-346
    numpy.load(path, dtype, *dims, device)   npy.mojo:349-397
    numpy.load_dyn(path, dtype, rank, device) npy.mojo:400-453

A CUDA tensor streams between the file and HBM through the library's pinned
staging (nmx_npy_load / nmx_npy_save); a CPU tensor is read or written by the
same library code with no CUDA call.  `device=None` loads to the host, as
numax's `ctx=None` does.  Files are byte-identical to numpy.save's, and the
failures numax raises on (bad magic / .npz, Fortran order, big-endian or
mismatched descr, wrong rank or shape, short payload) raise here with
numax's messages.

A (count, n, n) stack saved by numpy loads straight into the batched
Cholesky's A layout (row-major matrices back to back), so
`cholesky_solve_batched` can take a `numpy.load` result as it is.
"""
from __future__ import annotations

import ctypes as C
import os

import torch

from . import _lib

_CODE = {
    torch.float32: 0, torch.float64: 1, torch.float16: 2, torch.int8: 3, torch.int16: 4,
    torch.int32: 5, torch.int64: 6, torch.uint8: 7, torch.uint16: 8, torch.uint32: 9,
    torch.uint64: 10, torch.bool: 11, torch.bfloat16: 12,
}
_MAX_RANK = 64


class NpyError(ValueError):
    """A `.npy` file that is not what the call asked for, or an I/O failure."""


def _raise(fn, code):
    raise NpyError(_lib.last_error() or f"{fn} failed ({code})")


def _target(device):
    """(ctx, stream, torch.device) for a load/save on `device` (None = host)."""
    if device is None:
        return None, None, torch.device("cpu")
    dev = torch.device(device)
    if dev.type == "cpu":
        return None, None, dev
    if dev.type != "cuda":
        raise ValueError(f"device must be CUDA or the host, got {dev}")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    return _lib.context(dev.index), torch.cuda.current_stream(dev).cuda_stream, dev


def _path(path) -> bytes:
    return os.fsencode(os.fspath(path))


class numpy:  # noqa: N801 -- numax's namespace name
    """NumPy `.npy` interchange, namespaced as numax's `numax.io.numpy`."""

    @staticmethod
    def save(a: torch.Tensor, path) -> None:
        """Write `a` (row-major) to `path` as numpy.save would."""
        if not isinstance(a, torch.Tensor):
            raise TypeError("a must be a torch.Tensor")
        if a.dtype not in _CODE:
            raise TypeError(f"numax.io.numpy.save: {a.dtype} has no .npy representation")
        a = a.contiguous()
        ctx, stream, _ = _target(a.device if a.device.type == "cuda" else None)
        shape = (C.c_int64 * max(a.dim(), 1))(*a.shape)
        rc = _lib.load().nmx_npy_save(ctx, _path(path), _CODE[a.dtype], a.dim(), shape,
                                      C.c_void_p(a.data_ptr() if a.numel() else 0), stream)
        if rc < 0:
            _raise("nmx_npy_save", rc)

    @staticmethod
    def _load(path, dtype, dims, device):
        if dtype not in _CODE:
            raise TypeError(f"numax.io.numpy.load: {dtype} has no .npy representation")
        rank = len(dims)
        if rank > _MAX_RANK:
            raise ValueError(f"rank {rank} exceeds {_MAX_RANK}")
        lib = _lib.load()
        # The header first, so the destination can be sized from the file.
        fcode, frank = C.c_int(), C.c_int()
        fshape = (C.c_int64 * _MAX_RANK)()
        rc = lib.nmx_npy_header(_path(path), C.byref(fcode), C.byref(frank), fshape, _MAX_RANK,
                                None)
        want = (C.c_int64 * max(rank, 1))(*dims)
        if rc < 0:
            # The load's own checks name the first failure in numax's order
            # (descr before Fortran order before the payload and the shape).
            msg = _lib.last_error()
            rc2 = lib.nmx_npy_load(None, _path(path), _CODE[dtype], rank, want, None, 0, None)
            raise NpyError(_lib.last_error() if rc2 < 0 else msg)
        ctx, stream, dev = _target(device)
        file_dims = [fshape[i] for i in range(frank.value)]
        # Room for the file's payload when it is the requested type and rank;
        # otherwise the library reports the mismatch before touching dst.
        fits = (fcode.value == _CODE[dtype] and frank.value == rank
                and all(d < 0 or d == f for d, f in zip(dims, file_dims)))
        alloc = file_dims if fits else [0]
        out = torch.empty(alloc, dtype=dtype, device=dev)
        nbytes = out.numel() * out.element_size()
        rc = lib.nmx_npy_load(ctx, _path(path), _CODE[dtype], rank, want,
                              C.c_void_p(out.data_ptr() if nbytes else 0), nbytes, stream)
        if rc < 0:
            _raise("nmx_npy_load", rc)
        return out

    @staticmethod
    def load(path, dtype: torch.dtype, *dims: int, device=None) -> torch.Tensor:
        """Read `path` at exactly the shape `dims`; raises if the file differs."""
        if any(d < 0 for d in dims):
            raise ValueError("dims must be non-negative")
        return numpy._load(path, dtype, list(dims), device)

    @staticmethod
    def load_dyn(path, dtype: torch.dtype, rank: int, device=None) -> torch.Tensor:
        """Read `path` at the shape its header carries; only the rank is checked."""
        return numpy._load(path, dtype, [-1] * rank, device)
