"""numax_b200 -- numax.linalg's dense-factorization hot path on B200 (sm_100a).

A drop-in for numax's linalg entry points over CUDA tensors: every call goes
through the C ABI of libnmxla.so (include/nmx_la.h), hand-written CUDA for
sm_100a.  There is no CPU fallback; without the built library or an sm_100
device the calls raise.
"""
from . import _lib
from .batched import (CholeskySolveBatch, EighBatch, cholesky_solve_batched, eigh_batched,
                      ragged_offsets)

__all__ = ["CholeskySolveBatch", "EighBatch", "cholesky_solve_batched", "eigh_batched",
           "ragged_offsets"]
