"""Kernel-level Reed-Solomon encoding and matrix commitment (no transcript).

    roots = rs_commit_batch(ctx, vectors, log_expansion=2)   # vectors: (count, 2^log_len) uint64

Each root is the matrix-commitment root irs_commit::commit computes for one
vector (cpp/include/whir/protocols/irs_commit.hpp:402-470): interleaving depth
2^log_depth, codeword length 2^log_expansion * 2^log_len / 2^log_depth, rows
hashed with BLAKE3, Merkle tree over the leaves.
"""
from __future__ import annotations

import ctypes
from typing import List

import numpy as np

from . import _lib
from .whir import Context


def rs_commit_batch(ctx: Context, vectors, log_expansion: int, log_depth: int = 4,
                    on_device_ptr: int | None = None, count: int | None = None,
                    log_len: int | None = None) -> List[bytes]:
    """Roots of `count` vectors of 2^log_len canonical words (host array, or a
    device pointer with count and log_len given)."""
    L = _lib.load()
    if on_device_ptr is None:
        v = np.ascontiguousarray(vectors, dtype=np.uint64)
        if v.ndim == 1:
            v = v.reshape(1, -1)
        count, size = v.shape
        log_len = size.bit_length() - 1
        if size != 1 << log_len:
            raise ValueError("vector length must be a power of two")
        ptr, where = v.ctypes.data, 0
    else:
        if count is None or log_len is None:
            raise ValueError("count and log_len are required with a device pointer")
        ptr, where = int(on_device_ptr), 1
    roots = ctypes.create_string_buffer(32 * count)
    _lib.check(L.whirgpu_rs_commit_batch(ctx.handle, ptr, where, count, log_len, log_expansion, log_depth, roots),
               ctx.handle)
    return [roots.raw[32 * k:32 * k + 32] for k in range(count)]


def rs_encode(ctx: Context, d_vectors: int, count: int, log_len: int, log_expansion: int, log_depth: int,
              d_tmp: int, d_planes: int) -> None:
    """Enqueues the encoder on the context stream (device pointers; see
    whirgpu_rs_encode for the plane layout)."""
    _lib.check(_lib.load().whirgpu_rs_encode(ctx.handle, d_vectors, count, log_len, log_expansion, log_depth, d_tmp,
                                              d_planes), ctx.handle)
