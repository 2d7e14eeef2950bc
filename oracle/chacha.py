"""Test infrastructure: the seeded Goldilocks sampler restated in numpy.

The benchmark's synthetic inputs are 64-bit words of a ChaCha20 keystream
(RFC 8439 block function; key = the seed as 8 little-endian bytes then 24 zero
bytes, nonce 0, block counter from 0); each little-endian word below
p = 2^64 - 2^32 + 1 is taken and the others are skipped.  The library's
whirgpu_sample_goldilocks computes the same stream; this restatement lets the
reference arm of the benchmark and the CPU baseline draw their inputs without
loading the GPU library (tests/test_capi_cpu.py checks the two agree, and an
RFC 8439 known-answer vector pins the block function).
"""
from __future__ import annotations

import numpy as np

P = 0xFFFFFFFF00000001
_CONST = np.array([0x61707865, 0x3320646E, 0x79622D32, 0x6B206574], dtype=np.uint32)


def _rotl(x, r):
    return (x << np.uint32(r)) | (x >> np.uint32(32 - r))


def chacha20_blocks(key_words, counter0: int, count: int, nonce=(0, 0, 0)) -> np.ndarray:
    """`count` consecutive 64-byte ChaCha20 blocks from block counter
    `counter0`, as a (count, 16) array of little-endian uint32 words."""
    assert counter0 + count <= 1 << 32, "block counter would wrap"
    s = np.empty((16, count), dtype=np.uint32)
    s[0:4] = _CONST[:, None]
    s[4:12] = np.asarray(key_words, dtype=np.uint32)[:, None]
    s[12] = np.arange(counter0, counter0 + count, dtype=np.uint64).astype(np.uint32)
    s[13:16] = np.asarray(nonce, dtype=np.uint32)[:, None]
    x = [s[i].copy() for i in range(16)]

    def qr(a, b, c, d):
        x[a] += x[b]; x[d] ^= x[a]; x[d] = _rotl(x[d], 16)
        x[c] += x[d]; x[b] ^= x[c]; x[b] = _rotl(x[b], 12)
        x[a] += x[b]; x[d] ^= x[a]; x[d] = _rotl(x[d], 8)
        x[c] += x[d]; x[b] ^= x[c]; x[b] = _rotl(x[b], 7)

    with np.errstate(over="ignore"):
        for _ in range(10):
            qr(0, 4, 8, 12); qr(1, 5, 9, 13); qr(2, 6, 10, 14); qr(3, 7, 11, 15)
            qr(0, 5, 10, 15); qr(1, 6, 11, 12); qr(2, 7, 8, 13); qr(3, 4, 9, 14)
        out = np.empty((count, 16), dtype=np.uint32)
        for i in range(16):
            out[:, i] = x[i] + s[i]
    return out


def sample_goldilocks(seed: int, count: int) -> np.ndarray:
    """`count` uniform Goldilocks words from the seeded ChaCha20 stream."""
    key = [seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF, 0, 0, 0, 0, 0, 0]
    out = np.empty(count, dtype=np.uint64)
    got, counter = 0, 0
    while got < count:
        # a word is rejected with probability 2^-32: one spare block per 2^26 words
        blocks = (count - got + 7) // 8 + 1 + (count - got) // (1 << 26)
        words = chacha20_blocks(key, counter, blocks).view(np.uint64).reshape(-1)
        counter += blocks
        keep = words[words < np.uint64(P)]
        take = min(count - got, keep.size)
        out[got:got + take] = keep[:take]
        got += take
    return out
