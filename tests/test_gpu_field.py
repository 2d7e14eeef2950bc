"""Device Goldilocks / Ext3 arithmetic (carry-chain PTX in csrc/gl.cuh) against
exact integer arithmetic, on edge values and random operands."""
import ctypes

import numpy as np
import pytest

from whirplonk_b200 import _lib, sample_goldilocks

pytestmark = pytest.mark.gpu
P = 0xFFFFFFFF00000001
EDGE = [0, 1, 2, P - 1, P - 2, 2**32 - 1, 2**32, 2**32 + 1, 2**63, 2**64 - 2**32, (2**64 - 1) - P, 0xFFFFFFFF00000000]


def run(op, a, b):
    L = _lib.load()
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    n = a.size // (3 if op == 3 else 1)
    out = np.zeros_like(a)
    assert L.whirgpu_debug_field_ops(a.ctypes.data, b.ctypes.data, out.ctypes.data, n, op) == _lib.OK
    return out


def operands(count, seed):
    a = sample_goldilocks(seed, count)
    b = sample_goldilocks(seed + 1, count)
    e = np.array(EDGE, dtype=np.uint64)
    ea, eb = np.meshgrid(e, e)
    return np.concatenate([ea.ravel(), a]), np.concatenate([eb.ravel(), b])


@pytest.mark.parametrize("op,fn", [(0, lambda x, y: (x + y) % P), (1, lambda x, y: (x - y) % P),
                                   (2, lambda x, y: (x * y) % P)])
def test_base_field_ops(op, fn):
    a, b = operands(200_000, 40 + op)
    got = run(op, a, b)
    want = [fn(int(x), int(y)) for x, y in zip(a.tolist(), b.tolist())]
    assert got.tolist() == want


def test_mul_accepts_noncanonical_operands():
    # gl_mul reduces any 64-bit operands (used after lazy sums); compare on words >= p too.
    rng = np.random.default_rng(3)
    a = np.concatenate([rng.integers(0, 2**63, 50_000, dtype=np.uint64) * 2 + 1,
                        np.array([2**64 - 1, P, P + 1], dtype=np.uint64)])
    b = np.concatenate([rng.integers(0, 2**63, 50_000, dtype=np.uint64) * 2,
                        np.array([2**64 - 1, 2**64 - 1, P], dtype=np.uint64)])
    got = run(2, a, b)
    assert got.tolist() == [(int(x) * int(y)) % P for x, y in zip(a.tolist(), b.tolist())]


def test_ext3_mul(oracle):
    a = sample_goldilocks(70, 3 * 20_000)
    b = sample_goldilocks(71, 3 * 20_000)
    got = run(3, a, b).reshape(-1, 3)
    A, B = a.reshape(-1, 3), b.reshape(-1, 3)
    for i in range(0, A.shape[0], 97):
        assert got[i].tolist() == oracle.e3_mul(A[i].tolist(), B[i].tolist())
    # X^3 = 2: (0,1,0)^3 = (2,0,0)
    x = np.array([0, 1, 0], dtype=np.uint64)
    x2 = run(3, x, x)
    assert run(3, x2, x).tolist() == [2, 0, 0]
