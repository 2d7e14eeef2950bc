"""Host checks of the coset-major codeword order (the Rust crate's order
without rs_in_order): the oracle's transpose_permute is the Rust function
(rust/src/algebra/ntt/transpose.rs:10-15: index -> row + col * rows with
(row, col) = (index / cols, index % cols)), it is a bijection of the codeword
rows, and committed row k of an RS codeword then holds the evaluation at
w_N^perm(k), as rust/src/algebra/ntt/cooley_tukey.rs:375-402 states.  The C
ABI rejects unknown orders without a GPU."""
import ctypes

import numpy as np

from whirplonk_b200 import _lib, sample_goldilocks

P = 0xFFFFFFFF00000001


def test_transpose_permute_is_the_rust_function(oracle):
    rng = np.random.default_rng(9)
    for rows, cols in [(2, 8), (4, 1024), (16, 64), (8, 1), (1, 32)]:
        for k in list(range(min(rows * cols, 64))) + [int(x) for x in rng.integers(0, rows * cols, 32)]:
            assert oracle.transpose_permute(k, rows, cols) == k // cols + (k % cols) * rows
        perm = [oracle.transpose_permute(k, rows, cols) for k in range(rows * cols)]
        assert sorted(perm) == list(range(rows * cols))


def test_committed_rows_are_evaluations_at_permuted_points(oracle):
    depth, m, e = 4, 8, 4
    N = m * e
    v = sample_goldilocks(77, depth * m)
    natural = oracle.rs_encode_base(v, N, depth)  # row i: evaluations at w_N^i of the depth blocks
    w = pow(7, (P - 1) // N, P)
    for k in range(N):
        point = pow(w, oracle.transpose_permute(k, e, m), P)
        row = natural[oracle.transpose_permute(k, e, m)]
        for b in range(depth):
            acc = 0
            for c in reversed(v[b * m:(b + 1) * m].tolist()):
                acc = (acc * point + c) % P
            assert int(row[b]) == acc


def test_codeword_order_setter_rejects_unknown_orders():
    L = _lib.load()
    assert L.whirgpu_set_codeword_order(None, 0) == _lib.E_INVALID
