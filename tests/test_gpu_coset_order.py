"""The Rust crate's coset-major codeword order (whirgpu_set_codeword_order).

Without its `rs_in_order` feature the Rust reference commits codeword rows
coset-major (rust/src/algebra/ntt/cooley_tukey.rs:375-480): committed row k is
the evaluation at w_N^(k / m + (k mod m) N / m) for message length m
(transpose_permute, rust/src/algebra/ntt/transpose.rs:10-15), and the opened
rows and their evaluation points follow.  There is no Rust toolchain and no
Rust golden in this order, so parity is pinned to the oracle's restatement
only: every GPU proof made in that order must equal the oracle's proof made in
that order.  The natural order stays the default and is what every other test
checks against the C++ reference."""
import numpy as np
import pytest

from whirplonk_b200 import Context, ProtocolParameters, prove_once, sample_goldilocks
from whirplonk_b200.whir import ENGINE_ID_BLAKE3, ENGINE_ID_SHA2

pytestmark = pytest.mark.gpu


def _params(k, rho, sec, pb, batch=1, sha2=False, unique=False):
    return ProtocolParameters(unique, rho, k, k, sec, pb, batch, ENGINE_ID_SHA2 if sha2 else ENGINE_ID_BLAKE3)


@pytest.fixture
def coset_ctx(oracle):
    ctx = Context(0)
    ctx.set_codeword_order(Context.ORDER_COSET_MAJOR)
    oracle.set_coset_major(True)
    try:
        yield ctx
    finally:
        oracle.set_coset_major(False)
        ctx.close()


@pytest.mark.parametrize("n,k,rho,sec,pb,sha2", [
    (8, 4, 1, 100, 20, False), (12, 4, 1, 100, 20, False), (14, 4, 2, 100, 20, False),
    (16, 4, 3, 100, 0, False), (13, 3, 2, 90, 16, True), (10, 2, 1, 80, 10, False),
])
def test_coset_major_proofs_match_oracle(coset_ctx, oracle, n, k, rho, sec, pb, sha2):
    p = _params(k, rho, sec, pb, sha2=sha2)
    coeffs = sample_goldilocks(3100 + n, 1 << n)
    points = sample_goldilocks(3200 + n, n * 3).reshape(1, n, 3)
    evals = np.array([coset_ctx.mle_evaluate(coeffs, points[0])], dtype=np.uint64)
    narg, hints, _ = prove_once(n, p, coeffs, points, evals, ctx=coset_ctx)
    onarg, ohints = oracle.prove(n, k, rho, sec, pb, points, coeffs, evals, sha2=sha2)
    assert narg == onarg and hints == ohints


def test_coset_major_several_vectors_and_witnesses(coset_ctx, oracle):
    n, k, rho, batch, nwit = 11, 4, 1, 3, 2
    p = _params(k, rho, 100, 20, batch=batch)
    nvec = batch * nwit
    coeffs = sample_goldilocks(3300, nvec << n).reshape(nvec, 1 << n)
    points = sample_goldilocks(3301, n * 3).reshape(1, n, 3)
    evals = np.array([coset_ctx.mle_evaluate(coeffs[v], points[0]) for v in range(nvec)], dtype=np.uint64)
    narg, hints, _ = prove_once(n, p, coeffs, points, evals, ctx=coset_ctx, num_witnesses=nwit)
    onarg, ohints = oracle.prove_multi(n, k, rho, 100, 20, points, coeffs, evals, batch, nwit)
    assert narg == onarg and hints == ohints


def test_coset_major_differs_from_natural_and_order_is_per_context(gpu_ctx, coset_ctx, oracle):
    n = 12
    p = _params(4, 1, 100, 20)
    coeffs = sample_goldilocks(3400, 1 << n)
    points = sample_goldilocks(3401, n * 3).reshape(1, n, 3)
    evals = np.array([gpu_ctx.mle_evaluate(coeffs, points[0])], dtype=np.uint64)
    coset = prove_once(n, p, coeffs, points, evals, ctx=coset_ctx)[:2]
    natural = prove_once(n, p, coeffs, points, evals, ctx=gpu_ctx)[:2]
    assert coset != natural
    oracle.set_coset_major(False)
    assert natural == oracle.prove(n, 4, 1, 100, 20, points, coeffs, evals)
    oracle.set_coset_major(True)
    coset_ctx.set_codeword_order(Context.ORDER_NATURAL)
    assert prove_once(n, p, coeffs, points, evals, ctx=coset_ctx)[:2] == natural
