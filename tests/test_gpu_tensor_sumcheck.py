"""The initial sumcheck by block evaluation (k_sc_tensor.cu) against the oracle.

A proof of one committed vector whose statement holds only MultilinearExtension
forms takes this path whenever the initial sumcheck has 1 to 5 rounds without
round PoW and at least 6 variables stay after it; its covector terms (the
forms, then the OOD points) are evaluated block by block in passes of two.
These cases cover one to nine terms (one to five passes, an odd last pass),
every folding factor from 1 to 5, the smallest remainder (n = k + 6, rows of
64 words), unique decoding (no OOD term), the base field as target field and a
large case; every proof must equal the oracle's byte for byte."""
import numpy as np
import pytest

from whirplonk_b200 import FIELD_GOLDILOCKS1, ProtocolParameters, prove_once, sample_goldilocks
from whirplonk_b200.whir import ENGINE_ID_BLAKE3

pytestmark = pytest.mark.gpu


def _case(ctx, n, npts, seed, base_points=False):
    coeffs = sample_goldilocks(seed, 1 << n)
    points = sample_goldilocks(seed + 1, npts * n * 3).reshape(npts, n, 3)
    if base_points:
        points[:, :, 1:] = 0
    evals = np.array([ctx.mle_evaluate(coeffs, points[i]) for i in range(npts)], dtype=np.uint64)
    return coeffs, points, evals


@pytest.mark.parametrize("n,k,rho,npts", [
    (10, 4, 1, 1),   # n = k + 6: rows of 64 words, one row per block
    (11, 5, 1, 1),   # folding factor 5: 32 blocks
    (12, 3, 2, 2),   # three terms: passes of two and one
    (13, 2, 1, 3),   # four terms
    (9, 1, 1, 2),    # folding factor 1: one block split, 8 rounds
    (15, 4, 3, 8),   # nine terms: five passes, the last of one
    (18, 4, 1, 1),   # config 1's shape
    (22, 4, 2, 1),   # rows of 1024 words, 2^12 rows per block
])
def test_tensor_initial_sumcheck_matches_oracle(gpu_ctx, oracle, n, k, rho, npts):
    p = ProtocolParameters.cli(security_level=100, pow_bits=20, folding_factor=k, log_inv_rate=rho)
    coeffs, points, evals = _case(gpu_ctx, n, npts, 4100 + 37 * n + npts)
    narg, hints, _ = prove_once(n, p, coeffs, points, evals, ctx=gpu_ctx)
    onarg, ohints = oracle.prove(n, k, rho, 100, 20, points, coeffs, evals)
    assert narg == onarg and hints == ohints


def test_tensor_initial_sumcheck_unique_decoding(gpu_ctx, oracle):
    """No OOD sample: the terms are the two forms alone."""
    n, k, rho = 12, 4, 1
    p = ProtocolParameters(True, rho, k, k, 100, 20, 1, ENGINE_ID_BLAKE3)
    coeffs, points, evals = _case(gpu_ctx, n, 2, 4300)
    narg, hints, _ = prove_once(n, p, coeffs, points, evals, ctx=gpu_ctx)
    forms = [("mle", points[i]) for i in range(2)]
    onarg, ohints = oracle.prove_forms(n, k, rho, 100, 20, forms, coeffs, evals, unique=True)
    assert narg == onarg and hints == ohints


def test_tensor_initial_sumcheck_base_field_target(gpu_ctx, oracle):
    """Identity<Goldilocks>: every term and challenge in the base field.  Over the
    64-bit field the derived PoW bits grow with the security level, so the level is
    kept low enough for the grinds to stay short (as in test_gpu_field1)."""
    n, k, rho, sec, pb = 13, 4, 1, 36, 12
    p = ProtocolParameters.cli(security_level=sec, pow_bits=pb, folding_factor=k, log_inv_rate=rho)
    coeffs, points, evals = _case(gpu_ctx, n, 2, 4400, base_points=True)
    narg, hints, _ = prove_once(n, p, coeffs, points, evals, ctx=gpu_ctx, target_field=FIELD_GOLDILOCKS1)
    forms = [("mle", points[i]) for i in range(2)]
    onarg, ohints = oracle.prove_forms(n, k, rho, sec, pb, forms, coeffs, evals, field1=True)
    assert narg == onarg and hints == ohints
