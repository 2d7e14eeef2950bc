"""Parity of the GPU prover with the oracle: whole proofs (narg + hints) must be
byte-identical to the CPU restatement (oracle/liboracle.so) and, where the
reference build is present (oracle/_ref), to the unmodified reference prover."""
import numpy as np
import pytest

from oracle.refio import ref_available, run_reference
from whirplonk_b200 import ProtocolParameters, prove_once, sample_goldilocks

pytestmark = pytest.mark.gpu


def first_diff(a: bytes, b: bytes):
    for i in range(min(len(a), len(b))):
        if a[i] != b[i]:
            return i
    return None if len(a) == len(b) else min(len(a), len(b))


def make_case(n, seed, npts=1):
    coeffs = sample_goldilocks(seed, 1 << n)
    points = sample_goldilocks(seed + 1000, npts * n * 3).reshape(npts, n, 3)
    return coeffs, points


def check_against_oracle(gpu_ctx, oracle, n, k, rho, sec, pb, seed, npts=1):
    params = ProtocolParameters.cli(security_level=sec, pow_bits=pb, folding_factor=k, log_inv_rate=rho)
    coeffs, points = make_case(n, seed, npts)
    evals = np.array([gpu_ctx.mle_evaluate(coeffs, points[i]) for i in range(npts)], dtype=np.uint64)
    for i in range(npts):
        assert (oracle.mle_eval_base(coeffs, points[i]) == evals[i]).all()
    narg, hints, claim = prove_once(n, params, coeffs, points, evals, ctx=gpu_ctx)
    onarg, ohints = oracle.prove(n, k, rho, sec, pb, points, coeffs, evals)
    assert len(narg) == len(onarg), (len(narg), len(onarg))
    assert narg == onarg, f"narg differs at byte {first_diff(narg, onarg)} of {len(onarg)}"
    assert hints == ohints, f"hints differ at byte {first_diff(hints, ohints)} (len {len(hints)} vs {len(ohints)})"
    return narg, hints, claim


@pytest.mark.parametrize(
    "n,k,rho,sec,pb",
    [
        (4, 4, 1, 100, 20),    # no WHIR rounds, final sumcheck of 0 rounds
        (5, 4, 1, 100, 20),    # final sumcheck of 1 round
        (8, 4, 1, 100, 20),    # one round
        (10, 4, 1, 100, 20),
        (12, 4, 1, 100, 20),
        (9, 2, 2, 80, 10),     # folding factor 2 (rows of 4 / 12 words)
        (12, 3, 2, 100, 20),   # folding factor 3
        (14, 4, 1, 100, 20),
        (13, 1, 1, 64, 16),    # folding factor 1: 12 rounds
        (16, 4, 3, 100, 0),    # rate 1/8, no PoW
    ],
)
def test_prove_matches_oracle(gpu_ctx, oracle, n, k, rho, sec, pb):
    check_against_oracle(gpu_ctx, oracle, n, k, rho, sec, pb, seed=n * 100 + k)


def test_prove_two_statements(gpu_ctx, oracle):
    check_against_oracle(gpu_ctx, oracle, 11, 4, 1, 100, 20, seed=77, npts=2)


def test_prove_c1_config(gpu_ctx, oracle):
    """Config 1: n = 18, folding 4, rate 1/2, 100-bit security, 20 PoW bits."""
    check_against_oracle(gpu_ctx, oracle, 18, 4, 1, 100, 20, seed=18)


def test_prove_deterministic(gpu_ctx, oracle):
    a = check_against_oracle(gpu_ctx, oracle, 10, 4, 2, 100, 20, seed=5)
    b = check_against_oracle(gpu_ctx, oracle, 10, 4, 2, 100, 20, seed=5)
    assert a[0] == b[0] and a[1] == b[1]


def test_special_values(gpu_ctx, oracle):
    """0, 1, p-1, p-2, 2^32-1, 2^32 and reduced 2^64-1 (the reference CUDA tests'
    edge values) spread through the vector."""
    n, P = 12, 0xFFFFFFFF00000001
    coeffs = sample_goldilocks(9, 1 << n)
    specials = np.array([0, 1, P - 1, P - 2, 2**32 - 1, 2**32, (2**64 - 1) - P], dtype=np.uint64)
    coeffs[::7] = np.resize(specials, coeffs[::7].shape)
    point = sample_goldilocks(10, n * 3).reshape(1, n, 3)
    params = ProtocolParameters.cli()
    ev = np.array(gpu_ctx.mle_evaluate(coeffs, point[0]), dtype=np.uint64).reshape(1, 3)
    narg, hints, _ = prove_once(n, params, coeffs, point, ev, ctx=gpu_ctx)
    onarg, ohints = oracle.prove(n, 4, 1, 100, 20, point, coeffs, ev)
    assert narg == onarg and hints == ohints


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("n,rho", [(20, 1), (24, 2)])
def test_prove_matches_reference_large(gpu_ctx, n, rho):
    """Full-size configs against the unmodified reference prover (config 3 is n=24, rate 1/4);
    the reference also verifies its own proof, so the bytes are an accepted proof."""
    params = ProtocolParameters.cli(log_inv_rate=rho)
    coeffs, points = make_case(n, 1234 + n)
    ev = np.array(gpu_ctx.mle_evaluate(coeffs, points[0]), dtype=np.uint64).reshape(1, 3)
    ref = run_reference(n, 4, rho, 100, 20, points, coeffs, verify=True)
    assert (ref.evaluations == ev).all()
    assert ref.verify_ok == 1.0
    narg, hints, _ = prove_once(n, params, coeffs, points, ev, ctx=gpu_ctx)
    assert narg == ref.narg, f"narg differs at byte {first_diff(narg, ref.narg)}"
    assert hints == ref.hints, f"hints differ at byte {first_diff(hints, ref.hints)}"


def test_replayed_graphs_follow_inputs_statements_and_plans(gpu_ctx, oracle):
    """Commit and prove replay graphs captured on a workspace's first call: later
    calls of the same shape with other coefficients and points, with another
    statement count (its own graph) and after an NTT plan change (re-captured)
    must all still equal the oracle's proofs."""
    import ctypes

    from whirplonk_b200 import _lib
    from whirplonk_b200.autotune import load as load_plans

    n, k, rho = 12, 4, 2
    for seed, npts in [(501, 1), (502, 1), (503, 2), (504, 1), (505, 2)]:
        check_against_oracle(gpu_ctx, oracle, n, k, rho, 100, 20, seed=seed, npts=npts)
    L = _lib.load()
    plan = _lib.NttPlan()
    ln = n - k + rho
    _lib.check(L.whirgpu_ntt_get_plan(ln, rho, ctypes.byref(plan)))
    forced = _lib.NttPlan(ln, rho, 2, (1, ln - 1, 0), (255, 255, 255), 3, 0)
    try:
        assert L.whirgpu_ntt_set_plan(ctypes.byref(forced)) == _lib.OK
        check_against_oracle(gpu_ctx, oracle, n, k, rho, 100, 20, seed=506)
    finally:
        L.whirgpu_ntt_clear_plans()
        load_plans()
    check_against_oracle(gpu_ctx, oracle, n, k, rho, 100, 20, seed=507)
