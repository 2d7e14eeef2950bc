"""Unique decoding (ProtocolParameters.unique_decoding: no OOD samples) and
proofs without any constraint: with no linear form the prover squeezes the
folding randomness directly, runs the skip-PoW and folds the vector without a
sumcheck (whir_prover.hpp:211-218).  GPU proofs must equal the reference
prover's fixtures, the oracle and a live reference run, alone and in a batch."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle.refio import ref_available, run_reference
from tests.golden.forms import form_inputs
from whirplonk_b200 import Context, Covector, MultilinearExtension, ProtocolParameters, prove_once
from whirplonk_b200.batch import Batch, ProofRequest
from whirplonk_b200.whir import ENGINE_ID_BLAKE3, ENGINE_ID_SHA2

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
UNIQUE = json.load(open(os.path.join(HERE, "golden", "reference_proofs.json")))["unique"]


def params(k=4, rho=1, batch=1, sha2=False):
    return ProtocolParameters(True, rho, k, k, 100, 20, batch, ENGINE_ID_SHA2 if sha2 else ENGINE_ID_BLAKE3)


def to_forms(forms):
    return [MultilinearExtension(d) if kind == "mle" else Covector(d) for kind, d in forms]


@pytest.mark.parametrize("case", UNIQUE, ids=lambda c: f"n{c['n']}-{'-'.join(c['kinds']) or 'none'}"
                                                       f"-b{c['batch_size']}w{c['num_witnesses']}{c['hash']}")
def test_unique_decoding_matches_reference_fixtures(gpu_ctx, case):
    n, batch, nwit = case["n"], case["batch_size"], case["num_witnesses"]
    coeffs, forms = form_inputs(n, case["seed"], case["kinds"], batch * nwit)
    evals = np.array(case["evaluations"], dtype=np.uint64).reshape(-1, 3)
    narg, hints, claim = prove_once(n, params(case["k"], case["rho"], batch, case["hash"] == "sha2"), coeffs, None,
                                    evals, ctx=gpu_ctx, num_witnesses=nwit, forms=to_forms(forms))
    assert (len(narg), len(hints)) == (case["narg_len"], case["hints_len"])
    assert hashlib.sha256(narg).hexdigest() == case["narg_sha256"]
    assert hashlib.sha256(hints).hexdigest() == case["hints_sha256"]
    if "narg" in case:
        assert narg.hex() == case["narg"] and hints.hex() == case["hints"]
    assert len(claim.evaluation_point) == n


@pytest.mark.parametrize("n,k,rho,batch,nwit", [(8, 4, 1, 1, 1), (13, 3, 2, 1, 1), (15, 4, 1, 3, 2),
                                                (20, 4, 1, 1, 1), (4, 4, 1, 2, 1)])
def test_statement_free_matches_oracle(gpu_ctx, oracle, n, k, rho, batch, nwit):
    coeffs, _ = form_inputs(n, 7300 + n, (), batch * nwit)
    empty = np.zeros((0, 3), dtype=np.uint64)
    narg, hints, claim = prove_once(n, params(k, rho, batch), coeffs, None, empty, ctx=gpu_ctx, num_witnesses=nwit,
                                    forms=[])
    onarg, ohints = oracle.prove_forms(n, k, rho, 100, 20, [], coeffs, empty, batch, nwit, unique=True)
    assert narg == onarg and hints == ohints
    assert claim.rlc_coefficients == []


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_statement_free_matches_live_reference(gpu_ctx):
    n = 18
    coeffs, _ = form_inputs(n, 7400, (), 2)
    ref = run_reference(n, 4, 1, 100, 20, None, coeffs, verify=True, batch_size=2, forms=[], unique=True)
    assert ref.verify_ok == 1.0
    narg, hints, _ = prove_once(n, params(batch=2), coeffs, None, np.zeros((0, 3), dtype=np.uint64), ctx=gpu_ctx,
                                forms=[])
    assert narg == ref.narg and hints == ref.hints


def test_unique_decoding_in_a_batch():
    ctx = Context(0)
    try:
        reqs, expected = [], []
        for i, (n, npts) in enumerate([(10, 0), (12, 1), (9, 0), (14, 2)]):
            coeffs, forms = form_inputs(n, 7500 + i, ("mle",) * npts, 1)
            pts = np.array([d for _, d in forms], dtype=np.uint64).reshape(npts, n, 3)
            ev = np.array([ctx.mle_evaluate(coeffs[0], pts[j]) for j in range(npts)], dtype=np.uint64).reshape(-1, 3)
            reqs.append(ProofRequest(n, params(rho=1 + i % 2), coeffs[0], pts, ev))
            expected.append(prove_once(n, params(rho=1 + i % 2), coeffs[0], pts, ev, ctx=ctx)[:2])
        with Batch(ctx, reqs, Batch.GRAPH) as b:
            b.run()
            for i in range(len(reqs)):
                assert b.proof(i) == expected[i], f"batched request {i}"
    finally:
        ctx.close()
