"""The SHA-2 hash engine (ProtocolParameters.hash_id = SHA-2): leaves, Merkle
nodes and proof of work use SHA-256 (irs_commit.hpp:62-74, whir.hpp:134-140).
GPU proofs must equal the oracle's, the reference prover's committed SHA-2
fixtures and a live reference run; SHA-2 and BLAKE3 proofs mixed in one batch
or server must each equal the same proof made alone."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle.refio import ref_available, run_reference
from whirplonk_b200 import Context, ProtocolParameters, prove_once, sample_goldilocks
from whirplonk_b200.batch import Batch, ProofRequest, Server
from whirplonk_b200.whir import ENGINE_ID_SHA2

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
PROOFS = [c for c in json.load(open(os.path.join(HERE, "golden", "reference_proofs.json")))["cases"]
          if c["hash"] == "sha2"]


def sha2_params(k=4, rho=1, sec=100, pb=20):
    return ProtocolParameters.cli(security_level=sec, pow_bits=pb, folding_factor=k, log_inv_rate=rho,
                                  hash_id=ENGINE_ID_SHA2)


@pytest.mark.parametrize("n,k,rho,sec,pb", [(6, 2, 1, 90, 12), (10, 4, 2, 100, 20), (12, 3, 1, 100, 16),
                                            (14, 4, 3, 100, 20), (16, 4, 1, 100, 0)])
def test_sha2_prove_matches_oracle(gpu_ctx, oracle, n, k, rho, sec, pb):
    coeffs = sample_goldilocks(700 + n, 1 << n)
    points = sample_goldilocks(800 + n, n * 3).reshape(1, n, 3)
    evals = np.array([gpu_ctx.mle_evaluate(coeffs, points[0])], dtype=np.uint64)
    narg, hints, _ = prove_once(n, sha2_params(k, rho, sec, pb), coeffs, points, evals, ctx=gpu_ctx)
    onarg, ohints = oracle.prove(n, k, rho, sec, pb, points, coeffs, evals, sha2=True)
    assert narg == onarg and hints == ohints
    bnarg, _, _ = prove_once(n, ProtocolParameters.cli(security_level=sec, pow_bits=pb, folding_factor=k,
                                                       log_inv_rate=rho), coeffs, points, evals, ctx=gpu_ctx)
    assert bnarg != narg  # the engine changes the commitment


@pytest.mark.parametrize("case", PROOFS, ids=lambda c: f"n{c['n']}r{c['rho']}p{c['pow_bits']}")
def test_sha2_prove_matches_reference_fixtures(gpu_ctx, case):
    n = case["n"]
    coeffs = sample_goldilocks(case["seed"], 1 << n)
    points = sample_goldilocks(case["seed"] + 5000, case["n_points"] * n * 3).reshape(case["n_points"], n, 3)
    evals = np.array(case["evaluations"], dtype=np.uint64)
    narg, hints, _ = prove_once(n, sha2_params(case["k"], case["rho"], case["security"], case["pow_bits"]), coeffs,
                                points, evals, ctx=gpu_ctx)
    assert hashlib.sha256(narg).hexdigest() == case["narg_sha256"]
    assert hashlib.sha256(hints).hexdigest() == case["hints_sha256"]


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_sha2_prove_matches_live_reference(gpu_ctx):
    n, rho = 18, 2
    coeffs = sample_goldilocks(4321, 1 << n)
    points = sample_goldilocks(4322, n * 3).reshape(1, n, 3)
    ref = run_reference(n, 4, rho, 100, 20, points, coeffs, verify=True, sha2=True)
    assert ref.verify_ok == 1.0
    narg, hints, _ = prove_once(n, sha2_params(rho=rho), coeffs, points, ref.evaluations, ctx=gpu_ctx)
    assert narg == ref.narg and hints == ref.hints


def test_sha2_and_blake3_mixed_batch_and_server():
    ctx = Context(0)
    try:
        reqs, expected = [], []
        for i, (n, sha2) in enumerate([(10, True), (10, False), (12, True), (9, False), (11, True), (12, False)]):
            p = sha2_params(rho=1 + i % 3) if sha2 else ProtocolParameters.cli(log_inv_rate=1 + i % 3)
            c = sample_goldilocks(9100 + i, 1 << n)
            pts = sample_goldilocks(9200 + i, n * 3).reshape(1, n, 3)
            ev = np.array(ctx.mle_evaluate(c, pts), dtype=np.uint64).reshape(1, 3)
            reqs.append(ProofRequest(n, p, c, pts, ev))
            expected.append(prove_once(n, p, c, pts, ev, ctx=ctx)[:2])
        with Batch(ctx, reqs, Batch.GRAPH) as b:
            b.run()
            for i in range(len(reqs)):
                assert b.proof(i) == expected[i], f"batched request {i}"
        srv = Server(ctx, hbm_budget=0, max_inflight=4)
        tickets = [srv.submit(r) for r in reqs]
        for i, t in enumerate(tickets):
            res = srv.poll(t, timeout_ms=60_000)
            assert res.status == 0 and (res.narg, res.hints) == expected[i], f"served request {i}"
        srv.close()
    finally:
        ctx.close()
