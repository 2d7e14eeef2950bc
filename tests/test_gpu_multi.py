"""Several committed vectors (ProtocolParameters.batch_size > 1) and several
witnesses proven together (Config::prove over witnesses.size() commitments,
whir_prover.hpp:56-200): rows of batch_size * 2^k elements (BLAKE3 tree mode
above 1024 bytes), OOD values of every vector, OOD completion across
witnesses, the vector RLC fused into the covector pass, the Ext3 initial
sumcheck and the first opening weighted by vector_rlc (x) eq.  GPU proofs must
equal the reference prover's fixtures, the oracle and a live reference run;
batch_size > 1 requests in a batch or server must equal the same proof alone."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle.refio import ref_available, run_reference
from whirplonk_b200 import Context, ProtocolParameters, prove_once, sample_goldilocks
from whirplonk_b200._lib import WhirGpuError
from whirplonk_b200.batch import Batch, ProofRequest, Server
from whirplonk_b200.whir import ENGINE_ID_BLAKE3, ENGINE_ID_SHA2

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
MULTI = json.load(open(os.path.join(HERE, "golden", "reference_proofs.json")))["multi"]


def params(k=4, rho=1, sec=100, pb=20, batch=1, sha2=False):
    return ProtocolParameters(False, rho, k, k, sec, pb, batch, ENGINE_ID_SHA2 if sha2 else ENGINE_ID_BLAKE3)


def mle_evals(ctx, coeffs, points):
    """Form-major claimed values: form f on vector v at f * V + v."""
    return np.array([ctx.mle_evaluate(coeffs[v], points[f]) for f in range(points.shape[0])
                     for v in range(coeffs.shape[0])], dtype=np.uint64).reshape(-1, 3)


@pytest.mark.parametrize("case", MULTI, ids=lambda c: f"n{c['n']}k{c['k']}r{c['rho']}"
                                                      f"b{c['batch_size']}w{c['num_witnesses']}{c['hash']}")
def test_multi_vector_prove_matches_reference_fixtures(gpu_ctx, case):
    n, batch, nwit = case["n"], case["batch_size"], case["num_witnesses"]
    nvec = batch * nwit
    coeffs = sample_goldilocks(case["seed"], nvec << n).reshape(nvec, 1 << n)
    points = sample_goldilocks(case["seed"] + 5000, case["n_points"] * n * 3).reshape(case["n_points"], n, 3)
    evals = np.array(case["evaluations"], dtype=np.uint64).reshape(-1, 3)
    if case["n_points"]:
        assert np.array_equal(mle_evals(gpu_ctx, coeffs, points), evals)
    p = params(case["k"], case["rho"], case["security"], case["pow_bits"], batch, case["hash"] == "sha2")
    narg, hints, _ = prove_once(n, p, coeffs, points, evals, ctx=gpu_ctx, num_witnesses=nwit)
    assert (len(narg), len(hints)) == (case["narg_len"], case["hints_len"])
    assert hashlib.sha256(narg).hexdigest() == case["narg_sha256"]
    assert hashlib.sha256(hints).hexdigest() == case["hints_sha256"]
    if "narg" in case:
        assert narg.hex() == case["narg"] and hints.hex() == case["hints"]


@pytest.mark.parametrize("n,k,rho,batch,nwit,npts,sha2", [
    (8, 4, 1, 2, 1, 1, False), (13, 4, 1, 3, 2, 2, False), (14, 5, 2, 8, 1, 1, False),
    (12, 4, 1, 32, 1, 1, False),   # 4096-byte rows: four BLAKE3 chunks
    (11, 6, 1, 4, 2, 1, False),    # 2048-byte rows from the folding factor
    (10, 3, 2, 4, 8, 1, True),     # eight witnesses, SHA-256
    (17, 4, 1, 2, 2, 3, False), (4, 4, 1, 5, 1, 1, False),  # no round: the final opening covers the batch
    (9, 4, 1, 64, 1, 2, False),    # the 64-vector limit: 8192-byte rows, eight BLAKE3 chunks
    (9, 4, 1, 8, 8, 1, True),      # 8 witnesses x 8 vectors, SHA-256
])
def test_multi_vector_prove_matches_oracle(gpu_ctx, oracle, n, k, rho, batch, nwit, npts, sha2):
    nvec = batch * nwit
    coeffs = sample_goldilocks(3000 + n + nvec, nvec << n).reshape(nvec, 1 << n)
    points = sample_goldilocks(3100 + n, npts * n * 3).reshape(npts, n, 3)
    evals = mle_evals(gpu_ctx, coeffs, points)
    narg, hints, claim = prove_once(n, params(k, rho, batch=batch, sha2=sha2), coeffs, points, evals, ctx=gpu_ctx,
                                    num_witnesses=nwit)
    onarg, ohints = oracle.prove_multi(n, k, rho, 100, 20, points, coeffs, evals, batch, nwit, sha2=sha2)
    assert narg == onarg and hints == ohints
    assert len(claim.evaluation_point) == n


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_multi_vector_prove_matches_live_reference(gpu_ctx):
    n, batch, nwit = 18, 4, 2
    nvec = batch * nwit
    coeffs = sample_goldilocks(5150, nvec << n).reshape(nvec, 1 << n)
    points = sample_goldilocks(5151, 2 * n * 3).reshape(2, n, 3)
    ref = run_reference(n, 4, 1, 100, 20, points, coeffs, verify=True, batch_size=batch, num_witnesses=nwit)
    assert ref.verify_ok == 1.0
    narg, hints, _ = prove_once(n, params(batch=batch), coeffs, points, ref.evaluations, ctx=gpu_ctx,
                                num_witnesses=nwit)
    assert narg == ref.narg and hints == ref.hints


def test_multi_vector_full_size_properties(gpu_ctx):
    """n = 22 with 4 vectors: the proof is deterministic, and a batch of one
    vector differs from the same vector committed with a second one."""
    n, batch = 22, 4
    coeffs = sample_goldilocks(6160, batch << n).reshape(batch, 1 << n)
    points = sample_goldilocks(6161, n * 3).reshape(1, n, 3)
    evals = mle_evals(gpu_ctx, coeffs, points)
    a = prove_once(n, params(batch=batch), coeffs, points, evals, ctx=gpu_ctx)[:2]
    b = prove_once(n, params(batch=batch), coeffs, points, evals, ctx=gpu_ctx)[:2]
    assert a == b
    one = prove_once(n, params(), coeffs[0], points, evals[:1], ctx=gpu_ctx)[:2]
    assert one[0][:32] != a[0][:32]  # the root commits to every row


def test_multi_vector_device_input(gpu_ctx):
    import torch

    n, batch, nwit = 12, 3, 2
    nvec = batch * nwit
    coeffs = sample_goldilocks(6170, nvec << n).reshape(nvec, 1 << n)
    points = sample_goldilocks(6171, n * 3).reshape(1, n, 3)
    evals = mle_evals(gpu_ctx, coeffs, points)
    host = prove_once(n, params(batch=batch), coeffs, points, evals, ctx=gpu_ctx, num_witnesses=nwit)[:2]
    dev = torch.from_numpy(coeffs.view(np.int64).copy()).cuda()
    torch.cuda.synchronize()
    got = prove_once(n, params(batch=batch), None, points, evals, ctx=gpu_ctx, on_device_ptr=dev.data_ptr(),
                     num_witnesses=nwit)[:2]
    assert got == host


def test_multi_vector_batch_and_server_identity():
    ctx = Context(0)
    try:
        reqs, expected = [], []
        for i, (n, batch) in enumerate([(10, 2), (11, 1), (12, 4), (9, 3), (12, 1), (10, 8)]):
            p = params(rho=1 + i % 2, batch=batch)
            c = sample_goldilocks(9400 + i, batch << n).reshape(batch, 1 << n)
            pts = sample_goldilocks(9500 + i, n * 3).reshape(1, n, 3)
            ev = mle_evals(ctx, c, pts)
            reqs.append(ProofRequest(n, p, c, pts, ev))
            expected.append(prove_once(n, p, c, pts, ev, ctx=ctx)[:2])
        with Batch(ctx, reqs, Batch.GRAPH) as b:
            b.run()
            for i in range(len(reqs)):
                assert b.proof(i) == expected[i], f"batched request {i}"
        srv = Server(ctx, hbm_budget=8 << 30, max_inflight=4)
        try:
            tickets = [srv.submit(r) for r in reqs]
            for i, t in enumerate(tickets):
                res = srv.poll(t, timeout_ms=60_000)
                assert res.status == 0 and (res.narg, res.hints) == expected[i], f"served request {i}"
        finally:
            srv.close()
    finally:
        ctx.close()


def test_multi_vector_limits(gpu_ctx):
    n = 8
    coeffs = sample_goldilocks(6180, 65 << n).reshape(65, 1 << n)
    points = sample_goldilocks(6181, n * 3).reshape(1, n, 3)
    evals = np.zeros((65, 3), dtype=np.uint64)
    with pytest.raises(WhirGpuError):  # more than 64 vectors
        prove_once(n, params(batch=65), coeffs, points, evals, ctx=gpu_ctx)
    with pytest.raises(WhirGpuError):  # more than 8 witnesses
        prove_once(n, params(batch=1), coeffs[:9], points, evals[:9], ctx=gpu_ctx, num_witnesses=9)
    # the context stays usable
    ev = mle_evals(gpu_ctx, coeffs[:2], points)
    narg, _, _ = prove_once(n, params(batch=2), coeffs[:2], points, ev, ctx=gpu_ctx)
    assert len(narg) > 0
