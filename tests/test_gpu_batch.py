"""Batches and the serving loop: every proof made in a mix is byte-identical to
the same proof made alone (and to the oracle), whatever the mode, the
interleaving and the admission order; HBM-budget admission holds."""
import threading
import time

import numpy as np
import pytest

from whirplonk_b200 import Context, ProtocolParameters, prove_once, sample_goldilocks
from whirplonk_b200.batch import Batch, ProofRequest, Server

pytestmark = pytest.mark.gpu


def make_requests(ctx, specs, seed0=3000):
    reqs = []
    for i, (n, rho) in enumerate(specs):
        params = ProtocolParameters.cli(log_inv_rate=rho)
        coeffs = sample_goldilocks(seed0 + i, 1 << n)
        pts = sample_goldilocks(seed0 + 500 + i, n * 3).reshape(1, n, 3)
        ev = np.array(ctx.mle_evaluate(coeffs, pts), dtype=np.uint64).reshape(1, 3)
        reqs.append(ProofRequest(n, params, coeffs, pts, ev))
    return reqs


def alone(ctx, r):
    narg, hints, _ = prove_once(r.num_variables, r.params, r.coeffs, r.points, r.evaluations, ctx=ctx)
    return narg, hints


SPECS = [(12, 1), (8, 3), (14, 2), (10, 1), (12, 3), (9, 2), (13, 1), (12, 1), (11, 2), (15, 3)]


@pytest.mark.parametrize("mode", [Batch.GRAPH, Batch.STREAMS, Batch.PLAIN])
def test_batch_matches_alone(gpu_ctx, mode):
    reqs = make_requests(gpu_ctx, SPECS)
    expected = [alone(gpu_ctx, r) for r in reqs]
    with Batch(gpu_ctx, reqs, mode) as b:
        for _ in range(2):  # the same batch program runs again on fresh copies of the inputs
            b.run()
            for i, e in enumerate(expected):
                assert b.proof(i) == e, f"request {i} {SPECS[i]} differs in mode {mode}"


def test_batch_matches_oracle(gpu_ctx, oracle):
    reqs = make_requests(gpu_ctx, [(10, 2), (11, 1)], seed0=4000)
    with Batch(gpu_ctx, reqs, Batch.GRAPH) as b:
        b.run()
        for i, r in enumerate(reqs):
            rho = r.params.starting_log_inv_rate
            onarg, ohints = oracle.prove(r.num_variables, 4, rho, 100, 20, r.points, r.coeffs, r.evaluations)
            assert b.proof(i) == (onarg, ohints)


MANY = [(8 + (i * 7) % 8, 1 + i % 3) for i in range(48)]


def test_server_mix_matches_alone():
    """Heavy overlap (16 proofs in flight, CTAs of concurrent kernels starting
    late) must not change a byte: PoW minimum nonces, openings, all of it."""
    ctx = Context(0)
    try:
        reqs = make_requests(ctx, SPECS * 2 + MANY, seed0=5000)
        expected = [alone(ctx, r) for r in reqs]
        srv = Server(ctx, hbm_budget=0, max_inflight=16)
        tickets = []
        for r in reqs:  # requests keep arriving while earlier ones run
            tickets.append(srv.submit(r))
            time.sleep(0.0005)
        for i, t in enumerate(tickets):
            res = srv.poll(t, timeout_ms=60_000)
            assert res is not None and res.status == 0
            assert (res.narg, res.hints) == expected[i], f"served request {i} differs"
            assert res.total_ms >= res.queue_ms >= 0
        st = srv.stats()
        assert st["admitted"] == len(reqs) and st["peak_inflight"] > 1
        srv.close()
    finally:
        ctx.close()


def test_server_hbm_budget_admission():
    from whirplonk_b200 import _lib
    from whirplonk_b200.whir import Config

    ctx = Context(0)
    try:
        reqs = make_requests(ctx, [(14, 2)] * 4 + [(10, 1)] * 4, seed0=6000)
        expected = [alone(ctx, r) for r in reqs]
        big = Config.from_params(1 << 14, reqs[0].params).workspace_bytes()
        small = Config.from_params(1 << 10, reqs[-1].params).workspace_bytes()
        assert big > small > 0
        srv = Server(ctx, hbm_budget=big - 1, max_inflight=8)
        with pytest.raises(_lib.WhirGpuError):
            srv.submit(reqs[0])  # a request that can never fit is refused at submit
        srv.close()
        budget = big + 2 * small  # one large proof and two small ones at a time
        srv = Server(ctx, hbm_budget=budget, max_inflight=8)
        tickets = [srv.submit(r) for r in reqs]
        for i, t in enumerate(tickets):
            res = srv.poll(t, timeout_ms=60_000)
            assert res.status == 0 and (res.narg, res.hints) == expected[i]
        st = srv.stats()
        assert st["admitted"] == len(reqs)
        assert 0 < st["peak_bytes"] <= budget
        srv.close()
    finally:
        ctx.close()


def test_server_device_inputs_and_eviction():
    """Device-resident coefficients are served like host ones, and a budget
    too small to cache every shape's workspace evicts idle ones (and their
    captured programs) without changing any proof."""
    import torch

    ctx = Context(0)
    try:
        specs = [(13, 1), (11, 2), (12, 3), (10, 1), (13, 1), (11, 2), (12, 3), (10, 1)]
        reqs = make_requests(ctx, specs, seed0=7000)
        expected = [alone(ctx, r) for r in reqs]
        dev = [torch.from_numpy(np.asarray(r.coeffs).view(np.int64)).cuda() for r in reqs]
        torch.cuda.synchronize()
        dreqs = [ProofRequest(r.num_variables, r.params, d.data_ptr(), r.points, r.evaluations, on_device=True)
                 for r, d in zip(reqs, dev)]
        from whirplonk_b200.whir import Config

        sizes = [Config.from_params(1 << n, reqs[i].params).workspace_bytes() for i, (n, _) in enumerate(specs)]
        budget = max(sizes) + min(sizes)  # at most two shapes resident at once
        ctx2 = Context(0)  # empty workspace cache: every shape change must evict
        srv = Server(ctx2, hbm_budget=budget, max_inflight=4)
        for rounds in range(2):
            tickets = [srv.submit(r) for r in (dreqs if rounds == 0 else reqs)]
            for i, t in enumerate(tickets):
                res = srv.poll(t, timeout_ms=60_000)
                assert res.status == 0 and (res.narg, res.hints) == expected[i], f"request {i} round {rounds}"
        st = srv.stats()
        assert st["peak_bytes"] <= budget
        # four shapes through a cache that holds two: workspaces were allocated
        # for each and idle ones evicted; what stays cached fits the budget
        ws = ctx2.workspace_stats()
        assert ws["allocations"] >= 4 and ws["evictions"] >= 1, ws
        assert 0 < ws["cached_bytes"] <= budget, ws
        srv.close()
        ctx2.close()
    finally:
        ctx.close()
