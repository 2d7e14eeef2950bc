"""Kernel-level RS encoding + matrix commitment (config 2 shapes) and the NTT
pass-plan autotuner: roots and codewords against the oracle, every plan gives
the same codeword, proofs are independent of the installed plans."""
import ctypes

import numpy as np
import pytest

from whirplonk_b200 import Context, ProtocolParameters, _lib, prove_once, sample_goldilocks
from whirplonk_b200.autotune import current_plan, tune
from whirplonk_b200.autotune import load as load_plans
from whirplonk_b200.rs import rs_commit_batch, rs_encode

pytestmark = pytest.mark.gpu
P = 0xFFFFFFFF00000001


def oracle_root(oracle, v, log_exp, depth=16):
    m = v.size // depth
    N = m << log_exp
    rows = oracle.rs_encode_base(v, N, depth)  # N x depth
    leaves = b"".join(oracle.blake3(rows[i].tobytes()) for i in range(N))
    return oracle.merkle_root(leaves)


@pytest.mark.parametrize("log_len,log_exp,count", [(8, 1, 1), (10, 2, 3), (12, 3, 2), (12, 4, 1), (14, 2, 1),
                                                   (6, 4, 2), (4, 1, 1)])
def test_rs_commit_roots_match_oracle(gpu_ctx, oracle, log_len, log_exp, count):
    v = sample_goldilocks(900 + log_len * 7 + log_exp, count << log_len).reshape(count, -1)
    roots = rs_commit_batch(gpu_ctx, v, log_exp)
    for k in range(count):
        assert roots[k] == oracle_root(oracle, v[k], log_exp), f"vector {k}"


@pytest.mark.parametrize("log_len,count", [(16, 64), (20, 4), (24, 1)])
@pytest.mark.parametrize("log_exp", [1, 2, 3, 4])
def test_rs_commit_roots_at_kernel_level_sizes(gpu_ctx, oracle, log_len, log_exp, count):
    """The kernel-level workload's sizes: 2^16 words x 64 vectors, 2^20 x 4 and
    2^24 x 1, expansions 2, 4, 8 and 16, rows of 16 elements; every root equals
    the oracle's matrix commitment of the same vector."""
    v = sample_goldilocks(7000 + 17 * log_len + log_exp, count << log_len).reshape(count, -1)
    roots = rs_commit_batch(gpu_ctx, v, log_exp)
    N = ((1 << log_len) // 16) << log_exp
    for k in range(count):
        assert roots[k] == oracle.rs_commit_root(v[k], N, 16), f"vector {k}"


@pytest.mark.parametrize("log_len,log_exp,count", [(8, 12, 2), (10, 14, 1), (12, 8, 3), (9, 10, 2), (6, 16, 1)])
def test_rs_commit_roots_high_expansion(gpu_ctx, oracle, log_len, log_exp, count):
    """Expansions 2^8 .. 2^16: the message fits one row of the second pass, so
    the first pass is skipped and the last one applies the inter-pass factors
    to the message itself; roots equal the oracle's."""
    v = sample_goldilocks(7700 + 31 * log_len + log_exp, count << log_len).reshape(count, -1)
    roots = rs_commit_batch(gpu_ctx, v, log_exp)
    N = ((1 << log_len) // 16) << log_exp
    for k in range(count):
        assert roots[k] == oracle.rs_commit_root(v[k], N, 16), f"vector {k}"


def test_rs_encode_planes_match_oracle(gpu_ctx, oracle):
    import torch

    log_len, log_exp, count = 13, 3, 2
    v = sample_goldilocks(77, count << log_len)
    m = (1 << log_len) // 16
    N = m << log_exp
    dv = torch.from_numpy(v.view(np.int64)).cuda()
    tmp = torch.empty(count * 16 * N, dtype=torch.int64, device="cuda")
    out = torch.empty_like(tmp)
    rs_encode(gpu_ctx, dv.data_ptr(), count, log_len, log_exp, 4, tmp.data_ptr(), out.data_ptr())
    torch.cuda.synchronize()
    got = out.cpu().numpy().view(np.uint64).reshape(count, 16, N)
    for k in range(count):
        rows = oracle.rs_encode_base(v[k << log_len:(k + 1) << log_len], N, 16)
        assert np.array_equal(got[k], rows.T)


def test_rs_encode_full_size_spot_values(gpu_ctx):
    """2^22 words, expansion 4: codeword entries at random positions equal the
    direct evaluation sum_j x_j w_N^(i j) (Horner on the host)."""
    import torch

    log_len, log_exp = 22, 2
    v = sample_goldilocks(31337, 1 << log_len)
    m = (1 << log_len) // 16
    N = m << log_exp
    dv = torch.from_numpy(v.view(np.int64)).cuda()
    tmp = torch.empty(16 * N, dtype=torch.int64, device="cuda")
    out = torch.empty_like(tmp)
    rs_encode(gpu_ctx, dv.data_ptr(), 1, log_len, log_exp, 4, tmp.data_ptr(), out.data_ptr())
    torch.cuda.synchronize()
    planes = out.cpu().numpy().view(np.uint64).reshape(16, N)
    w = pow(7, (P - 1) // N, P)
    rng = np.random.default_rng(5)
    for b, i in [(0, 0), (15, N - 1)] + [(int(rng.integers(16)), int(rng.integers(N))) for _ in range(3)]:
        x = pow(w, i, P)
        acc = 0
        for c in reversed(v[b * m:(b + 1) * m].tolist()):
            acc = (acc * x + c) % P
        assert int(planes[b, i]) == acc, (b, i)


def test_rs_commit_device_input_and_batch_consistency(gpu_ctx):
    import torch

    v = sample_goldilocks(4242, 6 << 16).reshape(6, -1)
    host_roots = rs_commit_batch(gpu_ctx, v, 2)
    dv = torch.from_numpy(v.reshape(-1).view(np.int64)).cuda()
    dev_roots = rs_commit_batch(gpu_ctx, None, 2, on_device_ptr=dv.data_ptr(), count=6, log_len=16)
    assert host_roots == dev_roots
    singles = [rs_commit_batch(gpu_ctx, v[k], 2)[0] for k in range(6)]
    assert singles == host_roots


def test_autotune_plans_agree_and_proofs_unchanged(gpu_ctx, oracle):
    L = _lib.load()
    n, rho = 14, 2
    params = ProtocolParameters.cli(log_inv_rate=rho)
    coeffs = sample_goldilocks(88, 1 << n)
    pts = sample_goldilocks(89, 3 * n).reshape(1, n, 3)
    ev = np.array(gpu_ctx.mle_evaluate(coeffs, pts), dtype=np.uint64).reshape(1, 3)
    L.whirgpu_ntt_clear_plans()
    before = prove_once(n, params, coeffs, pts, ev, ctx=gpu_ctx)[:2]
    from whirplonk_b200.autotune import lde_shapes

    res = tune(gpu_ctx, lde_shapes(n, params), reps=2, log=lambda *_: None)
    assert res and all("rejected" not in r for r in res)
    for r in res:
        assert current_plan(r["log_n"], r["log_expansion"])["log_radix"] == r["log_radix"]
    # force a deliberately different valid plan on the initial shape, too
    ln, lx, _ = lde_shapes(n, params)[0]
    forced = _lib.NttPlan(ln, lx, 3, (1, ln - 2, 1), (255, 255, 255))
    assert L.whirgpu_ntt_set_plan(ctypes.byref(forced)) == _lib.OK
    after = prove_once(n, params, coeffs, pts, ev, ctx=gpu_ctx)[:2]
    L.whirgpu_ntt_clear_plans()
    L.whirgpu_ntt_load_default_plans()
    assert before == after
    onarg, ohints = oracle.prove(n, 4, rho, 100, 20, pts, coeffs, ev)
    assert before == (onarg, ohints)


def _pipelined(ln, lx, minb):
    """The shape's current plan with persistent pipelined passes."""
    plan = _lib.NttPlan()
    _lib.check(_lib.load().whirgpu_ntt_get_plan(ln, lx, ctypes.byref(plan)))
    plan.min_blocks = minb
    plan.pipelined = 1
    return plan


@pytest.mark.parametrize("log_len,log_exp,minb", [(20, 2, 3), (18, 3, 4), (16, 5, 2), (24, 1, 3), (12, 4, 4)])
def test_pipelined_passes_match_oracle(gpu_ctx, oracle, log_len, log_exp, minb):
    """Persistent pipelined passes (the next tile's copies in flight while the
    current one is transformed) give the oracle's roots."""
    L = _lib.load()
    ln = log_len - 4 + log_exp
    plan = _pipelined(ln, log_exp, minb)
    assert L.whirgpu_ntt_set_plan(ctypes.byref(plan)) == _lib.OK
    try:
        count = 2 if log_len <= 20 else 1
        v = sample_goldilocks(9100 + log_len + log_exp, count << log_len).reshape(count, -1)
        roots = rs_commit_batch(gpu_ctx, v, log_exp)
        N = ((1 << log_len) // 16) << log_exp
        for k in range(count):
            assert roots[k] == oracle.rs_commit_root(v[k], N, 16), f"vector {k}"
    finally:
        L.whirgpu_ntt_clear_plans()
        load_plans()


def test_pipelined_plans_proof_matches_oracle(gpu_ctx, oracle):
    """A whole proof with every LDE of its schedule on pipelined passes."""
    from whirplonk_b200.autotune import lde_shapes

    L = _lib.load()
    n, rho = 18, 2
    params = ProtocolParameters.cli(log_inv_rate=rho)
    try:
        for ln, lx, _ in lde_shapes(n, params):
            plan = _pipelined(ln, lx, 3)
            assert L.whirgpu_ntt_set_plan(ctypes.byref(plan)) == _lib.OK
        coeffs = sample_goldilocks(91, 1 << n)
        pts = sample_goldilocks(92, 3 * n).reshape(1, n, 3)
        ev = np.array(gpu_ctx.mle_evaluate(coeffs, pts), dtype=np.uint64).reshape(1, 3)
        got = prove_once(n, params, coeffs, pts, ev, ctx=gpu_ctx)[:2]
        assert got == oracle.prove(n, 4, rho, 100, 20, pts, coeffs, ev)
    finally:
        L.whirgpu_ntt_clear_plans()
        load_plans()
