"""Zero-knowledge WHIR (ZkConfig<Goldilocks>) on the GPU: every proof must equal,
byte for byte, the reference prover's proof for the same polynomials, forms and
DeterministicRng seed (the "zk" fixtures of reference_proofs.json, made by
oracle/_ref/ref_zk_driver, which the reference's verifier accepted)."""
import hashlib
import json
import os

import numpy as np
import pytest

from tests.zk_cases import case_config, case_params, case_seed, case_statement
from whirplonk_b200 import ProverState, cli_domain_separator
from whirplonk_b200._lib import WhirGpuError
from whirplonk_b200.zk import DeterministicRng, prove_zk_once

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ZK = json.load(open(os.path.join(HERE, "golden", "reference_proofs.json")))["zk"]


def rng_words_oracle(oracle, seed, domain, first, count):
    """DeterministicRng (deterministic_rng.hpp:16-98) over the oracle's BLAKE3."""
    d = domain.encode()
    pre = b"WHIR_DETERMINISTIC_RNG_V1" + len(d).to_bytes(4, "little") + d + seed
    stream = b""
    c = first // 4
    while len(stream) < 8 * (first - 4 * (first // 4) + count):
        stream += oracle.blake3(pre + c.to_bytes(8, "little"))
        c += 1
    skip = 8 * (first % 4)
    return np.frombuffer(stream[skip:skip + 8 * count], dtype=np.uint64)


def test_deterministic_rng_matches_construction(gpu_ctx, oracle):
    seed = bytes(range(32))
    for domain, first, count in (("WHIR_ZK:mask", 0, 37), ("x" * 100, 5, 50), ("", 3, 1)):
        got = DeterministicRng(seed, domain).words(first, count, gpu_ctx)
        assert np.array_equal(got, rng_words_oracle(oracle, seed, domain, first, count))


@pytest.mark.parametrize("case", ZK, ids=lambda c: f"n{c['n']}_s{c['seed']}")
def test_zk_proof_equals_reference(gpu_ctx, case):
    cfg = case_config(case)
    polys, forms, evals = case_statement(case)
    narg, hints = prove_zk_once(case["n"], case_params(case), polys, forms, evals, case_seed(case), ctx=gpu_ctx,
                                config=cfg)
    assert (len(narg), len(hints)) == (case["narg_len"], case["hints_len"])
    assert hashlib.sha256(narg).hexdigest() == case["narg_sha256"]
    assert hashlib.sha256(hints).hexdigest() == case["hints_sha256"]


def test_zk_proof_from_device_input_and_reuse(gpu_ctx):
    """Coefficients already in HBM give the same proof; a witness proves once."""
    import torch

    case = ZK[1]
    cfg = case_config(case)
    polys, forms, evals = case_statement(case)
    dev = torch.from_numpy(polys.view(np.int64).copy()).cuda()
    torch.cuda.synchronize()
    ps = ProverState.from_ds(cli_domain_separator(case_params(case)), b"", gpu_ctx)
    rng = DeterministicRng(case_seed(case))
    w = cfg.commit(ps, None, rng, on_device_ptr=dev.data_ptr())
    claim = cfg.prove(ps, polys, w, forms, evals, rng)
    narg, _ = ps.proof()
    assert hashlib.sha256(narg).hexdigest() == case["narg_sha256"]
    # the blinded proof's FinalClaim: one base-field coordinate per variable, one
    # RLC coefficient per form, the first being 1 (geometric_challenge)
    assert len(claim.evaluation_point) == case["n"] and all(c[1] == c[2] == 0 for c in claim.evaluation_point)
    assert len(claim.rlc_coefficients) == len(forms) and claim.rlc_coefficients[0] == (1, 0, 0)
    with pytest.raises(WhirGpuError):
        cfg.prove(ps, polys, w, forms, evals, rng)


def test_zk_masks_follow_the_seed(gpu_ctx):
    """Another RNG seed gives other masks, hence other commitments and another
    proof of the same statement."""
    case = ZK[0]
    cfg = case_config(case)
    polys, forms, evals = case_statement(case)
    seed = bytearray(case_seed(case))
    seed[31] ^= 1
    narg, _ = prove_zk_once(case["n"], case_params(case), polys, forms, evals, bytes(seed), ctx=gpu_ctx, config=cfg)
    assert len(narg) == case["narg_len"]
    assert hashlib.sha256(narg).hexdigest() != case["narg_sha256"]


GOLD_ZK = json.load(open(os.path.join(HERE, "golden", "reference_goldens.json")))["whir_zk"]


def test_reference_zk_dump(gpu_ctx):
    """The reference's own ZK dumper (cpp/tests/dump_whir_zk.cpp): canonical
    domain separator, SHA-2, explicit policy, Covector of ones, seed 0..31."""
    from whirplonk_b200 import Covector, ProtocolParameters
    from whirplonk_b200.whir import ENGINE_ID_SHA2
    from whirplonk_b200.zk import BlindingSizePolicy, ZkConfig, whir_zk_domain_separator
    n = 8
    p = ProtocolParameters(False, 1, 2, 2, 16, 0, 1, ENGINE_ID_SHA2)
    pol = BlindingSizePolicy(4, 4, 4, 4, 3)
    cfg = ZkConfig.from_params(1 << n, p, 1, pol).disable_pow()
    poly = np.array(GOLD_ZK["input_vector0"], dtype=np.uint64)
    assert np.array_equal(poly, (np.arange(1 << n, dtype=np.uint64) * 17 + 3))
    ones = np.zeros((1 << n, 3), dtype=np.uint64)
    ones[:, 0] = 1
    ev = int(sum(int(x) for x in poly) % 0xFFFFFFFF00000001)
    _, ds = whir_zk_domain_separator(1 << n, 1, p, pol, "whir_zk_0")
    narg, hints = prove_zk_once(n, p, poly.reshape(1, -1), [Covector(ones)], [(ev, 0, 0)], bytes(range(32)),
                                ctx=gpu_ctx, config=cfg, ds=ds)
    assert narg.hex() == GOLD_ZK["narg"]
    assert hints.hex() == GOLD_ZK["hints"]


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(HERE), "oracle", "_ref", "ref_zk_driver")),
                    reason="oracle/_ref not built")
def test_zk_n24_matches_live_reference(gpu_ctx):
    """The largest size of the WHIR workloads (2^24 coefficients, rate 1/4,
    100-bit parameters, derived policy, PoW off): the GPU's ZK proof equals the
    reference ZK prover's."""
    from oracle.refio import run_reference_zk
    from whirplonk_b200 import MultilinearExtension, ProtocolParameters, sample_goldilocks
    from whirplonk_b200.zk import ZkConfig

    n, seed = 24, 4242
    p = ProtocolParameters(False, 2, 4, 4, 100, 20, 1)
    poly = sample_goldilocks(seed, 1 << n).reshape(1, -1)
    point = np.zeros((n, 3), dtype=np.uint64)
    point[:, 0] = sample_goldilocks(seed + 1, n)
    ref = run_reference_zk(n, 4, 2, 100, 20, [("mle", point[:, 0])], poly, seed, no_pow=True, verify=False)
    cfg = ZkConfig.from_params(1 << n, p, 1).disable_pow()
    narg, hints = prove_zk_once(n, p, poly, [MultilinearExtension(point)], [(int(ref.evaluations[0]), 0, 0)],
                                int(seed).to_bytes(8, "little") + bytes(24), ctx=gpu_ctx, config=cfg)
    assert narg == ref.narg and hints == ref.hints
