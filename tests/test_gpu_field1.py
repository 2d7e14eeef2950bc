"""The base field as the target field (Identity<Goldilocks>, the CLI's
--field Goldilocks1) and Configs built field by field: GPU proofs must equal
the reference's committed whole-proof golden dump (cpp/dump_output/whir_output,
byte-identical in the Rust and C++ versions), the reference prover's
Goldilocks1 fixtures, the oracle and a live reference run."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle.refio import ref_available, run_reference
from tests.golden.forms import form_inputs
from whirplonk_b200 import (FIELD_GOLDILOCKS1, Config, Covector, DomainSeparator, MultilinearExtension,
                            ProtocolParameters, ProverState, prove_once)
from whirplonk_b200 import _lib
from whirplonk_b200._lib import WhirGpuError
from whirplonk_b200.whir import ENGINE_ID_BLAKE3, ENGINE_ID_SHA2

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_goldens.json")))
FIELD1 = json.load(open(os.path.join(HERE, "golden", "reference_proofs.json")))["field1"]
P = 0xFFFFFFFF00000001


def params(k=4, rho=1, sec=40, pb=10, batch=1, sha2=False, unique=False):
    return ProtocolParameters(unique, rho, k, k, sec, pb, batch, ENGINE_ID_SHA2 if sha2 else ENGINE_ID_BLAKE3)


def golden_config(case):
    """cpp/tests/dump_whir.cpp:run_case's Config, field by field."""
    size = case["vector_size"]
    c = _lib.WhirConfig()
    c.field = FIELD_GOLDILOCKS1
    c.batch_size = case["num_vectors"]
    for i, b in enumerate(ENGINE_ID_SHA2):
        c.hash_id[i] = b
    c.initial_committer = _lib.IrsConfig(size, 2 * size, 1, min(size, 3), 1)
    c.initial_sumcheck = _lib.SumcheckConfig(0, _lib.NO_POW)
    c.initial_skip_pow = _lib.NO_POW
    c.num_rounds = 0
    c.final_sumcheck = _lib.SumcheckConfig(size.bit_length() - 1, _lib.NO_POW)
    c.final_pow = _lib.NO_POW
    return c


def golden_ds(case):
    proto = hashlib.sha3_512(bytes([0x19, 0xBE, 0xEF])).digest()
    label = f"whir_{case['case']}".encode()
    return DomainSeparator(proto, hashlib.sha3_256(bytes([0x60 + len(label)]) + label).digest())


@pytest.mark.parametrize("case", GOLD["whir"], ids=lambda c: f"case{c['case']}")
def test_reference_whir_golden(gpu_ctx, case):
    size, nvec = case["vector_size"], case["num_vectors"]
    coeffs = np.array(case["inputs"], dtype=np.uint64)
    ones = np.zeros((size, 3), dtype=np.uint64)
    ones[:, 0] = 1
    evals = [(sum(v) % P, 0, 0) for v in case["inputs"]]
    config = Config.custom(golden_config(case))
    ps = ProverState.from_ds(golden_ds(case), b"", gpu_ctx)
    w = config.commit(ps, coeffs)
    claim = config.prove(ps, coeffs, [w], [Covector(ones)], evals)
    narg, hints = ps.proof()
    assert narg.hex() == case["narg"]
    assert hints.hex() == case["hints"]
    assert [e[0] for e in claim.evaluation_point] == case["eval_point"]
    assert all(e[1] == 0 and e[2] == 0 for e in claim.evaluation_point)
    assert [r[0] for r in claim.rlc_coefficients] == case["rlc_coeffs"]
    del nvec


@pytest.mark.parametrize("case", FIELD1, ids=lambda c: f"n{c['n']}-{'-'.join(c['kinds']) or 'none'}"
                                                       f"-b{c['batch_size']}w{c['num_witnesses']}{c['hash']}")
def test_goldilocks1_matches_reference_fixtures(gpu_ctx, case):
    n, batch, nwit = case["n"], case["batch_size"], case["num_witnesses"]
    coeffs, forms = form_inputs(n, case["seed"], case["kinds"], batch * nwit, base_field=True)
    evals = np.array(case["evaluations"], dtype=np.uint64).reshape(-1, 3)
    p = params(case["k"], case["rho"], case["security"], case["pow_bits"], batch, case["hash"] == "sha2",
               case["unique_decoding"])
    fs = [MultilinearExtension(d) if kind == "mle" else Covector(d) for kind, d in forms]
    narg, hints, _ = prove_once(n, p, coeffs, None, evals, ctx=gpu_ctx, num_witnesses=nwit, forms=fs,
                                target_field=FIELD_GOLDILOCKS1)
    assert (len(narg), len(hints)) == (case["narg_len"], case["hints_len"])
    assert hashlib.sha256(narg).hexdigest() == case["narg_sha256"]
    assert hashlib.sha256(hints).hexdigest() == case["hints_sha256"]
    if "narg" in case:
        assert narg.hex() == case["narg"] and hints.hex() == case["hints"]


@pytest.mark.parametrize("n,k,rho,sec,pb,batch", [(9, 3, 1, 40, 10, 1), (13, 4, 1, 36, 12, 2), (16, 4, 2, 32, 10, 1)])
def test_goldilocks1_matches_oracle(gpu_ctx, oracle, n, k, rho, sec, pb, batch):
    coeffs, forms = form_inputs(n, 7700 + n, ("mle",), batch, base_field=True)
    evals = np.array([gpu_ctx.mle_evaluate(coeffs[v], forms[0][1]) for v in range(batch)], dtype=np.uint64)
    assert not evals[:, 1:].any()
    narg, hints, _ = prove_once(n, params(k, rho, sec, pb, batch), coeffs, None, evals, ctx=gpu_ctx,
                                forms=[MultilinearExtension(forms[0][1])], target_field=FIELD_GOLDILOCKS1)
    onarg, ohints = oracle.prove_forms(n, k, rho, sec, pb, forms, coeffs, evals, batch, 1, field1=True)
    assert narg == onarg and hints == ohints


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_goldilocks1_matches_live_reference(gpu_ctx):
    n = 16
    coeffs, forms = form_inputs(n, 7800, ("mle", "covector"), 1, base_field=True)
    ref = run_reference(n, 4, 1, 36, 12, None, coeffs, verify=True, forms=forms, field1=True)
    assert ref.verify_ok == 1.0
    fs = [MultilinearExtension(forms[0][1]), Covector(forms[1][1])]
    narg, hints, _ = prove_once(n, params(4, 1, 36, 12), coeffs, None, ref.evaluations, ctx=gpu_ctx, forms=fs,
                                target_field=FIELD_GOLDILOCKS1)
    assert narg == ref.narg and hints == ref.hints


def test_goldilocks1_rejects_extension_inputs(gpu_ctx):
    n = 8
    coeffs, forms = form_inputs(n, 7900, ("mle",), 1)  # Ext3 point: not a base-field statement
    evals = np.zeros((1, 3), dtype=np.uint64)
    with pytest.raises(WhirGpuError):
        prove_once(n, params(), coeffs, None, evals, ctx=gpu_ctx, forms=[MultilinearExtension(forms[0][1])],
                   target_field=FIELD_GOLDILOCKS1)
    bad = golden_config({"vector_size": 8, "num_vectors": 1})
    bad.initial_committer.interleaving_depth = 2  # depth must be 2^(initial sumcheck rounds) = 1
    ps = ProverState.from_ds(DomainSeparator(b"\0" * 64, b"\0" * 32), b"", gpu_ctx)
    with pytest.raises(WhirGpuError):
        Config.custom(bad).commit(ps, coeffs[0][:8])
