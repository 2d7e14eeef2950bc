"""Basefield<GoldilocksExt2> as the target field (the CLI's --field Goldilocks2,
Fp[X]/(X^2 - 7)): GPU proofs must equal the reference prover's
(oracle/_ref/ref_driver --field2) fixtures and a live reference run byte for
byte."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle.refio import ref_available, run_reference
from tests.golden.forms import form_inputs
from whirplonk_b200 import FIELD_GOLDILOCKS2, Covector, MultilinearExtension, ProtocolParameters, prove_once
from whirplonk_b200._lib import WhirGpuError
from whirplonk_b200.whir import ENGINE_ID_BLAKE3, ENGINE_ID_SHA2

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
FIELD2 = json.load(open(os.path.join(HERE, "golden", "reference_proofs.json")))["field2"]


def params(k=4, rho=1, sec=40, pb=10, batch=1, sha2=False, unique=False):
    return ProtocolParameters(unique, rho, k, k, sec, pb, batch, ENGINE_ID_SHA2 if sha2 else ENGINE_ID_BLAKE3)


@pytest.mark.parametrize("case", FIELD2, ids=lambda c: f"n{c['n']}-{'-'.join(c['kinds']) or 'none'}"
                                                       f"-b{c['batch_size']}w{c['num_witnesses']}{c['hash']}")
def test_goldilocks2_matches_reference_fixtures(gpu_ctx, case):
    n, batch, nwit = case["n"], case["batch_size"], case["num_witnesses"]
    coeffs, forms = form_inputs(n, case["seed"], case["kinds"], batch * nwit, ext2=True)
    evals = np.array(case["evaluations"], dtype=np.uint64).reshape(-1, 3)
    assert not evals[:, 2].any()
    p = params(case["k"], case["rho"], case["security"], case["pow_bits"], batch, case["hash"] == "sha2",
               case["unique_decoding"])
    fs = [MultilinearExtension(d) if kind == "mle" else Covector(d) for kind, d in forms]
    narg, hints, _ = prove_once(n, p, coeffs, None, evals, ctx=gpu_ctx, num_witnesses=nwit, forms=fs,
                                target_field=FIELD_GOLDILOCKS2)
    assert (len(narg), len(hints)) == (case["narg_len"], case["hints_len"])
    assert hashlib.sha256(narg).hexdigest() == case["narg_sha256"]
    assert hashlib.sha256(hints).hexdigest() == case["hints_sha256"]
    if "narg" in case:
        assert narg.hex() == case["narg"] and hints.hex() == case["hints"]


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_goldilocks2_matches_live_reference(gpu_ctx):
    n = 16
    coeffs, forms = form_inputs(n, 7900, ("mle", "covector"), 2, ext2=True)
    ref = run_reference(n, 4, 2, 48, 12, None, coeffs, verify=True, forms=forms, batch_size=2, field2=True)
    assert ref.verify_ok == 1.0
    fs = [MultilinearExtension(forms[0][1]), Covector(forms[1][1])]
    narg, hints, _ = prove_once(n, params(4, 2, 48, 12, 2), coeffs, None, ref.evaluations, ctx=gpu_ctx, forms=fs,
                                target_field=FIELD_GOLDILOCKS2)
    assert narg == ref.narg and hints == ref.hints


def test_goldilocks2_rejects_cubic_inputs(gpu_ctx):
    """A form with a nonzero X^2 coefficient is not a GoldilocksExt2 element:
    the first message outside (c0, c1) sets the device error word."""
    n = 10
    coeffs, forms = form_inputs(n, 7901, ("covector",), 1)  # full Ext3 values
    evals = np.zeros((1, 3), dtype=np.uint64)
    with pytest.raises(WhirGpuError):
        prove_once(n, params(), coeffs, None, evals, ctx=gpu_ctx, forms=[Covector(forms[0][1])],
                   target_field=FIELD_GOLDILOCKS2)
    # the context stays usable
    coeffs, forms = form_inputs(n, 7902, ("mle",), 1, ext2=True)
    case = FIELD2[1]
    coeffs, forms = form_inputs(case["n"], case["seed"], case["kinds"], 1, ext2=True)
    evals = np.array(case["evaluations"], dtype=np.uint64).reshape(-1, 3)
    narg, _, _ = prove_once(case["n"], params(case["k"], case["rho"], case["security"], case["pow_bits"]), coeffs,
                            None, evals, ctx=gpu_ctx, forms=[MultilinearExtension(forms[0][1])],
                            target_field=FIELD_GOLDILOCKS2)
    assert hashlib.sha256(narg).hexdigest() == case["narg_sha256"]
