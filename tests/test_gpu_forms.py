"""Statements of dense Covector and MultilinearExtension linear forms
(linear_form.hpp:54-138, the two kinds the reference's callers construct):
whirgpu_prove_forms combines them in the given order; a covector adds
crlc_f * vector to the covector the sumcheck runs against (crlc_0 = 1,
whir_prover.hpp:157-163).  GPU proofs must equal the reference prover's
fixtures, the oracle and a live reference run."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle.refio import ref_available, run_reference
from tests.golden.forms import form_inputs
from whirplonk_b200 import Covector, MultilinearExtension, ProtocolParameters, prove_once
from whirplonk_b200._lib import WhirGpuError
from whirplonk_b200.whir import ENGINE_ID_BLAKE3, ENGINE_ID_SHA2

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
FORMS = json.load(open(os.path.join(HERE, "golden", "reference_proofs.json")))["forms"]


def params(k=4, rho=1, batch=1, sha2=False):
    return ProtocolParameters(False, rho, k, k, 100, 20, batch, ENGINE_ID_SHA2 if sha2 else ENGINE_ID_BLAKE3)


def to_forms(forms, device=None):
    out = []
    for kind, data in forms:
        if kind == "mle":
            out.append(MultilinearExtension(data))
        elif device is not None:
            out.append(Covector(device(data), on_device=True))
        else:
            out.append(Covector(data))
    return out


@pytest.mark.parametrize("case", FORMS, ids=lambda c: f"n{c['n']}-{'-'.join(c['kinds'])}"
                                                      f"-b{c['batch_size']}w{c['num_witnesses']}{c['hash']}")
def test_covector_statements_match_reference_fixtures(gpu_ctx, case):
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
    assert len(claim.rlc_coefficients) == len(forms)


@pytest.mark.parametrize("n,kinds,batch,device", [
    (13, ("covector",), 1, False), (13, ("covector",), 1, True),
    (15, ("mle", "covector", "covector", "mle"), 2, True),
    (16, ("covector", "mle"), 1, False),
])
def test_covector_statements_match_oracle(gpu_ctx, oracle, n, kinds, batch, device):
    import torch

    coeffs, forms = form_inputs(n, 7000 + n, kinds, batch)
    # claimed values: <covector, lift(v)> and MLE values, from the oracle's own evaluations
    evals = []
    for kind, data in forms:
        for v in range(batch):
            if kind == "mle":
                evals.append(list(gpu_ctx.mle_evaluate(coeffs[v], data)))
            else:
                P = (1 << 64) - (1 << 32) + 1
                c = data.astype(object)
                x = coeffs[v].astype(object)
                evals.append([int(sum(c[:, j] * x) % P) for j in range(3)])
    evals = np.array(evals, dtype=np.uint64)
    keep = []

    def dev(a):
        t = torch.from_numpy(np.ascontiguousarray(a).view(np.int64).copy()).cuda()
        keep.append(t)
        return t.data_ptr()

    torch.cuda.synchronize()
    narg, hints, _ = prove_once(n, params(batch=batch), coeffs, None, evals, ctx=gpu_ctx,
                                forms=to_forms(forms, dev if device else None))
    onarg, ohints = oracle.prove_forms(n, 4, 1, 100, 20, forms, coeffs, evals, batch, 1)
    assert narg == onarg and hints == ohints


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_covector_statement_matches_live_reference(gpu_ctx):
    n, kinds = 18, ("covector", "mle")
    coeffs, forms = form_inputs(n, 7100, kinds, 2)
    ref = run_reference(n, 4, 2, 100, 20, None, coeffs, verify=True, batch_size=2, forms=forms)
    assert ref.verify_ok == 1.0
    narg, hints, _ = prove_once(n, params(rho=2, batch=2), coeffs, None, ref.evaluations, ctx=gpu_ctx,
                                forms=to_forms(forms))
    assert narg == ref.narg and hints == ref.hints


def test_bad_form_kind_is_rejected(gpu_ctx):
    from whirplonk_b200 import Config, ProverState, cli_domain_separator
    from whirplonk_b200 import _lib

    n = 8
    coeffs, forms = form_inputs(n, 7200, ("mle",), 1)
    p = params()
    cfg = Config.from_params(1 << n, p)
    ps = ProverState.from_ds(cli_domain_separator(p), b"", gpu_ctx)
    w = cfg.commit(ps, coeffs[0])
    bad = (_lib.LinearForm * 1)(_lib.LinearForm(7, 0, forms[0][1].ctypes.data))
    ev = np.zeros((1, 3), dtype=np.uint64)
    st = gpu_ctx._L.whirgpu_prove_forms(gpu_ctx.handle, w.handle, bad, 1, ev.ctypes.data, ps.handle, None, None)
    assert st == _lib.E_INVALID
    with pytest.raises(ValueError):  # a covector must have 2^n entries
        cfg.prove(ps, coeffs[0], [w], [Covector(np.zeros((5, 3), dtype=np.uint64))], [(0, 0, 0)])
    ev1 = np.array([gpu_ctx.mle_evaluate(coeffs[0], forms[0][1])], dtype=np.uint64)
    with pytest.raises(WhirGpuError):  # nine forms: above the eight this path holds
        cfg.prove(ps, coeffs[0], [w], [MultilinearExtension(forms[0][1])] * 9, [tuple(ev1[0])] * 9)
