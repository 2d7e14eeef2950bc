"""Shared setup of the zero-knowledge fixtures ("zk" in reference_proofs.json,
made by oracle/_ref/ref_zk_driver): parameters, policy and the base-field
statement of each case, as tests/golden/make_fixtures.py built them."""
from tests.golden.forms import form_inputs
from whirplonk_b200 import Covector, MultilinearExtension, ProtocolParameters
from whirplonk_b200.whir import ENGINE_ID_BLAKE3, ENGINE_ID_SHA2
from whirplonk_b200.zk import BlindingSizePolicy, ZkConfig


def case_params(case):
    """The driver's ProtocolParameters: pow_bits 0, batch 1, list decoding."""
    eng = ENGINE_ID_SHA2 if case["hash"] == "sha2" else ENGINE_ID_BLAKE3
    return ProtocolParameters(False, case["rho"], case["k"], case["k"], case["security"], 0, 1, eng)


def case_policy(case):
    return BlindingSizePolicy(*case["policy"], 3) if case["policy"] else None


def case_config(case):
    return ZkConfig.from_params(1 << case["n"], case_params(case), case["num_polynomials"],
                                case_policy(case)).disable_pow()


def case_statement(case):
    """(polynomials, forms, evaluations as Ext3 triples)."""
    n = case["n"]
    polys, forms = form_inputs(n, case["seed"], case["kinds"], case["num_polynomials"], base_field=True)
    objs = [MultilinearExtension(d) if kind == "mle" else Covector(d) for kind, d in forms]
    evals = [(int(x), 0, 0) for x in case["evaluations"]]
    return polys, objs, evals


def case_seed(case):
    return int(case["seed"]).to_bytes(8, "little") + bytes(24)
