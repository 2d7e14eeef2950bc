"""Zero-knowledge configuration (ZkConfig::from_params[_with_policy],
whir_zk.hpp:95-105, 270-289) against the reference's own derivation recorded in
the "zk" fixtures; host-only calls of the C ABI (no GPU)."""
import json
import os

import pytest

from tests.zk_cases import case_config, case_params
from whirplonk_b200._lib import WhirGpuError
from whirplonk_b200.whir import ProtocolParameters
from whirplonk_b200.zk import BlindingSizePolicy, ZkConfig

HERE = os.path.dirname(os.path.abspath(__file__))
ZK = json.load(open(os.path.join(HERE, "golden", "reference_proofs.json")))["zk"]


@pytest.mark.parametrize("case", ZK, ids=lambda c: f"n{c['n']}_s{c['seed']}")
def test_zk_config_matches_reference(case):
    cfg = case_config(case)
    assert cfg.num_witness_variables == case["n"]
    assert cfg.num_blinding_variables == case["num_blinding_variables"]
    assert cfg.blinded_in_domain_samples == case["blinded_queries"]
    assert cfg.blinding_batch_size == case["blinding_batch"]
    assert cfg.blinding_batch_size == case["num_polynomials"] * (case["n"] + 1)
    assert cfg.raw.blinding.initial_committer.vector_size == 2 << cfg.num_blinding_variables
    assert cfg.raw.blinded.field == 1 and cfg.raw.blinding.field == 1


def test_zk_config_rejects_what_the_reference_asserts():
    p = ProtocolParameters(False, 1, 4, 4, 80, 0, 1)
    with pytest.raises(WhirGpuError):  # num_blinding_variables would not be below num_witness_variables
        ZkConfig.from_params(1 << 10, p, 1)
    with pytest.raises(WhirGpuError):
        ZkConfig.from_params(1 << 12, ProtocolParameters(False, 1, 2, 2, 16, 0, 2), 1, BlindingSizePolicy(4, 4, 4, 4))
    small = ZkConfig.from_params(1 << 10, ProtocolParameters(False, 1, 2, 2, 16, 0, 1), 1, BlindingSizePolicy(4, 4, 4, 4))
    assert small.num_blinding_variables < 9


GOLD_ZK = json.load(open(os.path.join(HERE, "golden", "reference_goldens.json")))["whir_zk"]


def dumper_params():
    """cpp/tests/dump_whir_zk.cpp's parameters and policy."""
    from whirplonk_b200.whir import ENGINE_ID_SHA2

    return ProtocolParameters(False, 1, 2, 2, 16, 0, 1, ENGINE_ID_SHA2), BlindingSizePolicy(4, 4, 4, 4, 3)


def test_canonical_zk_domain_separator_matches_reference_dump():
    from whirplonk_b200.zk import whir_zk_domain_separator

    p, pol = dumper_params()
    cb, ds = whir_zk_domain_separator(1 << 8, 1, p, pol, "whir_zk_0")
    assert cb.hex() == GOLD_ZK["canonical_config"]
    assert ds.protocol_id.hex() == GOLD_ZK["ds_protocol_id"]
    assert ds.session_id.hex() == GOLD_ZK["ds_session_id"]
    # without a policy the derived one (q_delta from the parameters) fills the tail
    cb2, _ = whir_zk_domain_separator(1 << 8, 1, p, None, "s")
    assert len(cb2) == len(cb) and cb2[:-40] == cb[:-40] and cb2[-40:] != cb[-40:]
