"""Pins of the CPU oracle (oracle/liboracle.so) -- no GPU needed.

The oracle is trusted as the parity checker only because it reproduces
(a) every known-answer vector of the reference's own golden dumps that lies on
    the WHIR path (tests/golden/reference_goldens.json, extracted from
    cpp/dump_output/* by tests/golden/make_fixtures.py), and
(b) whole proofs of the unmodified reference prover on seeded inputs
    (tests/golden/reference_proofs.json), and, when oracle/_ref is built,
    fresh proofs of the reference prover run live.
"""
import hashlib
import json
import os
import struct

import numpy as np
import pytest

from oracle.refio import ref_available, run_reference
from whirplonk_b200 import sample_goldilocks

P = 0xFFFFFFFF00000001
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_goldens.json")))
PROOFS = json.load(open(os.path.join(HERE, "golden", "reference_proofs.json")))["cases"]


def test_fields_base(oracle):
    L = oracle.lib
    for case in GOLD["fields"]["base"]:
        a, b = case["inputs"]
        ops = case["ops"]
        assert L.oracle_fadd(a, b) == ops["add"][0]
        assert L.oracle_fsub(a, b) == ops["sub"][0]
        assert L.oracle_fsub(0, a) == ops["neg"][0]
        assert L.oracle_fmul(a, b) == ops["mul"][0]
        assert L.oracle_fmul(a, a) == ops["sq"][0]
        assert L.oracle_fpow(a, 10) == ops["pow10"][0]
        assert L.oracle_fmul(L.oracle_fpow(a, P - 2), a) == 1
        assert L.oracle_fpow(a, P - 2) == ops["inv"][0]


def test_fields_ext3(oracle):
    for case in GOLD["fields"]["ext3"]:
        x, y = case["inputs"][:3], case["inputs"][3:]
        assert oracle.e3_mul(x, y) == case["ops"]["mul"]
        assert oracle.e3_mul(x, x) == case["ops"]["sq"]
        assert [(u + v) % P for u, v in zip(x, y)] == case["ops"]["add"]


def test_blake3_known_answers(oracle):
    for case in GOLD["blake3"]:
        for msg, dig in zip(case["messages"], case["digests"]):
            assert oracle.blake3(bytes.fromhex(msg)).hex() == dig
    # empty message (BLAKE3 spec / blake3_engine.hpp:102-107)
    assert oracle.blake3(b"").hex() == "af1349b9f5f9a1a6a0404dea36dcc9499bcb25c9adc112b7cc9a93cae41f3262"


def test_merkle_known_answers(oracle):
    for case in GOLD["merkle"]:
        leaves = bytes.fromhex(case["leaves"])
        assert oracle.merkle_root(leaves).hex() == case["root"]
        assert [h.hex() for h in oracle.merkle_open(leaves, case["indices"])] == case["hints"]


def test_sha256_known_answers(oracle):
    """The reference's SHA-256 engine dumps (hash_output, sha2 cases) and hashlib."""
    for case in GOLD["sha2"]:
        for msg, dig in zip(case["messages"], case["digests"]):
            assert oracle.sha256(bytes.fromhex(msg)).hex() == dig
            assert hashlib.sha256(bytes.fromhex(msg)).hexdigest() == dig
    for n in (0, 55, 56, 63, 64, 119, 120, 128, 384):
        m = bytes((7 * i + 3) & 0xFF for i in range(n))
        assert oracle.sha256(m) == hashlib.sha256(m).digest()


def test_merkle_sha2_known_answers(oracle):
    for case in GOLD["merkle_sha2"]:
        leaves = bytes.fromhex(case["leaves"])
        assert oracle.merkle_root(leaves, sha2=True).hex() == case["root"]
        assert [h.hex() for h in oracle.merkle_open(leaves, case["indices"], sha2=True)] == case["hints"]


def test_matrix_commit_leaves(oracle):
    for case in GOLD["matrix_commit"]:
        for row, leaf in zip(case["rows"], case["leaves"]):
            assert oracle.blake3(bytes.fromhex(row)).hex() == leaf


def test_challenge_indices(oracle):
    for case in GOLD["indices"]:
        got = oracle.indices(bytes(case["entropy"]), case["num_leaves"], case["count"], case["dedup"])
        assert got == case["indices"]


def test_pow_known_answer(oracle):
    g = GOLD["pow"]
    ch = bytes.fromhex(g["challenge"])
    assert oracle.find_nonce(ch, g["threshold"]) == g["nonce"]
    msg = ch + struct.pack("<Q", g["nonce"]) + bytes(24)
    assert oracle.blake3(msg).hex() == g["hash"]


def test_sumcheck_transcript_base_field(oracle):
    """The reference's base-field sumcheck dump: SHAKE128 duplex, 40-byte challenge
    decoding, c0/c2 messages and folds (cpp/tests/dump_sumcheck.cpp)."""
    g = GOLD["sumcheck"]
    t = oracle.tx()
    t.absorb(bytes.fromhex(g["protocol_id"]))
    t.absorb(bytes.fromhex(g["session_id"]))
    a, b, s = list(g["a"]), list(g["b"]), g["sum"]
    for rnd in g["rounds"]:
        h = len(a) // 2
        c0 = sum(a[i] * b[i] for i in range(h)) % P
        c2 = sum((a[h + i] - a[i]) * (b[h + i] - b[i]) for i in range(h)) % P
        assert (c0, c2) == (rnd["c0"], rnd["c2"])
        t.message(struct.pack("<Q", c0))
        t.message(struct.pack("<Q", c2))
        r = t.challenge_base()
        assert r == rnd["r"]
        a = [(a[i] + r * (a[h + i] - a[i])) % P for i in range(h)]
        b = [(b[i] + r * (b[h + i] - b[i])) % P for i in range(h)]
        c1 = (s - 2 * c0 - c2) % P
        s = ((c2 * r + c1) * r + c0) % P
        assert s == rnd["sum"]
    assert t.narg().hex() == g["narg"]


def _case_inputs(case):
    n = case["n"]
    coeffs = sample_goldilocks(case["seed"], 1 << n)
    points = sample_goldilocks(case["seed"] + 5000, case["n_points"] * n * 3).reshape(case["n_points"], n, 3)
    return coeffs, points


@pytest.mark.parametrize("case", PROOFS,
                         ids=lambda c: f"n{c['n']}k{c['k']}r{c['rho']}s{c['security']}p{c['pow_bits']}{c['hash']}")
def test_oracle_proofs_match_reference_fixtures(oracle, case):
    coeffs, points = _case_inputs(case)
    evals = np.array(case["evaluations"], dtype=np.uint64)
    for i in range(case["n_points"]):
        assert [int(x) for x in oracle.mle_eval_base(coeffs, points[i])] == case["evaluations"][i]
    narg, hints = oracle.prove(case["n"], case["k"], case["rho"], case["security"], case["pow_bits"], points, coeffs,
                               evals, sha2=case["hash"] == "sha2")
    assert (len(narg), len(hints)) == (case["narg_len"], case["hints_len"])
    assert hashlib.sha256(narg).hexdigest() == case["narg_sha256"]
    assert hashlib.sha256(hints).hexdigest() == case["hints_sha256"]
    if "narg" in case:
        assert narg.hex() == case["narg"] and hints.hex() == case["hints"]


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("n,k,rho,sec,pb,seed,sha2", [(6, 2, 1, 90, 12, 901, False), (11, 4, 2, 100, 20, 902, False),
                                                      (15, 3, 1, 100, 18, 903, False), (9, 4, 2, 100, 20, 904, True)])
def test_oracle_matches_live_reference(oracle, n, k, rho, sec, pb, seed, sha2):
    coeffs = sample_goldilocks(seed, 1 << n)
    points = sample_goldilocks(seed + 1, n * 3).reshape(1, n, 3)
    ref = run_reference(n, k, rho, sec, pb, points, coeffs, verify=True, sha2=sha2)
    assert ref.verify_ok == 1.0
    narg, hints = oracle.prove(n, k, rho, sec, pb, points, coeffs, ref.evaluations, sha2=sha2)
    assert narg == ref.narg and hints == ref.hints


MULTI = json.load(open(os.path.join(HERE, "golden", "reference_proofs.json")))["multi"]


def _multi_inputs(case):
    n, nvec = case["n"], case["batch_size"] * case["num_witnesses"]
    coeffs = sample_goldilocks(case["seed"], nvec << n).reshape(nvec, 1 << n)
    points = sample_goldilocks(case["seed"] + 5000, case["n_points"] * n * 3).reshape(case["n_points"], n, 3)
    return coeffs, points


@pytest.mark.parametrize("case", MULTI, ids=lambda c: f"n{c['n']}k{c['k']}r{c['rho']}"
                                                      f"b{c['batch_size']}w{c['num_witnesses']}{c['hash']}")
def test_oracle_multi_vector_proofs_match_reference_fixtures(oracle, case):
    """Several committed vectors: rows of batch_size * 2^k elements, OOD values of
    every vector, OOD completion across witnesses, the vector RLC and the
    first opening weighted by vector_rlc (x) eq."""
    coeffs, points = _multi_inputs(case)
    nvec = coeffs.shape[0]
    for i in range(case["n_points"]):
        for j in range(nvec):
            assert [int(x) for x in oracle.mle_eval_base(coeffs[j], points[i])] == case["evaluations"][i * nvec + j]
    evals = np.array(case["evaluations"], dtype=np.uint64).reshape(-1, 3)
    narg, hints = oracle.prove_multi(case["n"], case["k"], case["rho"], case["security"], case["pow_bits"], points,
                                     coeffs, evals, case["batch_size"], case["num_witnesses"],
                                     sha2=case["hash"] == "sha2")
    assert (len(narg), len(hints)) == (case["narg_len"], case["hints_len"])
    assert hashlib.sha256(narg).hexdigest() == case["narg_sha256"]
    assert hashlib.sha256(hints).hexdigest() == case["hints_sha256"]
    if "narg" in case:
        assert narg.hex() == case["narg"] and hints.hex() == case["hints"]


def test_blake3_multi_chunk_tree(oracle):
    """Messages above one chunk take the tree path without error and give
    distinct digests at every chunk boundary.  Its values are pinned end to
    end by the multi-vector reference proofs above, whose leaves are rows of
    1280, 1536 and 2048 bytes."""
    msg = bytes((i * 7 + 3) & 0xFF for i in range(4096 + 17))
    seen = {oracle.blake3(msg[:m]) for m in (1024, 1025, 2048, 2049, 3072, 4096, 4113)}
    assert len(seen) == 7


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("n,k,rho,batch,nwit,seed,sha2", [(8, 4, 1, 2, 2, 911, False), (10, 5, 1, 5, 1, 912, False),
                                                          (9, 4, 2, 3, 2, 913, True), (7, 2, 1, 40, 1, 914, False)])
def test_oracle_multi_vector_matches_live_reference(oracle, n, k, rho, batch, nwit, seed, sha2):
    nvec = batch * nwit
    coeffs = sample_goldilocks(seed, nvec << n).reshape(nvec, 1 << n)
    points = sample_goldilocks(seed + 1, 2 * n * 3).reshape(2, n, 3)
    ref = run_reference(n, k, rho, 100, 20, points, coeffs, verify=True, sha2=sha2, batch_size=batch,
                        num_witnesses=nwit)
    assert ref.verify_ok == 1.0
    narg, hints = oracle.prove_multi(n, k, rho, 100, 20, points, coeffs, ref.evaluations, batch, nwit, sha2=sha2)
    assert narg == ref.narg and hints == ref.hints


FORMS = json.load(open(os.path.join(HERE, "golden", "reference_proofs.json")))["forms"]


@pytest.mark.parametrize("case", FORMS, ids=lambda c: f"n{c['n']}-{'-'.join(c['kinds'])}"
                                                      f"-b{c['batch_size']}w{c['num_witnesses']}{c['hash']}")
def test_oracle_covector_statements_match_reference_fixtures(oracle, case):
    """Statements that mix MultilinearExtension and dense Covector forms
    (linear_form.hpp:54-138): the covector accumulates scalar * vector."""
    from tests.golden.forms import form_inputs

    coeffs, forms = form_inputs(case["n"], case["seed"], case["kinds"], case["batch_size"] * case["num_witnesses"])
    evals = np.array(case["evaluations"], dtype=np.uint64).reshape(-1, 3)
    narg, hints = oracle.prove_forms(case["n"], case["k"], case["rho"], case["security"], case["pow_bits"], forms,
                                     coeffs, evals, case["batch_size"], case["num_witnesses"],
                                     sha2=case["hash"] == "sha2")
    assert (len(narg), len(hints)) == (case["narg_len"], case["hints_len"])
    assert hashlib.sha256(narg).hexdigest() == case["narg_sha256"]
    assert hashlib.sha256(hints).hexdigest() == case["hints_sha256"]
    if "narg" in case:
        assert narg.hex() == case["narg"] and hints.hex() == case["hints"]


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built")
def test_oracle_covector_statement_matches_live_reference(oracle):
    from tests.golden.forms import form_inputs

    n, kinds = 12, ("covector", "mle", "covector")
    coeffs, forms = form_inputs(n, 921, kinds, 2)
    ref = run_reference(n, 4, 2, 100, 20, None, coeffs, verify=True, batch_size=2, forms=forms)
    assert ref.verify_ok == 1.0
    narg, hints = oracle.prove_forms(n, 4, 2, 100, 20, forms, coeffs, ref.evaluations, 2, 1)
    assert narg == ref.narg and hints == ref.hints


UNIQUE = json.load(open(os.path.join(HERE, "golden", "reference_proofs.json")))["unique"]


@pytest.mark.parametrize("case", UNIQUE, ids=lambda c: f"n{c['n']}-{'-'.join(c['kinds']) or 'none'}"
                                                       f"-b{c['batch_size']}w{c['num_witnesses']}{c['hash']}")
def test_oracle_unique_decoding_matches_reference_fixtures(oracle, case):
    """Unique decoding (no OOD samples); without linear forms the proof has no
    constraint: the folding randomness is squeezed directly, the skip-PoW runs
    and the vector is folded without a sumcheck (whir_prover.hpp:211-218)."""
    from tests.golden.forms import form_inputs

    coeffs, forms = form_inputs(case["n"], case["seed"], case["kinds"], case["batch_size"] * case["num_witnesses"])
    evals = np.array(case["evaluations"], dtype=np.uint64).reshape(-1, 3)
    narg, hints = oracle.prove_forms(case["n"], case["k"], case["rho"], case["security"], case["pow_bits"], forms,
                                     coeffs, evals, case["batch_size"], case["num_witnesses"],
                                     sha2=case["hash"] == "sha2", unique=True)
    assert (len(narg), len(hints)) == (case["narg_len"], case["hints_len"])
    assert hashlib.sha256(narg).hexdigest() == case["narg_sha256"]
    assert hashlib.sha256(hints).hexdigest() == case["hints_sha256"]
    if "narg" in case:
        assert narg.hex() == case["narg"] and hints.hex() == case["hints"]


def whir_golden_config(case):
    """The Config of cpp/tests/dump_whir.cpp:run_case as oracle/GPU config words:
    depth 1, codeword 2x, min(size, 3) queries, 1 OOD sample, no initial
    sumcheck round, no STIR round, final sumcheck to size 1, no PoW."""
    size = case["vector_size"]
    none = (1 << 64) - 1
    log_size = size.bit_length() - 1
    return [size, 2 * size, 1, min(size, 3), 1, 0, none, none, 0, log_size, none, none]


def whir_golden_ds(case):
    proto = hashlib.sha3_512(bytes([0x19, 0xBE, 0xEF])).digest()
    label = f"whir_{case['case']}".encode()
    sess = hashlib.sha3_256(bytes([0x60 + len(label)]) + label).digest()
    return proto + sess


@pytest.mark.parametrize("case", GOLD["whir"], ids=lambda c: f"case{c['case']}")
def test_oracle_matches_reference_whir_golden(oracle, case):
    """Whole proofs of the reference's WHIR golden dump (C++ and Rust identical):
    Identity<Goldilocks>, SHA-2 Merkle, a hand-built Config, one all-ones
    Covector form, several vectors in cases 3 and 4."""
    P = 0xFFFFFFFF00000001
    size = case["vector_size"]
    coeffs = np.array(case["inputs"], dtype=np.uint64)
    ones = np.zeros((size, 3), dtype=np.uint64)
    ones[:, 0] = 1
    evals = np.array([[sum(v) % P, 0, 0] for v in case["inputs"]], dtype=np.uint64)
    narg, hints, ep = oracle.prove_config(whir_golden_config(case), whir_golden_ds(case), [("covector", ones)], coeffs,
                                          evals, batch_size=case["num_vectors"], deg=1, sha2=True)
    assert narg.hex() == case["narg"]
    assert hints.hex() == case["hints"]
    assert [int(x) for x in ep[:, 0]] == case["eval_point"] and not ep[:, 1:].any()


FIELD1 = json.load(open(os.path.join(HERE, "golden", "reference_proofs.json")))["field1"]


@pytest.mark.parametrize("case", FIELD1, ids=lambda c: f"n{c['n']}-{'-'.join(c['kinds']) or 'none'}"
                                                       f"-b{c['batch_size']}w{c['num_witnesses']}{c['hash']}")
def test_oracle_goldilocks1_matches_reference_fixtures(oracle, case):
    """Identity<Goldilocks> (the CLI's --field Goldilocks1): challenges, sums and
    messages in the base field, field_size_bits 64 in from_params."""
    from tests.golden.forms import form_inputs

    coeffs, forms = form_inputs(case["n"], case["seed"], case["kinds"], case["batch_size"] * case["num_witnesses"],
                                base_field=True)
    evals = np.array(case["evaluations"], dtype=np.uint64).reshape(-1, 3)
    narg, hints = oracle.prove_forms(case["n"], case["k"], case["rho"], case["security"], case["pow_bits"], forms,
                                     coeffs, evals, case["batch_size"], case["num_witnesses"],
                                     sha2=case["hash"] == "sha2", unique=case["unique_decoding"], field1=True)
    assert (len(narg), len(hints)) == (case["narg_len"], case["hints_len"])
    assert hashlib.sha256(narg).hexdigest() == case["narg_sha256"]
    assert hashlib.sha256(hints).hexdigest() == case["hints_sha256"]
    if "narg" in case:
        assert narg.hex() == case["narg"] and hints.hex() == case["hints"]
