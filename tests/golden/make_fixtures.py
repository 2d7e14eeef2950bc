#!/usr/bin/env python3
"""Regenerates the committed fixtures in tests/golden/ (run in a container that
has the reference checkout; the tests only read the JSON files).

1. reference_goldens.json -- the known-answer vectors of the reference's own
   golden dumps (cpp/dump_output/*/golden_*_cpp.txt, identical to the
   *_rs.txt dumps of the Rust crate for these sections), restricted to the
   sections on the WHIR path: whole WHIR proofs (whir_output, Identity<Goldilocks>,
   identical in the Rust and C++ dumps), field arithmetic (base, Ext3), BLAKE3 hashes,
   Merkle roots and opening hints, matrix-commit leaves, challenge indices and
   proof of work; plus the base-field sumcheck transcript, taken from the
   reference's sumcheck dumper rebuilt from its current sources (its committed
   dump predates the current transcript, see sumcheck()).  Inputs that the
   dumpers draw from their LCG (cpp/tests/dump_hash.cpp,
   dump_matrix_commit.cpp) are regenerated here with the same LCG rule and
   stored next to the outputs.
2. reference_proofs.json -- whole proofs of the unmodified reference prover
   (oracle/_ref/ref_driver, built by oracle/Makefile) on seeded inputs:
   lengths and SHA-256 digests of narg and hints (full bytes for the smallest);
   "multi" holds proofs over several committed vectors (batch_size > 1,
   several witnesses), including rows wider than one BLAKE3 chunk; "forms"
   statements that mix MultilinearExtension and dense Covector linear forms;
   "unique" proofs under unique decoding, including statement-free ones;
   "field1" proofs over Identity<Goldilocks> (the CLI's --field Goldilocks1);
   "field2" proofs over Basefield<GoldilocksExt2> (--field Goldilocks2);
   "zk" zero-knowledge WHIR proofs (oracle/_ref/ref_zk_driver, masks from the
   reference's DeterministicRng with the case's seed).
"""
import hashlib
import json
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
DUMPS = os.path.join(os.environ.get("WHIR_REFERENCE_CPP", "/root/reference/cpp"), "dump_output")

MASK = (1 << 64) - 1


class Lcg:  # the dumpers' generator: s = s * 6364136223846793005 + 1442695040888963407
    def __init__(self, seed):
        self.s = seed

    def next(self):
        self.s = (self.s * 6364136223846793005 + 1442695040888963407) & MASK
        return self.s


def read(path):
    raw = open(path, "rb").read()
    if raw[:2] in (b"\xff\xfe", b"\xfe\xff"):
        return raw.decode("utf-16")
    return raw.decode("utf-8")


def sections(text):
    out, cur = {}, None
    for line in text.splitlines():
        m = re.match(r"# SECTION (\S+)", line)
        if m:
            cur = m.group(1)
            out[cur] = []
        elif cur:
            out[cur].append(line.rstrip())
    return out


def cases(lines):
    res, cur = [], None
    for ln in lines:
        if ln.startswith("CASE"):
            cur = {"head": ln, "rows": []}
            res.append(cur)
        elif cur is not None and ln.strip():
            cur["rows"].append(ln.strip())
    return res


def fields():
    sec = sections(read(f"{DUMPS}/field_ouput/golden_fields_cpp.txt"))
    out = {}
    for name in ("base", "ext3"):
        lst = []
        for c in cases(sec[name]):
            ins = [int(x) for x in c["head"].split()[2:]]
            ops = {}
            for r in c["rows"]:
                parts = r.split()
                ops[parts[0]] = [int(x) for x in parts[1:]]
            lst.append({"inputs": ins, "ops": ops})
        out[name] = lst
    return out


def hashes(engine="blake3"):
    rng = Lcg(0xAAAAAAAAAAAAAAAA)

    def make_bytes(n):
        v = bytearray()
        while len(v) < n:
            w = rng.next()
            for _ in range(8):
                if len(v) < n:
                    v.append(w & 0xFF)
                    w >>= 8
        return bytes(v)

    spec = [("copy", 0, 2), ("copy", 16, 2), ("copy", 32, 3), ("blake3", 64, 1), ("blake3", 64, 4),
            ("blake3", 128, 2), ("blake3", 256, 1), ("blake3", 1024, 1), ("sha2", 0, 1), ("sha2", 31, 1),
            ("sha2", 32, 3), ("sha2", 64, 2), ("sha2", 100, 2)]
    got = cases(sections(read(f"{DUMPS}/hash_output/golden_hash_cpp.txt"))["hash"])
    out = []
    for (eng, size, cnt), c in zip(spec, got):
        data = make_bytes(size * cnt)
        assert f"{eng} size={size} count={cnt}" in c["head"], c["head"]
        if eng != engine:
            continue
        digests = [r.split()[1] for r in c["rows"]]
        out.append({"size": size, "messages": [data[i * size:(i + 1) * size].hex() for i in range(cnt)],
                    "digests": digests})
    return out


def merkle(engine="blake3"):
    got = cases(sections(read(f"{DUMPS}/merkle_tree_output/golden_merkle_tree_cpp.txt"))["merkle_tree"])
    spec = [("blake3", 16, [3, 5, 11]), ("blake3", 32, [0, 1, 2, 31]), ("sha2", 8, [2, 6])]
    out = []
    for (eng, nl, idx), c in zip(spec, got):
        if eng != engine:
            continue
        leaves = bytes(((i * 31 + j) & 0xFF) for i in range(nl) for j in range(32))
        rows = {r.split()[0]: r.split()[1] for r in c["rows"]}
        hints = [rows[f"hint{i}"] for i in range(int(rows["num_hints"]))]
        out.append({"leaves": leaves.hex(), "indices": idx, "root": rows["root"], "hints": hints})
    return out


def matrix_commit():
    rng = Lcg(0xBBBBBBBBBBBBBBBB)
    got = cases(sections(read(f"{DUMPS}/matrix_commit_output/golden_matrix_commit_cpp.txt"))["matrix_commit"])
    P = 0xFFFFFFFF00000001

    def fe():
        v = rng.next()
        return v - P if v >= P else v

    out = []
    # case 0: base rows (4 x 8), BLAKE3; case 1: Ext2 rows (2 x 8), BLAKE3 -- both LE words per element
    specs = [(4, 8, 1), (2, 8, 2), (3, 5, 3), (2, 4, 1), (3, 4, 1)]
    for ci, ((nr, nc, width), c) in enumerate(zip(specs, got)):
        words = [fe() for _ in range(nr * nc * width)]
        if ci > 1:
            continue  # SHA2 / Copy engines are not on the BLAKE3 path
        rows = []
        for r in range(nr):
            seg = words[r * nc * width:(r + 1) * nc * width]
            rows.append(b"".join(w.to_bytes(8, "little") for w in seg).hex())
        leaves = [x.split()[1] for x in c["rows"]]
        out.append({"rows": rows, "leaves": leaves})
    return out


def indices():
    got = cases(sections(read(f"{DUMPS}/indices_output/golden_indices_cpp.txt"))["challenge_indices"])
    ent = [[0x01, 0x23, 0x45, 0x67, 0x89], [0x01, 0x23, 0x45, 0x67, 0x89],
           [0x01, 0x23, 0x45, 0x67, 0x89, 0xAB, 0xCD, 0xEF, 0x12, 0x34],
           [0x12, 0x34, 0x56, 0x78, 0x9A, 0xBC, 0xDE, 0xF0, 0x11, 0x22, 0x33, 0x44],
           [0x20, 0x40, 0x20, 0x60, 0x40], [], [], []]
    out = []
    for e, c in zip(ent, got):
        m = re.search(r"num_leaves=(\d+) count=(\d+) dedup=(\w+)", c["head"])
        idx = [int(x) for x in c["rows"][0].split()[1:]] if c["rows"] else []
        out.append({"num_leaves": int(m.group(1)), "count": int(m.group(2)), "dedup": m.group(3) == "true",
                    "entropy": e, "indices": idx})
    return out


def pow_golden():
    c = cases(sections(read(f"{DUMPS}/pow_output/golden_pow_cpp.txt"))["pow"])[0]
    rows = {r.split()[0]: r.split()[1] for r in c["rows"]}
    return {"challenge": "aa" * 32, "threshold": 1 << 60, "nonce": int(rows["nonce"]), "hash": rows["hash"]}


def sumcheck():
    """Base-field sumcheck transcript of cpp/tests/dump_sumcheck.cpp, taken from
    the dumper rebuilt from the current reference sources (oracle/_ref/dump_sumcheck).
    The committed dump (sumcheck_output/golden_sumcheck_cpp.txt) agrees on round 0's
    c0/c2 but not on the challenges: it predates the current transcript."""
    exe = os.path.join(ROOT, "oracle", "_ref", "dump_sumcheck")
    text = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    lines = sections(text)["sumcheck"]
    out = {"rounds": []}
    for ln in lines:
        parts = ln.split()
        if not parts:
            continue
        if parts[0] == "vector_a":
            out["a"] = [int(x) for x in parts[1:]]
        elif parts[0] == "vector_b":
            out["b"] = [int(x) for x in parts[1:]]
        elif parts[0] == "initial_sum":
            out["sum"] = int(parts[1])
        elif parts[0] == "proof_narg":
            out["narg"] = parts[1]
        elif parts[0] == "CASE" and parts[1] == "2":
            break
        m = re.match(r"round(\d+)_(c0|c2|r|sum)", parts[0])
        if m:
            i = int(m.group(1))
            while len(out["rounds"]) <= i:
                out["rounds"].append({})
            out["rounds"][i][m.group(2)] = int(parts[1])
    committed = sections(read(f"{DUMPS}/sumcheck_output/golden_sumcheck_cpp.txt"))["sumcheck"]
    old_r0 = [int(ln.split()[1]) for ln in committed if ln.strip().startswith("round0_r")][0]
    out["committed_dump_round0_r"] = old_r0
    out["source"] = "oracle/_ref/dump_sumcheck (current reference sources)"
    # domain separator of dump_sumcheck.cpp: SHA3-512 of CBOR uint 0xABCD, SHA3-256 of CBOR text "sumcheck_dump"
    out["protocol_id"] = hashlib.sha3_512(bytes([0x19, 0xAB, 0xCD])).hexdigest()
    out["session_id"] = hashlib.sha3_256(bytes([0x6D]) + b"sumcheck_dump").hexdigest()
    return out


PROOF_CASES = [  # (n, k, rho, security, pow_bits, seed, n_points[, hash engine])
    (4, 4, 1, 100, 20, 11, 1), (5, 4, 1, 100, 20, 12, 1), (8, 4, 1, 100, 20, 13, 1), (9, 2, 2, 80, 10, 14, 1),
    (10, 4, 1, 100, 20, 15, 2), (12, 3, 2, 100, 20, 16, 1), (13, 1, 1, 64, 16, 17, 1), (14, 4, 1, 100, 20, 18, 1),
    (16, 4, 3, 100, 0, 19, 1), (18, 4, 1, 100, 20, 20, 1), (20, 4, 2, 128, 20, 21, 1),
    (5, 4, 1, 100, 20, 31, 1, "sha2"), (10, 4, 2, 100, 20, 32, 1, "sha2"), (14, 4, 1, 100, 20, 33, 2, "sha2"),
    (16, 4, 3, 100, 16, 34, 1, "sha2"),
]


def proofs():
    from oracle.refio import run_reference
    from whirplonk_b200 import sample_goldilocks

    out = []
    for case in PROOF_CASES:
        n, k, rho, sec, pb, seed, npts = case[:7]
        sha2 = len(case) > 7 and case[7] == "sha2"
        coeffs = sample_goldilocks(seed, 1 << n)
        points = sample_goldilocks(seed + 5000, npts * n * 3).reshape(npts, n, 3)
        ref = run_reference(n, k, rho, sec, pb, points, coeffs, verify=True, sha2=sha2)
        assert ref.verify_ok == 1.0
        rec = {"n": n, "k": k, "rho": rho, "security": sec, "pow_bits": pb, "seed": seed, "n_points": npts,
               "hash": "sha2" if sha2 else "blake3",
               "evaluations": [[int(x) for x in row] for row in ref.evaluations],
               "narg_len": len(ref.narg), "hints_len": len(ref.hints),
               "narg_sha256": hashlib.sha256(ref.narg).hexdigest(),
               "hints_sha256": hashlib.sha256(ref.hints).hexdigest()}
        if n <= 5:
            rec["narg"] = ref.narg.hex()
            rec["hints"] = ref.hints.hex()
        out.append(rec)
    return out


MULTI_CASES = [  # (n, k, rho, security, pow_bits, seed, n_points, batch_size, num_witnesses, hash engine)
    (5, 4, 1, 100, 20, 41, 1, 2, 2, "blake3"),    # small enough to store the bytes
    (10, 4, 1, 100, 20, 42, 1, 2, 1, "blake3"),
    (12, 4, 2, 100, 20, 43, 2, 4, 1, "blake3"),
    (10, 4, 1, 100, 20, 44, 1, 1, 2, "blake3"),   # OOD completion across witnesses
    (12, 4, 1, 100, 20, 45, 1, 2, 3, "blake3"),
    (10, 4, 1, 100, 20, 46, 1, 16, 1, "blake3"),  # 2048-byte rows: two BLAKE3 chunks
    (12, 6, 1, 100, 20, 47, 1, 3, 1, "blake3"),   # 1536-byte rows
    (11, 4, 2, 100, 20, 48, 1, 3, 2, "sha2"),
    (14, 4, 1, 100, 20, 49, 0, 2, 2, "blake3"),   # OOD constraints only
    (16, 4, 1, 100, 20, 50, 1, 4, 1, "blake3"),
    (9, 3, 1, 100, 20, 51, 1, 9, 1, "sha2"),      # 576-byte rows, SHA-256 with 10 blocks
]


def proofs_multi():
    from oracle.refio import run_reference
    from whirplonk_b200 import sample_goldilocks

    out = []
    for (n, k, rho, sec, pb, seed, npts, batch, nwit, eng) in MULTI_CASES:
        nvec = batch * nwit
        coeffs = sample_goldilocks(seed, nvec << n).reshape(nvec, 1 << n)
        points = sample_goldilocks(seed + 5000, npts * n * 3).reshape(npts, n, 3)
        ref = run_reference(n, k, rho, sec, pb, points, coeffs, verify=True, sha2=eng == "sha2",
                            batch_size=batch, num_witnesses=nwit)
        assert ref.verify_ok == 1.0
        rec = {"n": n, "k": k, "rho": rho, "security": sec, "pow_bits": pb, "seed": seed, "n_points": npts,
               "batch_size": batch, "num_witnesses": nwit, "hash": eng,
               "evaluations": [[int(x) for x in row] for row in ref.evaluations],
               "narg_len": len(ref.narg), "hints_len": len(ref.hints),
               "narg_sha256": hashlib.sha256(ref.narg).hexdigest(),
               "hints_sha256": hashlib.sha256(ref.hints).hexdigest()}
        if n <= 5:
            rec["narg"] = ref.narg.hex()
            rec["hints"] = ref.hints.hex()
        out.append(rec)
    return out


FORMS_CASES = [  # (n, k, rho, seed, form kinds, batch_size, num_witnesses, hash engine)
    (5, 4, 1, 61, ("covector",), 1, 1, "blake3"),
    (10, 4, 1, 62, ("covector",), 1, 1, "blake3"),
    (11, 4, 2, 63, ("mle", "covector", "mle"), 1, 1, "blake3"),
    (12, 4, 1, 64, ("covector", "mle"), 2, 2, "blake3"),
    (9, 3, 1, 65, ("covector", "covector"), 1, 1, "sha2"),
    (14, 4, 1, 66, ("mle", "covector"), 3, 1, "blake3"),
]


def proofs_forms():
    from oracle.refio import run_reference
    from tests.golden.forms import form_inputs

    out = []
    for (n, k, rho, seed, kinds, batch, nwit, eng) in FORMS_CASES:
        coeffs, forms = form_inputs(n, seed, kinds, batch * nwit)
        ref = run_reference(n, k, rho, 100, 20, None, coeffs, verify=True, sha2=eng == "sha2", batch_size=batch,
                            num_witnesses=nwit, forms=forms)
        assert ref.verify_ok == 1.0
        rec = {"n": n, "k": k, "rho": rho, "security": 100, "pow_bits": 20, "seed": seed, "kinds": list(kinds),
               "batch_size": batch, "num_witnesses": nwit, "hash": eng,
               "evaluations": [[int(x) for x in row] for row in ref.evaluations],
               "narg_len": len(ref.narg), "hints_len": len(ref.hints),
               "narg_sha256": hashlib.sha256(ref.narg).hexdigest(),
               "hints_sha256": hashlib.sha256(ref.hints).hexdigest()}
        if n <= 5:
            rec["narg"] = ref.narg.hex()
            rec["hints"] = ref.hints.hex()
        out.append(rec)
    return out


UNIQUE_CASES = [  # unique decoding (no OOD samples): (n, k, rho, seed, form kinds, batch_size, num_witnesses, hash)
    (5, 4, 1, 71, (), 1, 1, "blake3"),            # no constraint at all: folds without a sumcheck
    (10, 4, 1, 72, (), 1, 1, "blake3"),
    (12, 4, 2, 73, ("mle",), 1, 1, "blake3"),
    (12, 4, 1, 74, (), 2, 2, "blake3"),
    (9, 3, 1, 75, ("covector",), 1, 1, "sha2"),
    (16, 4, 1, 76, (), 1, 1, "blake3"),
]


def proofs_unique():
    from oracle.refio import run_reference
    from tests.golden.forms import form_inputs

    out = []
    for (n, k, rho, seed, kinds, batch, nwit, eng) in UNIQUE_CASES:
        coeffs, forms = form_inputs(n, seed, kinds, batch * nwit)
        ref = run_reference(n, k, rho, 100, 20, None, coeffs, verify=True, sha2=eng == "sha2", batch_size=batch,
                            num_witnesses=nwit, forms=forms, unique=True)
        assert ref.verify_ok == 1.0
        rec = {"n": n, "k": k, "rho": rho, "security": 100, "pow_bits": 20, "seed": seed, "kinds": list(kinds),
               "batch_size": batch, "num_witnesses": nwit, "hash": eng, "unique_decoding": True,
               "evaluations": [[int(x) for x in row] for row in ref.evaluations],
               "narg_len": len(ref.narg), "hints_len": len(ref.hints),
               "narg_sha256": hashlib.sha256(ref.narg).hexdigest(),
               "hints_sha256": hashlib.sha256(ref.hints).hexdigest()}
        if n <= 5:
            rec["narg"] = ref.narg.hex()
            rec["hints"] = ref.hints.hex()
        out.append(rec)
    return out


WHIR_GOLDEN_SHAPES = [(1, 2), (1, 4), (1, 8), (3, 4), (4, 8)]  # (num_vectors, vector_size), cpp/tests/dump_whir.cpp:197-205


def whir_zk_golden():
    """The reference's zero-knowledge dumper (cpp/tests/dump_whir_zk.cpp, built
    unmodified into oracle/_ref/dump_whir_zk; no dump of it is committed in the
    reference): n = 8, SHA-2, policy (4, 4, 4, 4), polynomial 17 i + 3, an
    all-ones Covector, the canonical ZK domain separator with session
    "whir_zk_0", DeterministicRng(0..31, "WHIR_ZK:mask"), PoW off."""
    import subprocess

    exe = os.path.join(ROOT, "oracle", "_ref", "dump_whir_zk")
    text = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    rows = {}
    for line in text.splitlines():
        if line.startswith("    "):
            k, _, v = line.strip().partition(" ")
            rows[k] = v.split()
    assert rows["verify"] == ["1"] and rows["check_eof"] == ["1"]
    return {"canonical_config": rows["canonical_config"][0], "ds_protocol_id": rows["ds_protocol_id"][0],
            "ds_session_id": rows["ds_session_id"][0],
            "input_vector0": [int(x) for x in rows["input_vector0"]],
            "f_hat_vector0": [int(x) for x in rows["f_hat_vector0"]],
            "blinding_m_poly0": [int(x) for x in rows["blinding_m_poly0"]],
            "narg": rows["proof_narg"][0], "hints": rows["proof_hints"][0]}


def whir_golden():
    """The reference's whole-proof golden (cpp/tests/dump_whir.cpp; the Rust
    dump golden_whir_rs.txt is byte-identical to the C++ one): Identity<Goldilocks>,
    a Config built field by field (depth 1, codeword 2x, 1 OOD sample,
    min(size, 3) queries, SHA-2 Merkle, no initial sumcheck round, no STIR round,
    final sumcheck to size 1, no PoW), one all-ones Covector form, the domain
    separator SHA3-512(CBOR uint 0xBEEF) / SHA3-256(CBOR text "whir_<case>")."""
    rs = read(f"{DUMPS}/whir_output/golden_whir_rs.txt")
    cpp = read(f"{DUMPS}/whir_output/golden_whir_cpp.txt")
    assert rs.replace("\r", "") == cpp.replace("\r", ""), "Rust and C++ WHIR goldens differ"
    out = []
    for i, c in enumerate(cases(sections(rs)["whir"])):
        nvec, size = WHIR_GOLDEN_SHAPES[i]
        rows = {}
        for r in c["rows"]:
            k, _, v = r.partition(" ")
            rows[k] = v.split()
        rec = {"case": i, "num_vectors": nvec, "vector_size": size,
               "inputs": [[int(x) for x in rows[f"input_vector{v}"]] for v in range(nvec)],
               "witness_matrix": [int(x) for x in rows["witness_matrix"]],
               "ood_points": [int(x) for x in rows["ood_points"]],
               "ood_matrix": [int(x) for x in rows["ood_matrix"]],
               "eval_point": [int(x) for x in rows["eval_point"]],
               "rlc_coeffs": [int(x) for x in rows["rlc_coeffs"]],
               "narg": rows["proof_narg"][0], "hints": rows["proof_hints"][0],
               "check_eof": int(rows["check_eof"][0])}
        assert all(len(v) == size for v in rec["inputs"])
        out.append(rec)
    return out


FIELD1_CASES = [  # Identity<Goldilocks> (the CLI's --field Goldilocks1), from_params with field_size_bits 64:
    # (n, k, rho, security, pow_bits, seed, form kinds, batch_size, num_witnesses, hash, unique_decoding)
    (5, 4, 1, 40, 10, 81, ("mle",), 1, 1, "blake3", False),
    (10, 4, 1, 40, 10, 82, ("mle",), 1, 1, "blake3", False),
    (12, 4, 2, 40, 10, 83, ("mle", "covector"), 2, 1, "blake3", False),
    (14, 3, 1, 32, 8, 84, ("mle",), 1, 1, "sha2", False),
    (11, 4, 1, 40, 10, 85, (), 1, 1, "blake3", True),
    (12, 4, 1, 36, 10, 86, ("covector",), 2, 2, "blake3", False),
]


def proofs_field1():
    from oracle.refio import run_reference
    from tests.golden.forms import form_inputs

    out = []
    for (n, k, rho, sec, pb, seed, kinds, batch, nwit, eng, unique) in FIELD1_CASES:
        coeffs, forms = form_inputs(n, seed, kinds, batch * nwit, base_field=True)
        ref = run_reference(n, k, rho, sec, pb, None, coeffs, verify=True, sha2=eng == "sha2", batch_size=batch,
                            num_witnesses=nwit, forms=forms, unique=unique, field1=True)
        assert ref.verify_ok == 1.0
        rec = {"n": n, "k": k, "rho": rho, "security": sec, "pow_bits": pb, "seed": seed, "kinds": list(kinds),
               "batch_size": batch, "num_witnesses": nwit, "hash": eng, "unique_decoding": unique,
               "evaluations": [[int(x) for x in row] for row in ref.evaluations],
               "narg_len": len(ref.narg), "hints_len": len(ref.hints),
               "narg_sha256": hashlib.sha256(ref.narg).hexdigest(),
               "hints_sha256": hashlib.sha256(ref.hints).hexdigest()}
        if n <= 5:
            rec["narg"] = ref.narg.hex()
            rec["hints"] = ref.hints.hex()
        out.append(rec)
    return out


FIELD2_CASES = [  # Basefield<GoldilocksExt2> (the CLI's --field Goldilocks2):
    # (n, k, rho, security, pow_bits, seed, form kinds, batch_size, num_witnesses, hash, unique_decoding)
    (5, 4, 1, 40, 10, 91, ("mle",), 1, 1, "blake3", False),
    (10, 4, 1, 40, 10, 92, ("mle",), 1, 1, "blake3", False),
    (12, 4, 2, 40, 10, 93, ("mle", "covector"), 2, 1, "blake3", False),
    (14, 3, 1, 32, 8, 94, ("mle",), 1, 1, "sha2", False),
    (11, 4, 1, 40, 10, 95, (), 1, 1, "blake3", True),
    (12, 4, 1, 36, 10, 96, ("covector",), 2, 2, "blake3", False),
    (18, 4, 1, 60, 16, 97, ("mle",), 1, 1, "blake3", False),
]


def proofs_field2():
    from oracle.refio import run_reference
    from tests.golden.forms import form_inputs

    out = []
    for (n, k, rho, sec, pb, seed, kinds, batch, nwit, eng, unique) in FIELD2_CASES:
        coeffs, forms = form_inputs(n, seed, kinds, batch * nwit, ext2=True)
        ref = run_reference(n, k, rho, sec, pb, None, coeffs, verify=True, sha2=eng == "sha2", batch_size=batch,
                            num_witnesses=nwit, forms=forms, unique=unique, field2=True)
        assert ref.verify_ok == 1.0
        rec = {"n": n, "k": k, "rho": rho, "security": sec, "pow_bits": pb, "seed": seed, "kinds": list(kinds),
               "batch_size": batch, "num_witnesses": nwit, "hash": eng, "unique_decoding": unique,
               "evaluations": [[int(x) for x in row] for row in ref.evaluations],
               "narg_len": len(ref.narg), "hints_len": len(ref.hints),
               "narg_sha256": hashlib.sha256(ref.narg).hexdigest(),
               "hints_sha256": hashlib.sha256(ref.hints).hexdigest()}
        if n <= 5:
            rec["narg"] = ref.narg.hex()
            rec["hints"] = ref.hints.hex()
        out.append(rec)
    return out


ZK_CASES = [  # zero-knowledge WHIR (ZkConfig<Goldilocks>), every PoW disabled as the reference's dumper does:
    # (n, k, rho, security, seed, form kinds, num_polynomials, hash, policy (q_delta_1, q_delta_2, t1, t2) or None)
    (8, 2, 1, 16, 101, ("covector",), 1, "sha2", (4, 4, 4, 4)),   # the shape of cpp/tests/dump_whir_zk.cpp
    (10, 2, 1, 16, 102, ("mle",), 1, "blake3", (4, 4, 4, 4)),
    (12, 3, 2, 20, 103, ("mle", "covector"), 2, "blake3", (6, 6, 6, 6)),
    (16, 4, 1, 32, 104, ("mle",), 1, "blake3", None),
    (18, 4, 1, 40, 105, ("mle", "covector"), 1, "sha2", None),
    # the limits: 8 polynomials (64 blinding vectors), 7 forms (8 in the blinding proof)
    (7, 1, 1, 8, 106, ("mle", "covector", "mle", "covector", "mle", "mle", "covector"), 8, "blake3", (1, 1, 1, 1)),
]


def proofs_zk():
    from oracle.refio import run_reference_zk
    from tests.golden.forms import form_inputs

    out = []
    for (n, k, rho, sec, seed, kinds, npolys, eng, policy) in ZK_CASES:
        polys, forms = form_inputs(n, seed, kinds, npolys, base_field=True)
        ref = run_reference_zk(n, k, rho, sec, 0, [(kind, d[:, 0]) for kind, d in forms], polys, seed,
                               sha2=eng == "sha2", no_pow=True, policy=policy or (0, 0, 0, 0))
        assert ref.verify_ok == 1.0
        rec = {"n": n, "k": k, "rho": rho, "security": sec, "seed": seed, "kinds": list(kinds),
               "num_polynomials": npolys, "hash": eng, "policy": list(policy) if policy else None,
               "evaluations": [int(x) for x in ref.evaluations],
               "num_blinding_variables": ref.num_blinding_variables, "blinded_queries": ref.blinded_queries,
               "blinding_batch": ref.blinding_batch,
               "narg_len": len(ref.narg), "hints_len": len(ref.hints),
               "narg_sha256": hashlib.sha256(ref.narg).hexdigest(),
               "hints_sha256": hashlib.sha256(ref.hints).hexdigest()}
        out.append(rec)
    return out


def main():
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True, stdout=subprocess.DEVNULL)
    gold = {"fields": fields(), "blake3": hashes(), "merkle": merkle(), "matrix_commit": matrix_commit(),
            "indices": indices(), "pow": pow_golden(), "sumcheck": sumcheck(),
            "sha2": hashes("sha2"), "merkle_sha2": merkle("sha2"), "whir": whir_golden(), "whir_zk": whir_zk_golden()}
    with open(os.path.join(HERE, "reference_goldens.json"), "w") as f:
        json.dump(gold, f, indent=1)
    with open(os.path.join(HERE, "reference_proofs.json"), "w") as f:
        json.dump({"generator": "oracle/_ref/ref_driver (reference C++ prover, CLI domain separator, "
                                "seeded ChaCha20 inputs via whirgpu_sample_goldilocks)", "cases": proofs(),
                   "multi": proofs_multi(), "forms": proofs_forms(), "unique": proofs_unique(),
                   "field1": proofs_field1(), "field2": proofs_field2(), "zk": proofs_zk()}, f, indent=1)


if __name__ == "__main__":
    main()
