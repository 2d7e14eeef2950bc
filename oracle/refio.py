"""Test infrastructure: run the reference C++ prover (oracle/_ref/ref_driver)
and the CPU restatement (oracle/liboracle.so) on the same inputs.

Only the tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline and
reference arms use this module; the product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess
import tempfile
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")
ORACLE_SO = os.path.join(HERE, "liboracle.so")


@dataclass
class RefProof:
    narg: bytes
    hints: bytes
    evaluations: np.ndarray  # (num_points, 3) uint64
    commit_ms: float
    prove_ms: float
    verify_ok: float  # 1.0 accepted, 0.0 rejected, -1.0 not run


def write_input(path, n, k, rho, sec, pow_bits, points, coeffs, batch_size=1, num_witnesses=1, forms=None):
    """Input file of ref_driver.cpp (format documented there).  ``coeffs`` holds
    batch_size * num_witnesses vectors of 2^n words back to back.  ``forms``
    (optional) replaces ``points``: a list of ("mle", (n, 3) array) or
    ("covector", (2^n, 3) array) linear forms in statement order."""
    coeffs = np.ascontiguousarray(coeffs, dtype=np.uint64)
    nvec = batch_size * num_witnesses
    assert coeffs.size == nvec << n
    multi = nvec != 1
    with open(path, "wb") as f:
        if forms is not None:
            f.write(struct.pack("<II", 0x49524857, 3))
            f.write(struct.pack("<6Q", n, k, rho, sec, pow_bits, len(forms)))
            f.write(struct.pack("<2Q", batch_size, num_witnesses))
            for kind, data in forms:
                data = np.ascontiguousarray(data, dtype=np.uint64)
                assert data.size == 3 * (n if kind == "mle" else 1 << n)
                f.write(struct.pack("<Q", 0 if kind == "mle" else 1))
                f.write(data.tobytes())
        else:
            points = np.ascontiguousarray(points, dtype=np.uint64).reshape(-1, n, 3)
            f.write(struct.pack("<II", 0x49524857, 2 if multi else 1))
            f.write(struct.pack("<6Q", n, k, rho, sec, pow_bits, points.shape[0]))
            if multi:
                f.write(struct.pack("<2Q", batch_size, num_witnesses))
            f.write(points.tobytes())
        f.write(coeffs.tobytes())


def read_output(path, num_points, num_vectors=1) -> RefProof:
    with open(path, "rb") as f:
        b = f.read()
    pos = 0
    (ln,) = struct.unpack_from("<Q", b, pos); pos += 8
    narg = b[pos:pos + ln]; pos += ln
    (lh,) = struct.unpack_from("<Q", b, pos); pos += 8
    hints = b[pos:pos + lh]; pos += lh
    cnt = num_points * num_vectors
    ev = np.frombuffer(b, dtype=np.uint64, count=3 * cnt, offset=pos).reshape(cnt, 3).copy()
    pos += 24 * cnt
    cms, pms, vok = struct.unpack_from("<3d", b, pos)
    return RefProof(narg, hints, ev, cms, pms, vok)


def ref_available() -> bool:
    return os.access(REF_DRIVER, os.X_OK)


def run_reference(n, k, rho, sec, pow_bits, points, coeffs, verify=False, reps=1, threads=None,
                  timeout=3600, sha2=False, batch_size=1, num_witnesses=1, forms=None, unique=False,
                  field1=False, field2=False) -> RefProof:
    """Runs the unmodified reference prover (compiled in place by oracle/Makefile).
    With several vectors the evaluations come back form-major, (num_forms * V, 3).
    ``forms`` (see write_input) replaces ``points`` for mixed MLE / Covector statements."""
    if not ref_available():
        raise FileNotFoundError(f"{REF_DRIVER} not built (make -C oracle ref)")
    env = dict(os.environ)
    if threads is not None:
        env["OMP_NUM_THREADS"] = str(threads)
    npts = len(forms) if forms is not None else np.asarray(points).reshape(-1, n, 3).shape[0]
    with tempfile.TemporaryDirectory() as td:
        inp, out = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        write_input(inp, n, k, rho, sec, pow_bits, points, coeffs, batch_size, num_witnesses, forms)
        cmd = [REF_DRIVER, inp, out] + (["--verify"] if verify else []) + (["--reps", str(reps)] if reps > 1 else [])
        if sha2:
            cmd.append("--sha2")
        if unique:
            cmd.append("--unique")
        if field1:
            cmd.append("--field1")
        if field2:
            cmd.append("--field2")
        subprocess.run(cmd, check=True, env=env, timeout=timeout, stdout=subprocess.DEVNULL)
        return read_output(out, npts, batch_size * num_witnesses)


REF_ZK_DRIVER = os.path.join(HERE, "_ref", "ref_zk_driver")


@dataclass
class RefZkProof:
    narg: bytes
    hints: bytes
    evaluations: np.ndarray  # (num_forms * num_polys,) uint64, form-major
    verify_ok: float
    num_blinding_variables: int
    blinded_queries: int
    blinding_batch: int
    prove_ms: float = 0.0  # commit + prove inside the driver


def run_reference_zk(n, k, rho, sec, pow_bits, forms, polys, seed, sha2=False, no_pow=True, policy=(0, 0, 0, 0),
                     verify=True, timeout=3600, threads=None) -> RefZkProof:
    """Runs the reference zero-knowledge WHIR prover (oracle/_ref/ref_zk_driver).
    ``forms``: [("mle", (n,) words) | ("covector", (2^n,) words)] over the base
    field; ``polys``: (num_polys, 2^n).  ``policy`` (q_delta_1, q_delta_2, t1, t2),
    all 0 to derive it from the parameters."""
    polys = np.ascontiguousarray(polys, dtype=np.uint64).reshape(-1, 1 << n)
    with tempfile.TemporaryDirectory() as td:
        inp, out = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(inp, "wb") as f:
            f.write(struct.pack("<II", 0x4B5A4857, 1))
            f.write(struct.pack("<14Q", n, k, rho, sec, pow_bits, len(forms), polys.shape[0], int(sha2),
                                int(no_pow), *policy, seed))
            for kind, data in forms:
                data = np.ascontiguousarray(data, dtype=np.uint64).reshape(-1)
                assert data.size == (n if kind == "mle" else 1 << n)
                f.write(struct.pack("<Q", 0 if kind == "mle" else 1))
                f.write(data.tobytes())
            f.write(polys.tobytes())
        cmd = [REF_ZK_DRIVER, inp, out] + (["--verify"] if verify else [])
        env = dict(os.environ, OMP_NUM_THREADS=str(threads)) if threads else None
        subprocess.run(cmd, check=True, timeout=timeout, stdout=subprocess.DEVNULL, env=env)
        b = open(out, "rb").read()
    pos = 0
    (ln,) = struct.unpack_from("<Q", b, pos); pos += 8
    narg = b[pos:pos + ln]; pos += ln
    (lh,) = struct.unpack_from("<Q", b, pos); pos += 8
    hints = b[pos:pos + lh]; pos += lh
    cnt = len(forms) * polys.shape[0]
    ev = np.frombuffer(b, dtype=np.uint64, count=cnt, offset=pos).copy(); pos += 8 * cnt
    (vok,) = struct.unpack_from("<d", b, pos); pos += 8
    nbv, q, nb = struct.unpack_from("<3Q", b, pos)
    pos += 24
    (ms,) = struct.unpack_from("<d", b, pos)
    return RefZkProof(narg, hints, ev, vok, nbv, q, nb, ms)


class OracleTranscript:
    """The oracle's SHAKE128 prover transcript (absorb / message / squeeze)."""

    def __init__(self, lib):
        self.lib = lib
        self.h = lib.oracle_tx_new()

    def __del__(self):
        if self.h:
            self.lib.oracle_tx_free(self.h)
            self.h = None

    def absorb(self, data: bytes):
        self.lib.oracle_tx_absorb(self.h, data, len(data))

    def message(self, data: bytes):
        self.lib.oracle_tx_message(self.h, data, len(data))

    def squeeze(self, n: int) -> bytes:
        b = ctypes.create_string_buffer(n)
        self.lib.oracle_tx_squeeze(self.h, b, n)
        return b.raw

    def challenge_base(self) -> int:
        return int(self.lib.oracle_tx_challenge_base(self.h))

    def challenge_e3(self) -> list:
        o = (ctypes.c_uint64 * 3)()
        self.lib.oracle_tx_challenge_e3(self.h, o)
        return list(o)

    def narg(self) -> bytes:
        n = self.lib.oracle_tx_narg(self.h, None, 0)
        b = ctypes.create_string_buffer(max(n, 1))
        self.lib.oracle_tx_narg(self.h, b, n)
        return b.raw[:n]


class Oracle:
    """ctypes view of oracle/liboracle.so (the CPU restatement)."""

    def __init__(self, path: str = ORACLE_SO):
        self.lib = L = ctypes.CDLL(path)
        u64, sz, p = ctypes.c_uint64, ctypes.c_size_t, ctypes.c_void_p
        L.oracle_blake3.argtypes = [p, sz, p]
        L.oracle_sha3_256.argtypes = [p, sz, p]
        L.oracle_sha3_512.argtypes = [p, sz, p]
        L.oracle_shake128.argtypes = [p, sz, p, sz]
        L.oracle_fmul.argtypes = [u64, u64]; L.oracle_fmul.restype = u64
        for nm in ("oracle_fadd", "oracle_fsub", "oracle_fpow"):
            getattr(L, nm).argtypes = [u64, u64]
            getattr(L, nm).restype = u64
        L.oracle_indices.argtypes = [p, u64, u64, ctypes.c_int, p]
        L.oracle_indices.restype = sz
        L.oracle_root_of_unity.argtypes = [u64]; L.oracle_root_of_unity.restype = u64
        L.oracle_e3_mul.argtypes = [p, p, p]
        L.oracle_ntt.argtypes = [p, sz]
        L.oracle_set_coset_major.argtypes = [ctypes.c_int]
        L.oracle_transpose_permute.argtypes = [u64, u64, u64]; L.oracle_transpose_permute.restype = u64
        L.oracle_rs_encode_base.argtypes = [p, sz, u64, u64, p]
        L.oracle_rs_commit_root.argtypes = [p, sz, u64, u64, p]
        L.oracle_rs_encode_e3.argtypes = [p, sz, u64, u64, p]
        L.oracle_merkle_root.argtypes = [p, sz, p, p]
        L.oracle_merkle_open.argtypes = [p, sz, p, sz, p, sz]; L.oracle_merkle_open.restype = sz
        L.oracle_find_nonce.argtypes = [p, u64]; L.oracle_find_nonce.restype = u64
        L.oracle_tx_new.restype = p
        L.oracle_tx_free.argtypes = [p]
        L.oracle_tx_absorb.argtypes = [p, p, sz]
        L.oracle_tx_message.argtypes = [p, p, sz]
        L.oracle_tx_squeeze.argtypes = [p, p, sz]
        L.oracle_tx_challenge_base.argtypes = [p]; L.oracle_tx_challenge_base.restype = u64
        L.oracle_tx_challenge_e3.argtypes = [p, p]
        L.oracle_tx_narg.argtypes = [p, p, sz]; L.oracle_tx_narg.restype = sz
        L.oracle_cli_domain_separator.argtypes = [u64, u64, u64, u64, ctypes.c_int, p]
        L.oracle_whir_config.argtypes = [u64, u64, u64, u64, u64, ctypes.c_int, p, sz]
        L.oracle_whir_config.restype = sz
        L.oracle_mle_eval_base.argtypes = [p, u64, p, p]
        L.oracle_whir_prove.argtypes = [u64, u64, u64, u64, u64, ctypes.c_int, p, p, sz, p, p, sz, p, sz, p,
                                        ctypes.c_int]
        L.oracle_sha256.argtypes = [p, sz, p]
        L.oracle_sha256.restype = None
        L.oracle_merkle_root_sha2.argtypes = [p, sz, p]
        L.oracle_merkle_root_sha2.restype = None
        L.oracle_merkle_open_sha2.argtypes = [p, sz, p, sz, p, sz]
        L.oracle_merkle_open_sha2.restype = sz
        L.oracle_find_nonce_sha2.argtypes = [p, u64]
        L.oracle_find_nonce_sha2.restype = u64
        L.oracle_whir_prove.restype = ctypes.c_int
        L.oracle_whir_prove_multi.argtypes = [u64, u64, u64, u64, u64, ctypes.c_int, u64, u64, p, p, sz, p, p, sz,
                                              p, sz, p, ctypes.c_int]
        L.oracle_whir_prove_multi.restype = ctypes.c_int
        L.oracle_whir_prove_forms.argtypes = [u64, u64, u64, u64, u64, ctypes.c_int, u64, u64, p, p, sz, p, p, p,
                                              sz, p, sz, p, ctypes.c_int]
        L.oracle_whir_prove_forms.restype = ctypes.c_int
        L.oracle_whir_prove_config.argtypes = [p, sz, ctypes.c_int, ctypes.c_int, p, u64, u64, p, p, sz, p, p, p, sz,
                                               p, sz, p, p, sz]
        L.oracle_whir_prove_config.restype = ctypes.c_int

    # -- primitives -------------------------------------------------------
    def blake3(self, data: bytes) -> bytes:
        out = ctypes.create_string_buffer(32)
        self.lib.oracle_blake3(data, len(data), out)
        return out.raw

    def sha256(self, data: bytes) -> bytes:
        out = ctypes.create_string_buffer(32)
        self.lib.oracle_sha256(data, len(data), out)
        return out.raw

    def indices(self, entropy: bytes, N: int, count: int, dedup: bool) -> list:
        out = (ctypes.c_uint64 * max(count, 1))()
        k = self.lib.oracle_indices(bytes(entropy), N, count, int(dedup), out)
        return list(out[:k])

    def e3_mul(self, a, b) -> list:
        x = (ctypes.c_uint64 * 3)(*a)
        y = (ctypes.c_uint64 * 3)(*b)
        o = (ctypes.c_uint64 * 3)()
        self.lib.oracle_e3_mul(x, y, o)
        return list(o)

    def tx(self):
        return OracleTranscript(self.lib)

    def ntt(self, v) -> np.ndarray:
        a = np.ascontiguousarray(v, dtype=np.uint64).copy()
        self.lib.oracle_ntt(a.ctypes.data, a.size)
        return a

    def rs_encode_base(self, v, N, depth) -> np.ndarray:
        v = np.ascontiguousarray(v, dtype=np.uint64)
        out = np.empty((N, depth), dtype=np.uint64)
        self.lib.oracle_rs_encode_base(v.ctypes.data, v.size, N, depth, out.ctypes.data)
        return out

    def rs_encode_e3(self, v, N, depth) -> np.ndarray:
        v = np.ascontiguousarray(v, dtype=np.uint64).reshape(-1, 3)
        out = np.empty((N, depth, 3), dtype=np.uint64)
        self.lib.oracle_rs_encode_e3(v.ctypes.data, v.shape[0], N, depth, out.ctypes.data)
        return out

    def set_coset_major(self, on: bool) -> None:
        """Codeword order of later commitments and openings: natural (the C++
        reference) or coset-major (the Rust crate without rs_in_order)."""
        self.lib.oracle_set_coset_major(int(bool(on)))

    def transpose_permute(self, k, rows, cols) -> int:
        return int(self.lib.oracle_transpose_permute(k, rows, cols))

    def rs_commit_root(self, v, N, depth) -> bytes:
        """Matrix-commitment root of one base vector: RS encode (N rows of
        `depth` elements), BLAKE3 leaves, Merkle root, in one C call."""
        v = np.ascontiguousarray(v, dtype=np.uint64)
        out = ctypes.create_string_buffer(32)
        self.lib.oracle_rs_commit_root(v.ctypes.data, v.size, N, depth, out)
        return out.raw

    def merkle_root(self, leaves: bytes, sha2: bool = False) -> bytes:
        out = ctypes.create_string_buffer(32)
        if sha2:
            self.lib.oracle_merkle_root_sha2(leaves, len(leaves) // 32, out)
        else:
            self.lib.oracle_merkle_root(leaves, len(leaves) // 32, out, None)
        return out.raw

    def merkle_open(self, leaves: bytes, idx, sha2: bool = False) -> list:
        idx = np.ascontiguousarray(idx, dtype=np.uint64)
        cap = 64 * max(1, idx.size)
        out = ctypes.create_string_buffer(32 * cap)
        if sha2:
            cnt = self.lib.oracle_merkle_open_sha2(leaves, len(leaves) // 32, idx.ctypes.data, idx.size, out, cap)
            return [out.raw[32 * i:32 * i + 32] for i in range(cnt)]
        cnt = self.lib.oracle_merkle_open(leaves, len(leaves) // 32, idx.ctypes.data, idx.size, out, cap)
        return [out.raw[32 * i:32 * i + 32] for i in range(cnt)]

    def find_nonce(self, challenge: bytes, threshold: int, sha2: bool = False) -> int:
        if sha2:
            return self.lib.oracle_find_nonce_sha2(challenge, threshold)
        return self.lib.oracle_find_nonce(challenge, threshold)

    def domain_separator(self, rho, k, sec, pow_bits, unique=False) -> bytes:
        out = ctypes.create_string_buffer(96)
        self.lib.oracle_cli_domain_separator(rho, k, sec, pow_bits, int(unique), out)
        return out.raw

    def whir_config(self, n, rho, k, sec, pow_bits, unique=False) -> list:
        out = (ctypes.c_uint64 * 512)()
        cnt = self.lib.oracle_whir_config(n, rho, k, sec, pow_bits, int(unique), out, 512)
        return list(out[:cnt])

    def mle_eval_base(self, coeffs, point) -> np.ndarray:
        coeffs = np.ascontiguousarray(coeffs, dtype=np.uint64)
        point = np.ascontiguousarray(point, dtype=np.uint64)
        n = point.size // 3
        out = np.zeros(3, dtype=np.uint64)
        self.lib.oracle_mle_eval_base(coeffs.ctypes.data, n, point.ctypes.data, out.ctypes.data)
        return out

    def prove(self, n, k, rho, sec, pow_bits, points, coeffs, evaluations, sha2=False):
        coeffs = np.ascontiguousarray(coeffs, dtype=np.uint64)
        points = np.ascontiguousarray(points, dtype=np.uint64).reshape(-1, n, 3)
        evals = np.ascontiguousarray(evaluations, dtype=np.uint64).reshape(-1, 3)
        cap = 64 << 20
        narg = ctypes.create_string_buffer(cap)
        hints = ctypes.create_string_buffer(cap)
        lens = (ctypes.c_uint64 * 2)()
        rc = self.lib.oracle_whir_prove(n, rho, k, sec, pow_bits, 0, coeffs.ctypes.data, points.ctypes.data,
                                        points.shape[0], evals.ctypes.data, narg, cap, hints, cap, lens,
                                        int(sha2))
        if rc != 0:
            raise RuntimeError("oracle prove failed")
        return narg.raw[:lens[0]], hints.raw[:lens[1]]

    def prove_multi(self, n, k, rho, sec, pow_bits, points, coeffs, evaluations, batch_size, num_witnesses,
                    sha2=False):
        """Commit num_witnesses witnesses of batch_size vectors, prove them together.
        coeffs: (V, 2^n); evaluations: (num_points * V, 3), form-major."""
        coeffs = np.ascontiguousarray(coeffs, dtype=np.uint64)
        points = np.ascontiguousarray(points, dtype=np.uint64).reshape(-1, n, 3)
        evals = np.ascontiguousarray(evaluations, dtype=np.uint64).reshape(-1, 3)
        cap = 64 << 20
        narg = ctypes.create_string_buffer(cap)
        hints = ctypes.create_string_buffer(cap)
        lens = (ctypes.c_uint64 * 2)()
        rc = self.lib.oracle_whir_prove_multi(n, rho, k, sec, pow_bits, 0, batch_size, num_witnesses,
                                              coeffs.ctypes.data, points.ctypes.data, points.shape[0],
                                              evals.ctypes.data, narg, cap, hints, cap, lens, int(sha2))
        if rc != 0:
            raise RuntimeError("oracle prove failed")
        return narg.raw[:lens[0]], hints.raw[:lens[1]]

    def prove_forms(self, n, k, rho, sec, pow_bits, forms, coeffs, evaluations, batch_size=1, num_witnesses=1,
                    sha2=False, unique=False, field1=False):
        """Statement of mixed linear forms: ``forms`` is a list of ("mle", (n, 3))
        or ("covector", (2^n, 3)) arrays; evaluations: (num_forms * V, 3)."""
        coeffs = np.ascontiguousarray(coeffs, dtype=np.uint64)
        kinds = (ctypes.c_int * max(len(forms), 1))(*[0 if kd == "mle" else 1 for kd, _ in forms])
        data = np.concatenate([np.ascontiguousarray(d, dtype=np.uint64).reshape(-1) for _, d in forms]) \
            if forms else np.zeros(1, dtype=np.uint64)
        evals = np.ascontiguousarray(evaluations, dtype=np.uint64).reshape(-1, 3)
        cap = 64 << 20
        narg = ctypes.create_string_buffer(cap)
        hints = ctypes.create_string_buffer(cap)
        lens = (ctypes.c_uint64 * 2)()
        rc = self.lib.oracle_whir_prove_forms(n, rho, k, sec, pow_bits, int(unique), batch_size, num_witnesses,
                                              coeffs.ctypes.data, kinds, len(forms), data.ctypes.data,
                                              evals.ctypes.data, narg, cap, hints, cap, lens,
                                              int(sha2) | (2 if field1 else 0))
        if rc != 0:
            raise RuntimeError("oracle prove failed")
        return narg.raw[:lens[0]], hints.raw[:lens[1]]

    def prove_config(self, cfg_words, ds96, forms, coeffs, evaluations, batch_size=1, num_witnesses=1, deg=3,
                     sha2=False):
        """Commit + prove for an explicit Config (word layout in oracle_capi.cpp)
        and domain separator; returns (narg, hints, evaluation_point (k, 3))."""
        cfg = np.ascontiguousarray(cfg_words, dtype=np.uint64)
        coeffs = np.ascontiguousarray(coeffs, dtype=np.uint64)
        kinds = (ctypes.c_int * max(len(forms), 1))(*[0 if kd == "mle" else 1 for kd, _ in forms])
        data = np.concatenate([np.ascontiguousarray(d, dtype=np.uint64).reshape(-1) for _, d in forms]) \
            if forms else np.zeros(1, dtype=np.uint64)
        evals = np.ascontiguousarray(evaluations, dtype=np.uint64).reshape(-1, 3)
        cap = 16 << 20
        narg = ctypes.create_string_buffer(cap)
        hints = ctypes.create_string_buffer(cap)
        lens = (ctypes.c_uint64 * 3)()
        ep = np.zeros((64, 3), dtype=np.uint64)
        rc = self.lib.oracle_whir_prove_config(cfg.ctypes.data, cfg.size, deg, int(sha2), bytes(ds96), batch_size,
                                               num_witnesses, coeffs.ctypes.data, kinds, len(forms),
                                               data.ctypes.data, evals.ctypes.data, narg, cap, hints, cap, lens,
                                               ep.ctypes.data, 64)
        if rc != 0:
            raise RuntimeError("oracle prove failed")
        return narg.raw[:lens[0]], hints.raw[:lens[1]], ep[:lens[2]]
