"""Python mirror of the reference WHIR prover API over the C ABI.

Names and call order follow the reference C++ API so a caller of
``whir::protocols::whir::Config<Basefield<GoldilocksExt3>>`` reads the same:

    params = ProtocolParameters(security_level=100, pow_bits=20, ...)
    config = Config.from_params(1 << n, params)            # whir.hpp:118
    ps = ProverState.from_ds(cli_domain_separator(params))  # transcript.hpp:605
    witness = config.commit(ps, vectors)                    # whir.hpp:303 (batch_size vectors)
    claim = config.prove(ps, vectors, [witness],
                         [MultilinearExtension(point)], [evaluation])  # whir_prover.hpp:56
    narg, hints = ps.proof()                                # transcript.hpp:653

Field elements are canonical Goldilocks words (ints / uint64 arrays); an Ext3
element is a triple (c0, c1, c2).  The device work happens in libwhirgpu.so;
this module only marshals arguments.
"""
from __future__ import annotations

import ctypes
import weakref
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib

P = 0xFFFFFFFF00000001
ENGINE_ID_BLAKE3 = bytes.fromhex("03e01749ebcc0477924254eb482066b864a8dd4d77252464ca6f5b6f5cc05b4c")
ENGINE_ID_SHA2 = bytes.fromhex("018eaa247cb8957ab1e9fdac885450403c5e7bda1acaaa504e4cc8f2f76bb076")


@dataclass
class ProtocolParameters:
    """whir::ProtocolParameters (cpp/include/whir/parameters.hpp:25-34)."""

    unique_decoding: bool = False
    starting_log_inv_rate: int = 1
    initial_folding_factor: int = 4
    folding_factor: int = 4
    security_level: int = 100
    pow_bits: int = 20
    batch_size: int = 1
    hash_id: bytes = ENGINE_ID_BLAKE3

    @classmethod
    def cli(cls, security_level=100, pow_bits=20, folding_factor=4, log_inv_rate=1, hash_id=ENGINE_ID_BLAKE3):
        """Parameters as the reference CLI builds them (cpp/main.cpp:315-323)."""
        return cls(False, log_inv_rate, folding_factor, folding_factor, security_level, pow_bits, 1, hash_id)

    def to_c(self) -> _lib.WhirParams:
        c = _lib.WhirParams()
        c.unique_decoding = int(self.unique_decoding)
        c.starting_log_inv_rate = self.starting_log_inv_rate
        c.initial_folding_factor = self.initial_folding_factor
        c.folding_factor = self.folding_factor
        c.security_level = self.security_level
        c.pow_bits = self.pow_bits
        c.batch_size = self.batch_size
        for i, b in enumerate(self.hash_id):
            c.hash_id[i] = b
        return c


@dataclass
class DomainSeparator:
    """protocol_id (64 B) and session_id (32 B) (transcript.hpp:506-540)."""

    protocol_id: bytes
    session_id: bytes


def cli_domain_separator(params: ProtocolParameters) -> DomainSeparator:
    """make_rust_cli_domain_separator (cpp/main.cpp:203-215)."""
    L = _lib.load()
    out = ctypes.create_string_buffer(96)
    c = params.to_c()
    _lib.check(L.whirgpu_cli_domain_separator(ctypes.byref(c), out))
    return DomainSeparator(out.raw[:64], out.raw[64:])


class Context:
    """One GPU, one stream, a workspace cache bounded by `hbm_budget` bytes."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self._L = _lib.load()
        self.device = device
        h = ctypes.c_void_p()
        _lib.check(self._L.whirgpu_ctx_create(device, hbm_budget, ctypes.byref(h)))
        self.handle = h.value
        self._children = weakref.WeakSet()  # batches and servers: closed before the context

    def adopt(self, child):
        """Registers an object whose close() must run before the context goes."""
        self._children.add(child)

    def close(self):
        if self.handle:
            for ch in list(self._children):
                ch.close()
            self._L.whirgpu_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    ORDER_NATURAL, ORDER_COSET_MAJOR = 0, 1

    def set_codeword_order(self, order: int):
        """Codeword row order of later commitments: ORDER_NATURAL (the C++
        reference) or ORDER_COSET_MAJOR (the Rust crate without rs_in_order)."""
        _lib.check(self._L.whirgpu_set_codeword_order(self.handle, int(order)), self.handle)

    @property
    def stream(self) -> int:
        return self._L.whirgpu_stream(self.handle) or 0

    def set_timing(self, on: bool):
        _lib.check(self._L.whirgpu_set_timing(self.handle, int(on)), self.handle)

    def kernel_stats(self, reset: bool = False):
        launches = (ctypes.c_uint64 * _lib.NUM_FAMILIES)()
        ms = (ctypes.c_double * _lib.NUM_FAMILIES)()
        _lib.check(self._L.whirgpu_kernel_stats(self.handle, launches, ms, int(reset)), self.handle)
        return {name: (int(launches[i]), float(ms[i])) for i, name in enumerate(_lib.FAMILY_NAMES)}

    def last_io_bytes(self):
        h2d, d2h = ctypes.c_uint64(), ctypes.c_uint64()
        self._L.whirgpu_last_io_bytes(self.handle, ctypes.byref(h2d), ctypes.byref(d2h))
        return int(h2d.value), int(d2h.value)

    @staticmethod
    def launch_count() -> int:
        return int(_lib.load().whirgpu_launch_count())

    def workspace_stats(self) -> dict:
        """Workspace cache: bytes held, workspaces allocated, idle ones evicted."""
        vals = [ctypes.c_uint64() for _ in range(3)]
        _lib.check(self._L.whirgpu_workspace_stats(self.handle, *[ctypes.byref(v) for v in vals]), self.handle)
        return {"cached_bytes": vals[0].value, "allocations": vals[1].value, "evictions": vals[2].value}

    def mle_evaluate(self, coeffs, point, on_device_ptr: Optional[int] = None):
        """MultilinearExtension::evaluate of base coefficients at an Ext3 point."""
        point = np.ascontiguousarray(point, dtype=np.uint64).reshape(-1)
        n = point.size // 3
        out = np.zeros(3, dtype=np.uint64)
        if on_device_ptr is not None:
            _lib.check(self._L.whirgpu_mle_evaluate(self.handle, on_device_ptr, n, 1, point.ctypes.data,
                                                     out.ctypes.data), self.handle)
        else:
            coeffs = np.ascontiguousarray(coeffs, dtype=np.uint64)
            assert coeffs.size == 1 << n
            _lib.check(self._L.whirgpu_mle_evaluate(self.handle, coeffs.ctypes.data, n, 0, point.ctypes.data,
                                                     out.ctypes.data), self.handle)
        return tuple(int(x) for x in out)


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class ProverState:
    """Fiat-Shamir prover state (transcript.hpp:595-662), device-resident."""

    def __init__(self, ds: DomainSeparator, instance: bytes = b"", ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self._L = self.ctx._L
        h = ctypes.c_void_p()
        _lib.check(self._L.whirgpu_transcript_create(self.ctx.handle, ds.protocol_id, ds.session_id, instance or None,
                                                     len(instance), ctypes.byref(h)), self.ctx.handle)
        self.handle = h.value

    @classmethod
    def from_ds(cls, ds: DomainSeparator, instance: bytes = b"", ctx: Optional[Context] = None) -> "ProverState":
        return cls(ds, instance, ctx)

    def proof(self):
        """(narg_string, hints) once prove() has completed."""
        narg, hints = ctypes.c_void_p(), ctypes.c_void_p()
        ln, lh = ctypes.c_size_t(), ctypes.c_size_t()
        _lib.check(self._L.whirgpu_proof_get(self.handle, ctypes.byref(narg), ctypes.byref(ln), ctypes.byref(hints),
                                             ctypes.byref(lh)), self.ctx.handle)
        return ctypes.string_at(narg, ln.value), ctypes.string_at(hints, lh.value)

    def __del__(self):
        try:
            if self.handle:
                self._L.whirgpu_transcript_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


@dataclass
class MultilinearExtension:
    """MultilinearExtension linear form (linear_form.hpp:97-138): point[0] is
    the most significant variable."""

    point: Sequence  # num_variables Ext3 triples


@dataclass
class Covector:
    """Covector linear form (linear_form.hpp:54-91): a dense vector of 2^n Ext3
    values (an (2^n, 3) uint64 array), or a device pointer to one with
    on_device=True."""

    vector: object
    on_device: bool = False


@dataclass
class FinalClaim:
    """FinalClaim (whir.hpp:376-425) as the prover returns it."""

    evaluation_point: list
    rlc_coefficients: list
    linear_form_rlc: tuple = (0, 0, 0)
    valid: bool = True


class Witness:
    """Committed matrix (or matrices) in HBM.  One handle may stand for several
    consecutive commitments (``Config.commit_witnesses``); ``num_vectors`` is
    the number of vectors they hold together."""

    def __init__(self, handle, ctx: Context, vector_ptr_keepalive=None, num_vectors: int = 1,
                 num_witnesses: int = 1):
        self.handle = handle
        self.ctx = ctx
        self._keep = vector_ptr_keepalive
        self.num_vectors = num_vectors
        self.num_witnesses = num_witnesses

    def __del__(self):
        try:
            if self.handle:
                # after Context.close() the library has detached the witness; this frees its handle only
                self.ctx._L.whirgpu_witness_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


FIELD_GOLDILOCKS1, FIELD_GOLDILOCKS2, FIELD_GOLDILOCKS3 = (_lib.FIELD_GOLDILOCKS1, _lib.FIELD_GOLDILOCKS2,
                                                            _lib.FIELD_GOLDILOCKS3)


@dataclass
class Config:
    """Config<M> (whir.hpp:104-343) with M = Basefield<GoldilocksExt3> (field 3,
    the CLI's Goldilocks3), Basefield<GoldilocksExt2> (field 2, Goldilocks2) or
    Identity<Goldilocks> (field 1, Goldilocks1).
    ``from_params`` derives it as the reference does; ``custom`` takes one built
    field by field (``_lib.WhirConfig``), as the reference's golden dumpers do."""

    size: int
    params: ProtocolParameters
    schedule: list = field(default_factory=list)
    target_field: int = FIELD_GOLDILOCKS3
    cconfig: Optional[object] = None  # whirgpu_config when committing through whirgpu_commit_config

    @classmethod
    def from_params(cls, size: int, params: ProtocolParameters, target_field: int = FIELD_GOLDILOCKS3) -> "Config":
        if size <= 0 or size & (size - 1):
            raise ValueError("size must be a power of two")
        n = size.bit_length() - 1
        L = _lib.load()
        out = (ctypes.c_uint64 * 1024)()
        c = params.to_c()
        cnt = L.whirgpu_schedule(ctypes.byref(c), n, out, 1024)
        if cnt == 0:
            raise ValueError("invalid protocol parameters")
        cconfig = None
        if target_field != FIELD_GOLDILOCKS3:
            cconfig = _lib.WhirConfig()
            _lib.check(L.whirgpu_config_from_params(ctypes.byref(c), n, target_field, ctypes.byref(cconfig)))
        return cls(size, params, list(out[:cnt]), target_field, cconfig)

    @classmethod
    def custom(cls, cconfig) -> "Config":
        """A Config given field by field as a ``_lib.WhirConfig``."""
        size = int(cconfig.initial_committer.vector_size)
        params = ProtocolParameters(batch_size=int(cconfig.batch_size), hash_id=bytes(cconfig.hash_id))
        return cls(size, params, [], int(cconfig.field), cconfig)

    def workspace_bytes(self) -> int:
        """Device memory one proof of this shape occupies (HBM-budget unit)."""
        c = self.params.to_c()
        return int(_lib.load().whirgpu_workspace_bytes(ctypes.byref(c), self.num_variables))

    @property
    def num_variables(self) -> int:
        return self.size.bit_length() - 1

    def n_rounds(self) -> int:
        return self.schedule[0]

    def commit(self, prover_state: ProverState, vectors, on_device_ptr: Optional[int] = None) -> Witness:
        """irs_commit::Config::commit of params.batch_size vectors (a 1-D array
        when batch_size is 1, else batch_size rows)."""
        return self.commit_witnesses(prover_state, vectors, 1, on_device_ptr)

    def commit_witnesses(self, prover_state: ProverState, vectors, num_witnesses: int,
                         on_device_ptr: Optional[int] = None) -> Witness:
        """num_witnesses commits in a row on one transcript; ``vectors`` holds
        num_witnesses * batch_size rows, witness 0's first."""
        ctx = prover_state.ctx
        c = self.params.to_c()
        h = ctypes.c_void_p()
        nvec = self.params.batch_size * num_witnesses
        if on_device_ptr is not None:
            ptr, where, keep = on_device_ptr, 1, None
        else:
            keep = np.ascontiguousarray(vectors, dtype=np.uint64)
            if keep.size != self.size * nvec:
                raise ValueError("vectors != batch_size * num_witnesses vectors of the config size")
            ptr, where = keep.ctypes.data, 0
        if self.cconfig is not None:
            _lib.check(ctx._L.whirgpu_commit_config(ctx.handle, ctypes.byref(self.cconfig), ptr, num_witnesses, where,
                                                    prover_state.handle, ctypes.byref(h)), ctx.handle)
        else:
            _lib.check(ctx._L.whirgpu_commit_witnesses(ctx.handle, ctypes.byref(c), ptr, num_witnesses,
                                                       self.num_variables, where, prover_state.handle,
                                                       ctypes.byref(h)), ctx.handle)
        return Witness(h.value, ctx, keep, nvec, num_witnesses)

    def prove(self, prover_state: ProverState, vectors, witnesses: Sequence[Witness], linear_forms: Sequence,
              evaluations: Sequence) -> FinalClaim:
        """Config::prove; ``evaluations`` holds len(linear_forms) * num_vectors
        Ext3 values, form-major (whir_prover.hpp:77)."""
        ctx = prover_state.ctx
        if len(witnesses) != 1:
            raise ValueError("pass the one handle of commit / commit_witnesses")
        nvec = witnesses[0].num_vectors
        n = self.num_variables
        cforms = (_lib.LinearForm * max(len(linear_forms), 1))()
        keep = []
        for i, lf in enumerate(linear_forms):
            if isinstance(lf, MultilinearExtension):
                a = np.ascontiguousarray(np.asarray(lf.point, dtype=np.uint64).reshape(n, 3))
                cforms[i] = _lib.LinearForm(_lib.FORM_MLE, 0, a.ctypes.data)
            elif isinstance(lf, Covector):
                if lf.on_device:
                    cforms[i] = _lib.LinearForm(_lib.FORM_COVECTOR, 1, int(lf.vector))
                    keep.append(lf)
                    continue
                a = np.ascontiguousarray(lf.vector, dtype=np.uint64)
                if a.size != 3 * self.size:
                    raise ValueError("covector length != config size")
                cforms[i] = _lib.LinearForm(_lib.FORM_COVECTOR, 0, a.ctypes.data)
            else:
                raise TypeError("MultilinearExtension and Covector statements are on this path")
            keep.append(a)
        if len(evaluations) != len(linear_forms) * nvec:
            raise ValueError("evaluations != linear forms * committed vectors")
        ev = np.zeros((max(len(evaluations), 1), 3), dtype=np.uint64)
        for i, e in enumerate(evaluations):
            ev[i] = np.asarray(e, dtype=np.uint64).reshape(3)
        eval_point = np.zeros((n, 3), dtype=np.uint64)
        rlc = np.zeros((max(len(linear_forms), 1), 3), dtype=np.uint64)
        _lib.check(ctx._L.whirgpu_prove_forms(ctx.handle, witnesses[0].handle, cforms, len(linear_forms),
                                              ev.ctypes.data, prover_state.handle, eval_point.ctypes.data,
                                              rlc.ctypes.data), ctx.handle)
        return FinalClaim([tuple(int(x) for x in r) for r in eval_point],
                          [tuple(int(x) for x in r) for r in rlc[:len(linear_forms)]])


def prove_once(n: int, params: ProtocolParameters, coeffs, points, evaluations, ctx: Optional[Context] = None,
               ds: Optional[DomainSeparator] = None, on_device_ptr: Optional[int] = None, num_witnesses: int = 1,
               forms: Optional[Sequence] = None, target_field: int = FIELD_GOLDILOCKS3,
               config: Optional[Config] = None):
    """commit (num_witnesses witnesses of params.batch_size vectors) + prove with
    the CLI domain separator; returns (narg, hints, claim).  The statement is
    one MultilinearExtension per point, or ``forms`` (MultilinearExtension /
    Covector objects) when given; ``evaluations`` holds num_forms * num_vectors
    Ext3 values, form-major.  ``config`` (a Config, e.g. Config.custom) replaces
    the one from_params derives; ``target_field`` selects the embedding."""
    ctx = ctx or default_context()
    ds = ds or cli_domain_separator(params)
    config = config or Config.from_params(1 << n, params, target_field)
    ps = ProverState.from_ds(ds, b"", ctx)
    w = config.commit_witnesses(ps, coeffs, num_witnesses, on_device_ptr=on_device_ptr)
    if forms is None:
        pts = np.asarray(points, dtype=np.uint64).reshape(-1, n, 3)
        forms = [MultilinearExtension(pts[i]) for i in range(pts.shape[0])]
    claim = config.prove(ps, coeffs, [w], forms, [tuple(e) for e in np.asarray(evaluations).reshape(-1, 3)])
    narg, hints = ps.proof()
    return narg, hints, claim


def sample_goldilocks(seed: int, count: int) -> np.ndarray:
    """Seeded uniform canonical Goldilocks words (ChaCha20 keystream, rejection of words >= p)."""
    out = np.empty(count, dtype=np.uint64)
    _lib.load().whirgpu_sample_goldilocks(seed, out.ctypes.data, count)
    return out
