"""Python mirror of the reference zero-knowledge WHIR prover over the C ABI.

Names and call order follow ``whir::protocols::whir_zk::ZkConfig<Goldilocks>``
(cpp/include/whir/protocols/whir_zk/whir_zk.hpp, whir_zk_impl.hpp):

    config = ZkConfig.from_params(1 << n, params, num_polynomials)   # whir_zk.hpp:95
    ps = ProverState.from_ds(cli_domain_separator(params))
    rng = DeterministicRng(seed, "WHIR_ZK:mask")                      # deterministic_rng.hpp
    witness = config.commit(ps, polynomials, rng)                     # whir_zk_impl.hpp:42
    config.prove(ps, polynomials, witness, forms, evaluations, rng)   # whir_zk_impl.hpp:150
    narg, hints = ps.proof()

Everything is over the base field (Identity<Goldilocks>): forms carry Ext3
triples (x, 0, 0), evaluations likewise.  The device work happens in
libwhirgpu.so.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib
from .whir import Context, Covector, DomainSeparator, FinalClaim, MultilinearExtension, ProtocolParameters, \
    ProverState, cli_domain_separator, default_context


@dataclass
class BlindingSizePolicy:
    """BlindingSizePolicy (whir_zk.hpp:45-63); None in from_params derives it."""

    q_delta_1: int
    q_delta_2: int
    t1: int
    t2: int
    sumcheck_round_degree: int = 3

    def to_c(self) -> _lib.ZkPolicy:
        return _lib.ZkPolicy(self.q_delta_1, self.q_delta_2, self.t1, self.t2, self.sumcheck_round_degree)


def whir_zk_domain_separator(vector_size: int, num_polynomials: int, params: ProtocolParameters,
                             policy: Optional[BlindingSizePolicy], session: str):
    """canonical_config::whir_zk_domain_separator (canonical_config.hpp:76-87):
    (config bytes, DomainSeparator); policy None: the derived one."""
    cb = ctypes.create_string_buffer(_lib.ZK_CONFIG_BYTES)
    out = ctypes.create_string_buffer(96)
    c = params.to_c()
    pol = ctypes.byref(policy.to_c()) if policy is not None else None
    s = session.encode()
    _lib.check(_lib.load().whirgpu_zk_domain_separator(ctypes.byref(c), vector_size, num_polynomials, pol, s, len(s),
                                                       cb, out))
    return cb.raw, DomainSeparator(out.raw[:64], out.raw[64:])


@dataclass
class DeterministicRng:
    """DeterministicRng(seed, domain) (deterministic_rng.hpp:16-98): a 32-byte
    seed and a domain string; the stream is computed on the device."""

    seed: bytes
    domain: str = "WHIR_ZK:mask"

    def __post_init__(self):
        if len(self.seed) != 32:
            raise ValueError("seed must be 32 bytes")

    def words(self, first_word: int, count: int, ctx: Optional[Context] = None) -> np.ndarray:
        """u64() values first_word .. first_word + count - 1 of a fresh generator."""
        ctx = ctx or default_context()
        out = np.zeros(max(count, 1), dtype=np.uint64)
        d = self.domain.encode()
        _lib.check(ctx._L.whirgpu_deterministic_rng(ctx.handle, self.seed, d, len(d), first_word, out.ctypes.data,
                                                    count), ctx.handle)
        return out[:count]


class ZkWitness:
    """ZkWitness (whir_zk.hpp:222-229) in HBM: f_hat commitments, blinding
    vectors and their commitment.  Proves once."""

    def __init__(self, handle, ctx: Context, num_polynomials: int):
        self.handle = handle
        self.ctx = ctx
        self.num_polynomials = num_polynomials

    def __del__(self):
        try:
            if self.handle:
                self.ctx._L.whirgpu_zk_witness_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class ZkConfig:
    """ZkConfig<Goldilocks> (whir_zk.hpp:83-224)."""

    def __init__(self, raw: _lib.ZkConfig):
        self.raw = raw

    @classmethod
    def from_params(cls, size: int, params: ProtocolParameters, num_polynomials: int,
                    policy: Optional[BlindingSizePolicy] = None) -> "ZkConfig":
        """from_params / from_params_with_policy (whir_zk.hpp:95-105, 270-289)."""
        if size <= 0 or size & (size - 1):
            raise ValueError("size must be a power of two")
        raw = _lib.ZkConfig()
        c = params.to_c()
        pol = ctypes.byref(policy.to_c()) if policy is not None else None
        _lib.check(_lib.load().whirgpu_zk_config_from_params(ctypes.byref(c), size.bit_length() - 1, num_polynomials,
                                                             pol, ctypes.byref(raw)))
        return cls(raw)

    def disable_pow(self) -> "ZkConfig":
        """Every PoW threshold of both inner configs off, as the reference's ZK
        dumper does (cpp/tests/dump_whir_zk.cpp): over the 64-bit field the
        derived PoW bits are far above what a prover can grind."""
        for cfg in (self.raw.blinded, self.raw.blinding):
            cfg.initial_sumcheck.pow_threshold = _lib.NO_POW
            cfg.initial_skip_pow = _lib.NO_POW
            for r in range(cfg.num_rounds):
                cfg.round_configs[r].pow_threshold = _lib.NO_POW
                cfg.round_configs[r].sumcheck.pow_threshold = _lib.NO_POW
            cfg.final_sumcheck.pow_threshold = _lib.NO_POW
            cfg.final_pow = _lib.NO_POW
        return self

    @property
    def num_polynomials(self) -> int:
        return int(self.raw.num_polynomials)

    @property
    def num_witness_variables(self) -> int:
        return int(self.raw.num_witness_variables)

    @property
    def num_blinding_variables(self) -> int:
        return int(self.raw.num_blinding_variables)

    @property
    def interleaving_depth(self) -> int:
        return int(self.raw.blinded.initial_committer.interleaving_depth)

    @property
    def blinded_in_domain_samples(self) -> int:
        return int(self.raw.blinded.initial_committer.in_domain_samples)

    @property
    def blinding_batch_size(self) -> int:
        return int(self.raw.blinding.batch_size)

    def commit(self, prover_state: ProverState, polynomials, rng: DeterministicRng,
               on_device_ptr: Optional[int] = None) -> ZkWitness:
        """ZkConfig::commit: num_polynomials rows of 2^n base-field coefficients."""
        ctx = prover_state.ctx
        if on_device_ptr is not None:
            ptr, where, keep = on_device_ptr, 1, None
        else:
            keep = np.ascontiguousarray(polynomials, dtype=np.uint64)
            if keep.size != self.num_polynomials << self.num_witness_variables:
                raise ValueError("polynomials != num_polynomials vectors of the config size")
            ptr, where = keep.ctypes.data, 0
        d = rng.domain.encode()
        h = ctypes.c_void_p()
        _lib.check(ctx._L.whirgpu_zk_commit(ctx.handle, ctypes.byref(self.raw), ptr, where, rng.seed, d, len(d),
                                            prover_state.handle, ctypes.byref(h)), ctx.handle)
        del keep
        return ZkWitness(h.value, ctx, self.num_polynomials)

    def prove(self, prover_state: ProverState, polynomials, witness: ZkWitness, linear_forms: Sequence,
              evaluations: Sequence, rng: Optional[DeterministicRng] = None):
        """ZkConfig::prove; ``evaluations`` holds len(linear_forms) * num_polynomials
        values (ints or Ext3 triples with zero high parts), form-major.  Returns
        the blinded inner proof's FinalClaim, as the reference does."""
        ctx = prover_state.ctx
        n = self.num_witness_variables
        cforms = (_lib.LinearForm * max(len(linear_forms), 1))()
        keep = []
        for i, lf in enumerate(linear_forms):
            if isinstance(lf, MultilinearExtension):
                a = np.ascontiguousarray(np.asarray(lf.point, dtype=np.uint64).reshape(n, 3))
                cforms[i] = _lib.LinearForm(_lib.FORM_MLE, 0, a.ctypes.data)
            elif isinstance(lf, Covector):
                if lf.on_device:
                    cforms[i] = _lib.LinearForm(_lib.FORM_COVECTOR, 1, int(lf.vector))
                    continue
                a = np.ascontiguousarray(lf.vector, dtype=np.uint64)
                if a.size != 3 << n:
                    raise ValueError("covector length != config size")
                cforms[i] = _lib.LinearForm(_lib.FORM_COVECTOR, 0, a.ctypes.data)
            else:
                raise TypeError("MultilinearExtension and Covector statements are on this path")
            keep.append(a)
        if len(evaluations) != len(linear_forms) * witness.num_polynomials:
            raise ValueError("evaluations != linear forms * polynomials")
        ev = np.zeros((max(len(evaluations), 1), 3), dtype=np.uint64)
        for i, e in enumerate(evaluations):
            ev[i] = np.asarray(e, dtype=np.uint64).reshape(-1)[:3] if np.ndim(e) else (int(e), 0, 0)
        point = np.zeros((n, 3), dtype=np.uint64)
        rlc = np.zeros((max(len(linear_forms), 1), 3), dtype=np.uint64)
        _lib.check(ctx._L.whirgpu_zk_prove(ctx.handle, witness.handle, cforms, len(linear_forms), ev.ctypes.data,
                                           prover_state.handle, point.ctypes.data, rlc.ctypes.data), ctx.handle)
        return FinalClaim([tuple(int(x) for x in r) for r in point],
                          [tuple(int(x) for x in r) for r in rlc[:len(linear_forms)]])


def prove_zk_once(n: int, params: ProtocolParameters, polynomials, forms: Sequence, evaluations: Sequence,
                  seed: bytes, ctx: Optional[Context] = None, policy: Optional[BlindingSizePolicy] = None,
                  rng_domain: str = "WHIR_ZK:mask", config: Optional[ZkConfig] = None,
                  ds: Optional[DomainSeparator] = None):
    """commit + prove; the domain separator defaults to the CLI one of params.
    Returns (narg, hints)."""
    ctx = ctx or default_context()
    polys = np.ascontiguousarray(polynomials, dtype=np.uint64).reshape(-1, 1 << n)
    config = config or ZkConfig.from_params(1 << n, params, polys.shape[0], policy)
    ps = ProverState.from_ds(ds or cli_domain_separator(params), b"", ctx)
    rng = DeterministicRng(seed, rng_domain)
    w = config.commit(ps, polys, rng)
    config.prove(ps, polys, w, forms, evaluations, rng)
    return ps.proof()
