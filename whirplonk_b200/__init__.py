"""B200-native WHIR prover (commit + prove over Goldilocks with an Ext3, Ext2
or base-field target, BLAKE3 or SHA-256 Merkle commitments, and the
zero-knowledge ZkConfig<Goldilocks> in ``whirplonk_b200.zk``) behind the
reference C++ prover API.

The prover itself is libwhirgpu.so (hand-written sm_100a CUDA kernels behind
the C ABI in include/whirgpu.h); this package is its Python mirror.
"""
from .whir import (  # noqa: F401
    ENGINE_ID_BLAKE3,
    ENGINE_ID_SHA2,
    FIELD_GOLDILOCKS1,
    FIELD_GOLDILOCKS2,
    FIELD_GOLDILOCKS3,
    P,
    Config,
    Context,
    Covector,
    DomainSeparator,
    FinalClaim,
    MultilinearExtension,
    ProtocolParameters,
    ProverState,
    cli_domain_separator,
    default_context,
    prove_once,
    sample_goldilocks,
)
