"""ctypes binding of libwhirgpu.so (the C ABI in include/whirgpu.h).

The library is built in tree (``whirplonk_b200/libwhirgpu.so``) by
``__graft_entry__.build()``.  There is no CPU fallback: importing a prover
entry point without the library raises immediately.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libwhirgpu.so")

OK, E_INVALID, E_UNSUPPORTED, E_OOM, E_CUDA, E_DEVICE, E_TIMEOUT, E_TOO_LARGE = range(8)
STATUS_NAMES = {0: "OK", 1: "E_INVALID", 2: "E_UNSUPPORTED", 3: "E_OOM", 4: "E_CUDA", 5: "E_DEVICE", 6: "E_TIMEOUT",
                7: "E_TOO_LARGE"}
NOALLOC_MLE_MAX_VARS = 24
NUM_FAMILIES = 9
FAMILY_NAMES = ["ntt", "leaf_hash", "merkle", "ood", "sumcheck", "covector", "pow", "opening", "transcript"]

# Every symbol include/whirgpu.h declares.
EXPORTED = [
    "whirgpu_ctx_create", "whirgpu_ctx_destroy", "whirgpu_last_error", "whirgpu_stream", "whirgpu_set_codeword_order",
    "whirgpu_schedule",
    "whirgpu_workspace_bytes",
    "whirgpu_cli_domain_separator", "whirgpu_transcript_create", "whirgpu_transcript_destroy", "whirgpu_proof_get",
    "whirgpu_commit", "whirgpu_commit_witnesses", "whirgpu_config_from_params", "whirgpu_commit_config", "whirgpu_witness_destroy", "whirgpu_prove", "whirgpu_prove_forms", "whirgpu_mle_evaluate", "whirgpu_mle_evaluate_noalloc",
    "whirgpu_debug_field_ops", "whirgpu_sample_goldilocks", "whirgpu_chacha20_block", "whirgpu_host_alloc", "whirgpu_host_free",
    "whirgpu_set_timing", "whirgpu_kernel_stats", "whirgpu_launch_count", "whirgpu_last_io_bytes",
    "whirgpu_workspace_stats",
    "whirgpu_measure_int_peaks",
    "whirgpu_batch_create", "whirgpu_batch_run", "whirgpu_batch_proof", "whirgpu_batch_destroy",
    "whirgpu_server_create", "whirgpu_server_submit", "whirgpu_server_poll", "whirgpu_server_release",
    "whirgpu_server_stats", "whirgpu_server_destroy",
    "whirgpu_rs_encode", "whirgpu_rs_commit_batch",
    "whirgpu_ntt_autotune", "whirgpu_ntt_set_plan", "whirgpu_ntt_get_plan", "whirgpu_ntt_clear_plans",
    "whirgpu_ntt_list_plans", "whirgpu_ntt_load_plans", "whirgpu_ntt_save_plans", "whirgpu_ntt_load_default_plans",
    "whirgpu_zk_config_from_params", "whirgpu_zk_commit", "whirgpu_zk_prove", "whirgpu_zk_witness_destroy",
    "whirgpu_deterministic_rng", "whirgpu_zk_domain_separator",
]


class WhirParams(ctypes.Structure):
    """Mirror of whirgpu_params / whir::ProtocolParameters (same field order)."""

    _fields_ = [
        ("unique_decoding", ctypes.c_uint8),
        ("starting_log_inv_rate", ctypes.c_uint64),
        ("initial_folding_factor", ctypes.c_uint64),
        ("folding_factor", ctypes.c_uint64),
        ("security_level", ctypes.c_uint64),
        ("pow_bits", ctypes.c_uint64),
        ("batch_size", ctypes.c_uint64),
        ("hash_id", ctypes.c_uint8 * 32),
    ]


class Request(ctypes.Structure):
    """Mirror of whirgpu_request."""

    _fields_ = [
        ("num_variables", ctypes.c_uint64),
        ("params", WhirParams),
        ("coeffs", ctypes.c_void_p),
        ("coeffs_location", ctypes.c_int),
        ("points", ctypes.c_void_p),
        ("evaluations", ctypes.c_void_p),
        ("num_points", ctypes.c_uint64),
        ("protocol_id", ctypes.c_uint8 * 64),
        ("session_id", ctypes.c_uint8 * 32),
    ]


FORM_MLE, FORM_COVECTOR = 0, 1
FIELD_GOLDILOCKS1, FIELD_GOLDILOCKS2, FIELD_GOLDILOCKS3 = 1, 2, 3
MAX_ROUNDS = 24
NO_POW = (1 << 64) - 1
ZK_CONFIG_BYTES = 154


class IrsConfig(ctypes.Structure):
    """Mirror of whirgpu_irs_config (irs_commit::Config's shape fields)."""
    _fields_ = [("vector_size", ctypes.c_uint64), ("codeword_length", ctypes.c_uint64),
                ("interleaving_depth", ctypes.c_uint64), ("in_domain_samples", ctypes.c_uint64),
                ("out_domain_samples", ctypes.c_uint64)]


class SumcheckConfig(ctypes.Structure):
    _fields_ = [("num_rounds", ctypes.c_uint64), ("pow_threshold", ctypes.c_uint64)]


class RoundConfig(ctypes.Structure):
    _fields_ = [("irs_committer", IrsConfig), ("pow_threshold", ctypes.c_uint64), ("sumcheck", SumcheckConfig)]


class WhirConfig(ctypes.Structure):
    """Mirror of whirgpu_config (Config<M>, whir.hpp:104-116, plus the field M)."""
    _fields_ = [("field", ctypes.c_uint32), ("batch_size", ctypes.c_uint64), ("hash_id", ctypes.c_uint8 * 32),
                ("initial_committer", IrsConfig), ("initial_sumcheck", SumcheckConfig),
                ("initial_skip_pow", ctypes.c_uint64), ("num_rounds", ctypes.c_uint64),
                ("round_configs", RoundConfig * MAX_ROUNDS), ("final_sumcheck", SumcheckConfig),
                ("final_pow", ctypes.c_uint64)]


class ZkPolicy(ctypes.Structure):
    """Mirror of whirgpu_zk_policy (BlindingSizePolicy, whir_zk.hpp:45-63)."""
    _fields_ = [("q_delta_1", ctypes.c_uint64), ("q_delta_2", ctypes.c_uint64), ("t1", ctypes.c_uint64),
                ("t2", ctypes.c_uint64), ("sumcheck_round_degree", ctypes.c_uint64)]


class ZkConfig(ctypes.Structure):
    """Mirror of whirgpu_zk_config (ZkConfig<Goldilocks>, whir_zk.hpp:83-93)."""
    _fields_ = [("blinded", WhirConfig), ("blinding", WhirConfig), ("num_polynomials", ctypes.c_uint64),
                ("num_witness_variables", ctypes.c_uint64), ("num_blinding_variables", ctypes.c_uint64)]


class LinearForm(ctypes.Structure):
    """Mirror of whirgpu_linear_form."""
    _fields_ = [("kind", ctypes.c_uint32), ("location", ctypes.c_int), ("data", ctypes.c_void_p)]


class Result(ctypes.Structure):
    """Mirror of whirgpu_result."""

    _fields_ = [
        ("status", ctypes.c_int),
        ("narg", ctypes.c_void_p),
        ("narg_len", ctypes.c_size_t),
        ("hints", ctypes.c_void_p),
        ("hints_len", ctypes.c_size_t),
        ("queue_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
    ]


class NttPlan(ctypes.Structure):
    """Mirror of whirgpu_ntt_plan."""

    _fields_ = [
        ("log_n", ctypes.c_uint32),
        ("log_expansion", ctypes.c_uint32),
        ("npass", ctypes.c_uint32),
        ("log_radix", ctypes.c_uint32 * 3),
        ("log_cols", ctypes.c_uint32 * 3),
        ("min_blocks", ctypes.c_uint32),
        ("pipelined", ctypes.c_uint32),
    ]

    def as_dict(self):
        return {"log_n": self.log_n, "log_expansion": self.log_expansion, "npass": self.npass,
                "log_radix": list(self.log_radix), "log_cols": list(self.log_cols), "min_blocks": self.min_blocks,
                "pipelined": self.pipelined}


class WhirGpuError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load() -> ctypes.CDLL:
    """Loads libwhirgpu.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run __graft_entry__.build() (make -C whirplonk_b200/csrc)")
    L = ctypes.CDLL(LIB_PATH)
    p, sz, u64, i32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_int
    vp = ctypes.POINTER(ctypes.c_void_p)
    L.whirgpu_ctx_create.argtypes = [i32, u64, vp]
    L.whirgpu_ctx_destroy.argtypes = [p]
    L.whirgpu_last_error.argtypes = [p]
    L.whirgpu_last_error.restype = ctypes.c_char_p
    L.whirgpu_stream.argtypes = [p]
    L.whirgpu_stream.restype = p
    L.whirgpu_schedule.argtypes = [ctypes.POINTER(WhirParams), u64, p, sz]
    L.whirgpu_schedule.restype = sz
    L.whirgpu_workspace_bytes.argtypes = [ctypes.POINTER(WhirParams), u64]
    L.whirgpu_workspace_bytes.restype = u64
    L.whirgpu_cli_domain_separator.argtypes = [ctypes.POINTER(WhirParams), p]
    L.whirgpu_transcript_create.argtypes = [p, p, p, p, sz, vp]
    L.whirgpu_transcript_destroy.argtypes = [p]
    L.whirgpu_proof_get.argtypes = [p, vp, ctypes.POINTER(sz), vp, ctypes.POINTER(sz)]
    L.whirgpu_commit.argtypes = [p, ctypes.POINTER(WhirParams), p, u64, i32, p, vp]
    L.whirgpu_commit_witnesses.argtypes = [p, ctypes.POINTER(WhirParams), p, u64, u64, i32, p, vp]
    L.whirgpu_config_from_params.argtypes = [ctypes.POINTER(WhirParams), u64, ctypes.c_uint32, ctypes.POINTER(WhirConfig)]
    L.whirgpu_commit_config.argtypes = [p, ctypes.POINTER(WhirConfig), p, u64, i32, p, vp]
    L.whirgpu_witness_destroy.argtypes = [p]
    L.whirgpu_prove.argtypes = [p, p, p, sz, p, p, p, p]
    L.whirgpu_prove_forms.argtypes = [p, p, ctypes.POINTER(LinearForm), sz, p, p, p, p]
    L.whirgpu_mle_evaluate.argtypes = [p, p, u64, i32, p, p]
    L.whirgpu_mle_evaluate_noalloc.argtypes = [p, u64, p, p, p]
    L.whirgpu_debug_field_ops.argtypes = [p, p, p, u64, i32]
    L.whirgpu_sample_goldilocks.argtypes = [u64, p, sz]
    L.whirgpu_sample_goldilocks.restype = None
    L.whirgpu_chacha20_block.argtypes = [p, ctypes.c_uint32, p, p]
    L.whirgpu_chacha20_block.restype = None
    L.whirgpu_host_alloc.argtypes = [sz]
    L.whirgpu_host_alloc.restype = p
    L.whirgpu_host_free.argtypes = [p]
    L.whirgpu_set_timing.argtypes = [p, i32]
    L.whirgpu_kernel_stats.argtypes = [p, p, p, i32]
    L.whirgpu_set_codeword_order.argtypes = [p, ctypes.c_int]
    L.whirgpu_set_codeword_order.restype = ctypes.c_int
    L.whirgpu_measure_int_peaks.argtypes = [ctypes.c_int, p]
    L.whirgpu_measure_int_peaks.restype = ctypes.c_int
    L.whirgpu_workspace_stats.argtypes = [p, ctypes.POINTER(u64), ctypes.POINTER(u64), ctypes.POINTER(u64)]
    L.whirgpu_workspace_stats.restype = ctypes.c_int
    L.whirgpu_launch_count.argtypes = []
    L.whirgpu_launch_count.restype = u64
    L.whirgpu_last_io_bytes.argtypes = [p, ctypes.POINTER(u64), ctypes.POINTER(u64)]
    L.whirgpu_last_io_bytes.restype = None
    L.whirgpu_batch_create.argtypes = [p, ctypes.POINTER(Request), sz, i32, vp]
    L.whirgpu_batch_run.argtypes = [p]
    L.whirgpu_batch_proof.argtypes = [p, sz, vp, ctypes.POINTER(sz), vp, ctypes.POINTER(sz)]
    L.whirgpu_batch_destroy.argtypes = [p]
    L.whirgpu_batch_destroy.restype = None
    L.whirgpu_server_create.argtypes = [p, u64, ctypes.c_uint32, vp]
    L.whirgpu_server_submit.argtypes = [p, ctypes.POINTER(Request), ctypes.POINTER(u64)]
    L.whirgpu_server_poll.argtypes = [p, u64, ctypes.c_uint32, ctypes.POINTER(Result)]
    L.whirgpu_server_release.argtypes = [p, u64]
    L.whirgpu_server_release.restype = None
    L.whirgpu_server_stats.argtypes = [p, ctypes.POINTER(u64), ctypes.POINTER(u64), ctypes.POINTER(u64),
                                       ctypes.POINTER(u64)]
    L.whirgpu_server_stats.restype = None
    L.whirgpu_server_destroy.argtypes = [p]
    L.whirgpu_server_destroy.restype = None
    u32 = ctypes.c_uint32
    L.whirgpu_rs_encode.argtypes = [p, p, sz, u32, u32, u32, p, p]
    L.whirgpu_rs_commit_batch.argtypes = [p, p, i32, sz, u32, u32, u32, p]
    L.whirgpu_ntt_autotune.argtypes = [p, u32, u32, u32, u32, ctypes.POINTER(NttPlan),
                                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(u32)]
    L.whirgpu_ntt_set_plan.argtypes = [ctypes.POINTER(NttPlan)]
    L.whirgpu_ntt_get_plan.argtypes = [u32, u32, ctypes.POINTER(NttPlan)]
    L.whirgpu_ntt_clear_plans.argtypes = []
    L.whirgpu_ntt_clear_plans.restype = None
    L.whirgpu_ntt_list_plans.argtypes = [ctypes.POINTER(NttPlan), sz]
    L.whirgpu_ntt_list_plans.restype = sz
    L.whirgpu_ntt_load_plans.argtypes = [ctypes.c_char_p, ctypes.POINTER(sz)]
    L.whirgpu_ntt_save_plans.argtypes = [ctypes.c_char_p]
    L.whirgpu_ntt_load_default_plans.argtypes = []
    L.whirgpu_ntt_load_default_plans.restype = None
    L.whirgpu_zk_config_from_params.argtypes = [ctypes.POINTER(WhirParams), u64, u64, ctypes.POINTER(ZkPolicy),
                                                ctypes.POINTER(ZkConfig)]
    L.whirgpu_zk_commit.argtypes = [p, ctypes.POINTER(ZkConfig), p, i32, p, ctypes.c_char_p, sz, p, vp]
    L.whirgpu_zk_prove.argtypes = [p, p, ctypes.POINTER(LinearForm), sz, p, p, p, p]
    L.whirgpu_zk_witness_destroy.argtypes = [p]
    L.whirgpu_zk_witness_destroy.restype = None
    L.whirgpu_deterministic_rng.argtypes = [p, p, ctypes.c_char_p, sz, u64, p, sz]
    L.whirgpu_zk_domain_separator.argtypes = [ctypes.POINTER(WhirParams), u64, u64, ctypes.POINTER(ZkPolicy),
                                              ctypes.c_char_p, sz, p, p]
    for name in ("whirgpu_zk_config_from_params", "whirgpu_zk_commit", "whirgpu_zk_prove", "whirgpu_deterministic_rng",
                 "whirgpu_zk_domain_separator"):
        getattr(L, name).restype = i32
    for name in ("whirgpu_rs_encode", "whirgpu_rs_commit_batch", "whirgpu_ntt_autotune", "whirgpu_ntt_set_plan",
                 "whirgpu_ntt_get_plan", "whirgpu_ntt_load_plans", "whirgpu_ntt_save_plans"):
        getattr(L, name).restype = i32
    for name in ("whirgpu_ctx_create", "whirgpu_cli_domain_separator", "whirgpu_transcript_create",
                 "whirgpu_proof_get", "whirgpu_commit", "whirgpu_commit_witnesses", "whirgpu_config_from_params", "whirgpu_commit_config", "whirgpu_prove",
                 "whirgpu_prove_forms", "whirgpu_mle_evaluate",
                 "whirgpu_mle_evaluate_noalloc", "whirgpu_debug_field_ops", "whirgpu_batch_create",
                 "whirgpu_batch_run", "whirgpu_batch_proof", "whirgpu_server_create", "whirgpu_server_submit",
                 "whirgpu_server_poll",
                 "whirgpu_set_timing", "whirgpu_kernel_stats"):
        getattr(L, name).restype = i32
    _lib = L
    return L


def check(status: int, ctx=None):
    if status != OK:
        msg = ""
        if ctx:
            raw = load().whirgpu_last_error(ctx)
            msg = raw.decode() if raw else ""
        raise WhirGpuError(status, msg)
