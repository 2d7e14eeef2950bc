#!/usr/bin/env python3
"""Benchmark of the B200 WHIR prover (one JSON line on rank 0).

Workloads (all: folding factor 4, 100-bit security, 20 PoW bits, BLAKE3,
Goldilocks with Ext3 challenges, one MLE statement at a seeded Ext3 point, the
reference CLI domain separator, coefficients uniform in [0, p) from a seeded
ChaCha20 keystream):

  whir_served_mixed_n12_24 (default): a seeded stream of prove requests with
      num_variables uniform on [12, 24] (the size log-uniform on 2^12..2^24,
      rounded) and log_inv_rate uniform on {1, 2, 3}, served by the
      continuous-batching server (HBM-budget admission, captured per-proof
      programs, overlapping proofs).  A step = 32 requests.
        value : served proofs/s at saturation, coefficients resident in HBM
        e2e   : the same through the public API from pinned host buffers
        p50/p99 : latency (submit -> result) under Poisson arrivals at 80% of
                  the saturated rate, beside the plain path's under the same
                  arrivals; plain = one proof at a time through the public
                  single-proof API on the same requests
  whir_batch64_n14_22: 64 proofs, num_variables uniform on {14..22},
      log_inv_rate on {1, 2, 3}, in one captured CUDA graph.  A step = one run
      of the batch.
  whir_prove_n24_rate4 / _n22_rate4 / _n18_rate2: one plain proof per step.
  whir_zk_prove_n22_rate4: one zero-knowledge proof (ZkConfig<Goldilocks>:
      commit with DeterministicRng masks + prove) per step, n = 22, rate 1/4,
      one polynomial, one MLE statement at a seeded base-field point; every
      PoW off in both inner configs (over the 64-bit field the derived PoW
      bits are 37-58, far above what any prover grinds; the reference's own ZK
      dumper disables them the same way).

  rs_commit_n22x4_exp4: the kernel-level commitment -- 4 vectors of 2^22 words,
      expansion 4, rows of 16 elements (RS encode + BLAKE3 leaves + Merkle
      root per vector, no transcript); beside it the reference's own CUDA
      side-car on the same vectors (roots compared, vs_reference_gpu).

Every batched or served proof is checked byte-for-byte against the plain
path's proof of the same request.  Multi-GPU: independent replicas (each rank
its own stream of requests, no collective on the data path), weak scaling.

--impl reference times the reference C++ CPU prover (oracle/_ref/ref_driver,
built from the reference sources) with all host threads on the same request
multiset as the GPU arm: every distinct (num_variables, rate) shape of the
timed stream is proved once and the rate is the multiset's count over the sum
of count x time.  It loads nothing from whirplonk_b200 (inputs come from the
numpy restatement of the sampler, oracle/chacha.py) and warms up on a proof
that is not in the stream.  For the kernel-level workload it times the
reference's CUDA side-car instead (oracle/_ref/ref_gpu_driver).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "proofs/s & p50/p99 latency, mixed 2^12–2^24 batched vs plain GPU; 2^24 prove ms"
FOLD, SEC, POW = 4, 100, 20
WORKLOADS = {
    "whir_served_mixed_n12_24": {"kind": "served", "n": (12, 24), "dist": "log-uniform", "rho": (1, 2, 3),
                                 "per_step": 32, "seed": 11},
    "whir_batch64_n14_22": {"kind": "batch", "n": (14, 22), "dist": "uniform", "rho": (1, 2, 3), "count": 64,
                            "seed": 7},
    "whir_prove_n24_rate4": {"kind": "single", "n": 24, "rho": 2},
    "whir_prove_n22_rate4": {"kind": "single", "n": 22, "rho": 2},
    "whir_prove_n18_rate2": {"kind": "single", "n": 18, "rho": 1},
    "whir_zk_prove_n22_rate4": {"kind": "zk", "n": 22, "rho": 2},
    "rs_commit_n22x4_exp4": {"kind": "kernel", "log_len": 22, "count": 4, "log_exp": 2, "log_depth": 4,
                             "seed": 2222},
}
ZK_SEED = bytes(range(1, 9)) + bytes(24)  # the reference driver takes 8 seed bytes (the rest zero)
DEFAULT_WORKLOAD = "whir_served_mixed_n12_24"
FALLBACK_HBM_GBS = 6650.0
# Families whose kernels saturate the integer-ALU pipe before HBM (ncu summaries
# in profiles/): their HBM fraction is low by nature.
ALU_BOUND = {"ntt": "integer ALU pipe (67-76 % busy in ncu; butterflies of Goldilocks arithmetic)",
             "leaf_hash": "integer ALU pipe (80-90 % busy in ncu; BLAKE3 compressions)",
             "merkle": "integer ALU pipe (BLAKE3 compressions)"}
DATA = "synthetic (seeded ChaCha20 coefficients, seeded Ext3 points)"
DTYPE = "u64 (Goldilocks; Ext3 challenges)"


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-i", str(self.device),
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# algorithmic bytes per proof, per kernel family (formulas of the design doc)
# ---------------------------------------------------------------------------
def algorithmic_bytes(schedule, n, k):
    nr = schedule[0]
    init_N = schedule[1]
    d = 1 << k
    commits = [(1 << n, init_N, 1)]  # (message words per component, codeword length, components)
    for r in range(nr):
        vsize, N = schedule[6 + 6 * r], schedule[7 + 6 * r]
        commits.append((vsize, N, 3))
    lde = sum(8 * c * (v + N * d) for v, N, c in commits)
    leaf = sum(8 * c * d * N + 32 * N for v, N, c in commits)
    merkle = sum(3 * 32 * N for v, N, c in commits)
    # sumcheck: every round reads a, b and writes the folded halves
    sumcheck = 0
    size = 1 << n
    first = True
    for rounds in [k] * (nr + 1) + [schedule[6 + 6 * nr + 1]]:
        for _ in range(rounds):
            a_read = (8 if first else 24) * size
            sumcheck += a_read + 24 * size + 2 * 24 * (size // 2)
            first = False
            size //= 2
    return {"ntt": lde, "leaf_hash": leaf, "merkle": merkle, "sumcheck": sumcheck}


def algorithmic_units(schedule, n, k):
    """Per-proof operation counts of the integer-bound families: radix-2
    butterflies of the LDEs ((N/2) log2(m) per plane, the zero padding skipped),
    BLAKE3 compressions of the leaves (N ceil(row bytes / 64)) and of the Merkle
    trees (N - 1)."""
    nr = schedule[0]
    d = 1 << k
    commits = [(1 << n, schedule[1], 1)]
    for r in range(nr):
        commits.append((schedule[6 + 6 * r], schedule[7 + 6 * r], 3))
    bfly = leaf = merkle = 0
    for v, N, c in commits:
        m = max(v // d, 1)
        bfly += c * d * (N // 2) * int(math.log2(m))
        leaf += N * -(-(8 * c * d) // 64)
        merkle += N - 1
    return {"ntt": bfly, "leaf_hash": leaf, "merkle": merkle}


def measure_int_peaks(device):
    """whirgpu_measure_int_peaks: register-only rates of this GPU's integer pipes."""
    from whirplonk_b200 import _lib

    L = _lib.load()
    out = (ctypes.c_double * 8)()
    if L.whirgpu_measure_int_peaks(device, out) != 0:
        return None
    names = ["butterflies_per_s", "blake3_compressions_per_s", "mac64_per_s", "mad_lo_u32_per_s",
             "mad_wide_u32_per_s", "add3_u32_per_s", "lop3_per_s", "shf_per_s"]
    return dict(zip(names, list(out)))


def read_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def read_traffic(family, alg_bytes_per_proof):
    """DRAM bytes per proof of `family`: the measured traffic / algorithmic-bytes
    ratio of profiles/dram_traffic.json (one ncu-captured proof) times this
    workload's algorithmic bytes; None when the family was not captured."""
    path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        with open(path) as f:
            t = json.load(f)
        ratio = t["families"][family]["ratio"]
    except (OSError, ValueError, KeyError):
        return None
    return alg_bytes_per_proof * ratio


# ---------------------------------------------------------------------------
# workload: requests and their inputs
# ---------------------------------------------------------------------------
def draw_requests(w, count, seed, sampler):
    """(num_variables, log_inv_rate) pairs drawn from the seeded ChaCha20 stream
    (`sampler`: the library's whirgpu_sample_goldilocks on the GPU arm, its
    numpy restatement on the reference arm; both give the same words)."""
    words = sampler(seed, 2 * count)
    lo, hi = w["n"]
    out = []
    for i in range(count):
        a, b = int(words[2 * i]), int(words[2 * i + 1])
        if w["dist"] == "uniform":
            n = lo + a % (hi - lo + 1)
        else:  # size log-uniform on [2^lo, 2^hi]: n uniform on [lo, hi], rounded
            n = int(math.floor(lo + (hi - lo) * ((a >> 11) / float(1 << 53)) + 0.5))
        out.append((n, w["rho"][b % len(w["rho"])]))
    return out


def make_inputs(n, seed, sampler):
    coeffs = sampler(seed, 1 << n)
    point = sampler(seed + 7919, 3 * n).reshape(1, n, 3)
    return coeffs, point


def coeff_seed(rank, n):
    return 1000 * (rank + 1) + n


def point_seed(rank, n, rho):
    return 5000 * (rank + 1) + 31 * n + rho


def gpu_sampler(seed, count):
    from whirplonk_b200 import sample_goldilocks

    return sample_goldilocks(seed, count)


def params_for(rho):
    from whirplonk_b200 import ProtocolParameters

    return ProtocolParameters.cli(security_level=SEC, pow_bits=POW, folding_factor=FOLD, log_inv_rate=rho)


class Inputs:
    """One coefficient vector per num_variables (host, pinned host and device
    copies) and one statement per (num_variables, rate)."""

    def __init__(self, ctx, shapes, rank, device):
        import torch

        self.ctx, self.rank, self.device = ctx, rank, device
        self.host, self.pinned, self.dev, self.pts, self.evs = {}, {}, {}, {}, {}
        self._pinned_ptrs = []
        for n in sorted({n for n, _ in shapes}):
            coeffs, _ = make_inputs(n, coeff_seed(rank, n), gpu_sampler)
            self.host[n] = coeffs
            self.dev[n] = torch.from_numpy(coeffs.view(np.int64)).to(device)
            ptr = ctx._L.whirgpu_host_alloc(coeffs.nbytes)
            if not ptr:
                raise MemoryError("pinned allocation failed")
            self._pinned_ptrs.append(ptr)
            view = np.ctypeslib.as_array((ctypes.c_uint64 * coeffs.size).from_address(ptr))
            view[:] = coeffs
            self.pinned[n] = view
        for n, rho in sorted(set(shapes)):
            _, point = make_inputs(n, point_seed(rank, n, rho), gpu_sampler)
            self.pts[(n, rho)] = point
            self.evs[(n, rho)] = np.array(ctx.mle_evaluate(self.host[n], point), dtype=np.uint64).reshape(1, 3)
        torch.cuda.synchronize()

    def extend(self, shapes):
        """Adds the inputs of shapes not seen yet (same seeds as the constructor)."""
        import torch

        ctx, rank = self.ctx, self.rank
        for n in sorted({n for n, _ in shapes} - set(self.host)):
            coeffs, _ = make_inputs(n, coeff_seed(rank, n), gpu_sampler)
            self.host[n] = coeffs
            self.dev[n] = torch.from_numpy(coeffs.view(np.int64)).to(self.device)
            ptr = ctx._L.whirgpu_host_alloc(coeffs.nbytes)
            if not ptr:
                raise MemoryError("pinned allocation failed")
            self._pinned_ptrs.append(ptr)
            view = np.ctypeslib.as_array((ctypes.c_uint64 * coeffs.size).from_address(ptr))
            view[:] = coeffs
            self.pinned[n] = view
        for n, rho in sorted(set(shapes) - set(self.pts)):
            _, point = make_inputs(n, point_seed(rank, n, rho), gpu_sampler)
            self.pts[(n, rho)] = point
            self.evs[(n, rho)] = np.array(ctx.mle_evaluate(self.host[n], point), dtype=np.uint64).reshape(1, 3)
        torch.cuda.synchronize()

    def request(self, n, rho, where):
        from whirplonk_b200.batch import ProofRequest

        if where == "device":
            return ProofRequest(n, params_for(rho), self.dev[n].data_ptr(), self.pts[(n, rho)], self.evs[(n, rho)],
                                on_device=True)
        return ProofRequest(n, params_for(rho), self.pinned[n], self.pts[(n, rho)], self.evs[(n, rho)])

    def coeff_bytes(self, n):
        return 8 << n

    def close(self):
        for p in self._pinned_ptrs:
            self.ctx._L.whirgpu_host_free(p)
        self._pinned_ptrs = []
        self.dev.clear()


# ---------------------------------------------------------------------------
# reference CPU prover
# ---------------------------------------------------------------------------
def reference_proof_seconds(n, rho, coeffs, point, threads):
    """Commit + prove of one request by the reference C++ prover, on its own clock."""
    from oracle.refio import run_reference

    r = run_reference(n, FOLD, rho, SEC, POW, point, coeffs, threads=threads)
    return (r.commit_ms + r.prove_ms) / 1000.0


def workload_shapes(w, count_steps, sampler):
    if w["kind"] in ("single", "zk"):
        return [(w["n"], w["rho"])] * count_steps
    if w["kind"] == "batch":
        return draw_requests(w, w["count"], w["seed"], sampler)
    return draw_requests(w, w["per_step"] * count_steps, w["seed"], sampler)


def reference_multiset(shapes, steps, threads, inputs_of):
    """The reference prover's rate on the multiset `shapes`: every distinct
    (num_variables, rate) shape is proved once (the distinct shapes are spread
    over `steps` steps, largest first), and the rate is
    len(shapes) / sum over shapes of count(shape) * time(shape).
    inputs_of(n, rho) -> (coefficients, point) of the same request."""
    from collections import Counter

    counts = Counter(shapes)
    distinct = sorted(counts, key=lambda s: (-s[0], -s[1]))
    per_shape, step_s = {}, []
    for i in range(steps):
        t = 0.0
        for n, rho in distinct[i::steps]:
            coeffs, point = inputs_of(n, rho)
            per_shape[(n, rho)] = reference_proof_seconds(n, rho, coeffs, point, threads)
            t += per_shape[(n, rho)]
        step_s.append(t)
    weighted = sum(counts[s] * per_shape[s] for s in counts)
    return {"value": len(shapes) / weighted, "distinct": len(distinct), "count": len(shapes),
            "measured_s": sum(step_s), "step_s": step_s, "weighted_s": weighted,
            "per_shape_s": {f"{n},{rho}": round(t, 4) for (n, rho), t in sorted(per_shape.items())}}


def multiset_sample_text(m):
    return (f"same multiset as the GPU arm: the {m['count']} requests of the timed steps, {m['distinct']} distinct "
            f"(num_variables, rate) shapes, each proved once by the reference C++ prover (oracle/_ref, commit+prove "
            f"on its own clock, {m['measured_s']:.1f} s); value = {m['count']} / sum of count(shape) x time(shape) "
            f"= {m['count']} / {m['weighted_s']:.1f} s")


def config_of(name, w):
    cfg = {"workload": name, "folding_factor": FOLD, "security_level": SEC, "pow_bits": POW, "hash": "BLAKE3",
           "field": "Goldilocks3", "statement": "1 MLE evaluation at a seeded Ext3 point"}
    if w["kind"] == "zk":
        cfg.update(num_variables=w["n"], log_inv_rate=w["rho"], field="Identity<Goldilocks> (ZkConfig<Goldilocks>)",
                   statement="1 MLE evaluation at a seeded base-field point", num_polynomials=1,
                   pow_bits="disabled in both inner configs (as the reference's ZK dumper)",
                   masks="DeterministicRng(seed 01..08 then zeros, \"WHIR_ZK:mask\")")
    elif w["kind"] == "single":
        cfg.update(num_variables=w["n"], log_inv_rate=w["rho"])
    else:
        cfg.update(num_variables=f"{w['dist']} on [{w['n'][0]}, {w['n'][1]}]", log_inv_rate=list(w["rho"]),
                   seed=w["seed"])
        cfg.update(requests_per_step=w["per_step"] if w["kind"] == "served" else w["count"])
    cfg["l2"] = "working set of a step (GBs of codewords and trees) far above the 126 MB L2; no flush"
    return cfg


def zk_inputs(n, sampler):
    """Coefficients and a base-field MLE point (Ext3 layout, zero high parts)."""
    coeffs = sampler(1000 + n, 1 << n)
    point = np.zeros((n, 3), dtype=np.uint64)
    point[:, 0] = sampler(9000 + n, n)
    return coeffs, point


def zk_reference(n, rho, coeffs, point, threads):
    from oracle.refio import run_reference_zk

    return run_reference_zk(n, FOLD, rho, SEC, POW, [("mle", point[:, 0])], coeffs.reshape(1, -1),
                            int.from_bytes(ZK_SEED[:8], "little"), no_pow=True, verify=False, threads=threads)


WARMUP_SHAPE = (12, 1)  # the reference arm's warm-up proof: never a request of the timed stream
WARMUP_SEED = 424242


def kernel_vectors(w, sampler):
    return sampler(w["seed"], w["count"] << w["log_len"]).reshape(w["count"], -1)


def reference_gpu_commit(w, vectors, reps=3):
    """The reference's CUDA side-car (oracle/_ref/ref_gpu_driver: its NTT engine's
    GPU RS encode + BLAKE3 leaves, then its GPU Merkle tree, host buffers in and
    out) on the same vectors: (roots, ms per pass over the vectors), or None."""
    import struct
    import tempfile

    exe = os.path.join(ROOT, "oracle", "_ref", "ref_gpu_driver")
    if not os.access(exe, os.X_OK):
        return None
    with tempfile.TemporaryDirectory() as td:
        inp, out = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(inp, "wb") as f:
            f.write(struct.pack("<II5Q", 0x47505552, 1, w["count"], w["log_len"], w["log_exp"], w["log_depth"], reps))
            f.write(np.ascontiguousarray(vectors, dtype=np.uint64).tobytes())
        subprocess.run([exe, inp, out], check=True, timeout=600, stdout=subprocess.DEVNULL)
        with open(out, "rb") as f:
            b = f.read()
    roots = [b[32 * k:32 * k + 32] for k in range(w["count"])]
    (ms,) = struct.unpack_from("<d", b, 32 * w["count"])
    return roots, ms


def run_reference_kernel_arm(args, w, world):
    """Kernel-level commitment: the reference's own GPU path (its CUDA
    side-car, host buffers in and out), the same vectors as the GPU arm."""
    from oracle.chacha import sample_goldilocks as np_sampler

    vectors = kernel_vectors(w, np_sampler)
    r = reference_gpu_commit(w, vectors, reps=max(3, args.steps))
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_gpu_driver not built"}))
        return 0
    _, ms = r
    value = w["count"] / (ms / 1000.0)
    print(json.dumps({
        "impl": "reference", "metric": KERNEL_METRIC, "value": value, "unit": "commitments/s", "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 (Goldilocks)", "data": DATA,
        "config": kernel_config(args.workload, w), "parallelism": "the reference's CUDA side-car on 1 GPU",
        "e2e": {"value": value, "unit": "commitments/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu_note": "NttEngine::try_gpu_interleaved_rs_encode_blake3_matrix_leaves + gpu_blake3_merkle_tree "
                              "per vector, host in / host out (its API returns the codeword matrix to the host); "
                              "median of the timed passes after a warm-up pass",
    }))
    return 0


def run_reference_arm(args, rank, world):
    """The reference C++ CPU prover on the GPU arm's workload.  Loads nothing
    from whirplonk_b200: inputs come from the numpy restatement of the sampler
    (oracle/chacha.py), which draws the same words."""
    from oracle.chacha import sample_goldilocks as np_sampler
    from oracle.refio import ref_available

    if rank != 0:
        return 0
    w = WORKLOADS[args.workload]
    if w["kind"] == "zk":
        return run_reference_zk_arm(args, w, world)
    if w["kind"] == "kernel":
        return run_reference_kernel_arm(args, w, world)
    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_driver not built"}))
        return 0
    threads = os.cpu_count() or 1
    warm = max(args.warmup, 3)
    wn, wr = WARMUP_SHAPE
    wc, wp = make_inputs(wn, WARMUP_SEED, np_sampler)
    for _ in range(warm):
        reference_proof_seconds(wn, wr, wc, wp, threads)
    shapes = workload_shapes(w, args.steps, np_sampler)
    cache = {}

    def inputs_of(n, rho):
        if n not in cache:
            cache.clear()  # shapes arrive largest n first: keep one coefficient vector
            cache[n] = make_inputs(n, coeff_seed(0, n), np_sampler)[0]
        return cache[n], make_inputs(n, point_seed(0, n, rho), np_sampler)[1]

    m = reference_multiset(shapes, args.steps, threads, inputs_of)
    value = m["value"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "proofs/s", "n_gpus": world,
        "steps": args.steps, "warmup": warm, "ms_per_step": 1000.0 * m["measured_s"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": DTYPE, "data": DATA,
        "config": config_of(args.workload, w), "parallelism": f"host OpenMP, {threads} threads (reference C++ prover)",
        "ms_per_step_note": "measured reference CPU time per step (the distinct shapes spread over the steps); "
                            "value is the rate over the whole multiset, see cpu_baseline.sample",
        "reference_seconds_per_shape": m["per_shape_s"],
        "cpu_baseline": {"value": value, "unit": "proofs/s", "cores": threads, "kind": "reference",
                         "sample": multiset_sample_text(m)},
        "e2e": {"value": value, "unit": "proofs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_reference_zk_arm(args, w, world):
    from oracle.refio import REF_ZK_DRIVER

    if not os.path.exists(REF_ZK_DRIVER):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_zk_driver not built"}))
        return 0
    from oracle.chacha import sample_goldilocks as np_sampler

    threads = os.cpu_count() or 1
    n, rho = w["n"], w["rho"]
    coeffs, point = zk_inputs(n, np_sampler)
    warm = max(args.warmup, 3)
    times = [zk_reference(n, rho, coeffs, point, threads).prove_ms / 1000.0 for _ in range(warm + args.steps)]
    timed = times[warm:]
    total = sum(timed)
    value = len(timed) / total
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": "proofs/s", "n_gpus": world,
        "steps": args.steps, "warmup": warm, "ms_per_step": 1000.0 * total / len(timed), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 (Goldilocks)", "data": DATA,
        "config": config_of(args.workload, w), "parallelism": f"host OpenMP, {threads} threads (reference C++ ZK prover)",
        "p50_ms": 1000.0 * statistics.median(timed), "p99_ms": 1000.0 * max(timed),
        "cpu_baseline": {"value": value, "unit": "proofs/s", "cores": threads, "kind": "reference",
                         "sample": f"{len(timed)} zero-knowledge proofs (commit+prove, driver clock)"},
        "e2e": {"value": value, "unit": "proofs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
class Harness:
    """One rank: process group (NCCL on GPUs; gloo on the host, for the
    multi-process tests without a GPU), barriers, max / sum over ranks."""

    def __init__(self, rank, world, local_rank, backend=None):
        import torch

        self.torch = torch
        self.dist = None
        self.cuda = backend != "gloo"
        if world > 1:
            import datetime

            import torch.distributed as dist

            dist.init_process_group(backend or "nccl", timeout=datetime.timedelta(seconds=120))
            self.dist = dist
        if self.cuda:
            torch.cuda.set_device(local_rank)
        self.device = f"cuda:{local_rank}" if self.cuda else "cpu"
        self.rank, self.world, self.local_rank = rank, world, local_rank

    def barrier(self):
        if self.cuda:
            self.torch.cuda.synchronize()
        if self.dist is not None:
            self.dist.barrier()
        if self.cuda:
            self.torch.cuda.synchronize()

    def max_over_ranks(self, x):
        if self.dist is None:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(self, x):
        if self.dist is None:
            return x
        t = self.torch.tensor([x], dtype=self.torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def timed(self, stream, fn):
        """Device time (ms) of fn() between two events on `stream`, with the
        device synchronised on both sides (work on other streams included)."""
        torch = self.torch
        self.barrier()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        out = fn()
        torch.cuda.synchronize()
        b.record(stream)
        b.synchronize()
        self.barrier()
        return self.max_over_ranks(a.elapsed_time(b)), out

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()


def plain_prove(ctx, inputs, n, rho, where="device"):
    from whirplonk_b200 import prove_once

    if where == "device":
        narg, hints, _ = prove_once(n, params_for(rho), None, inputs.pts[(n, rho)], inputs.evs[(n, rho)], ctx=ctx,
                                    on_device_ptr=inputs.dev[n].data_ptr())
    else:
        narg, hints, _ = prove_once(n, params_for(rho), inputs.pinned[n], inputs.pts[(n, rho)],
                                    inputs.evs[(n, rho)], ctx=ctx)
    return narg, hints


def family_roofline(ctx, inputs, shapes):
    """Per-family device time over one plain pass of `shapes` (events on the
    launching stream) against the algorithmic bytes of the same proofs."""
    from whirplonk_b200.whir import Config

    ctx.set_timing(True)
    ctx.kernel_stats(reset=True)
    alg = {}
    for n, rho in shapes:
        plain_prove(ctx, inputs, n, rho)
        sched = Config.from_params(1 << n, params_for(rho)).schedule
        for f, v in algorithmic_bytes(sched, n, FOLD).items():
            alg[f] = alg.get(f, 0) + v
    fam = ctx.kernel_stats(reset=True)
    ctx.set_timing(False)
    fam_ms = {f: v[1] for f, v in fam.items()}
    units = {}
    for n, rho in shapes:
        sched = Config.from_params(1 << n, params_for(rho)).schedule
        for f, v in algorithmic_units(sched, n, FOLD).items():
            units[f] = units.get(f, 0) + v
    dominant = max(alg.keys(), key=lambda f: fam_ms.get(f, 0.0))
    peak, peak_kind = read_peaks()
    achieved = alg[dominant] / (fam_ms[dominant] / 1000.0) / 1e9
    per = len(shapes)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": read_traffic(dominant, alg[dominant] / per), "kernel": dominant, "peak_source": peak_kind,
            "algorithmic_bytes_per_proof": alg[dominant] / per, "ms_per_proof": fam_ms[dominant] / per,
            "traffic_unit": "DRAM bytes per proof of the family",
            "binding_limit": ALU_BOUND.get(dominant, "HBM")}
    sc_ms = fam_ms.get("sumcheck", 0.0) + fam_ms.get("covector", 0.0)
    sc_ach = alg["sumcheck"] / (sc_ms / 1000.0) / 1e9 if sc_ms > 0 else None
    roof_sc = {"bound": "hbm", "kernel": "sumcheck + covector", "achieved": sc_ach, "peak": peak, "unit": "GB/s",
               "frac": sc_ach / peak if sc_ach else None, "peak_source": peak_kind,
               "algorithmic_bytes_per_proof": alg["sumcheck"] / per, "ms_per_proof": sc_ms / per,
               "traffic": read_traffic("sumcheck", alg["sumcheck"] / per),
               "bytes_note": "per round on size s: (8 or 24) s + 24 s read, 2 x 24 s/2 written (a and the covector)"}
    extra = {"roofline_sumcheck": roof_sc}
    pk = measure_int_peaks(ctx.device)
    if pk:
        ri = {}
        for f, unit, pkey in (("ntt", "butterflies/s", "butterflies_per_s"),
                              ("leaf_hash", "BLAKE3 compressions/s", "blake3_compressions_per_s"),
                              ("merkle", "BLAKE3 compressions/s", "blake3_compressions_per_s")):
            if fam_ms.get(f, 0.0) > 0:
                a = units[f] / (fam_ms[f] / 1000.0)
                ri[f] = {"achieved": a, "peak": pk[pkey], "unit": unit, "frac": a / pk[pkey],
                         "units_per_proof": units[f] / per, "ms_per_proof": fam_ms[f] / per}
        extra["roofline_int"] = ri
        extra["int_peaks_measured"] = pk
    return roof, {f: round(v / per, 4) for f, v in fam_ms.items()}, extra


def cpu_sample(shapes, steps, inputs):
    """The reference prover on the multiset of requests the GPU arm timed
    (every distinct shape proved once; reference_multiset), on the same inputs."""
    from oracle.refio import ref_available

    if not ref_available():
        return None
    threads = os.cpu_count() or 1
    m = reference_multiset(shapes, steps, threads, lambda n, rho: (inputs.host[n], inputs.pts[(n, rho)]))
    return {"value": m["value"], "unit": "proofs/s", "cores": threads, "kind": "reference",
            "sample": multiset_sample_text(m)}


def pct(xs, q):
    xs = sorted(xs)
    return xs[min(len(xs) - 1, int(q * len(xs)))] if xs else None


def run_single(args, H, ctx, w):
    torch = H.torch
    n, rho = w["n"], w["rho"]
    inputs = Inputs(ctx, [(n, rho)], H.rank, H.device)
    stream = torch.cuda.ExternalStream(ctx.stream, device=H.device)
    ref_proof = plain_prove(ctx, inputs, n, rho)
    for _ in range(max(args.warmup, 3) - 1):
        plain_prove(ctx, inputs, n, rho)
    for _ in range(2):
        assert plain_prove(ctx, inputs, n, rho, "host") == ref_proof, "host and device inputs differ"

    clocks = ClockSampler(H.local_rank)
    clocks.start()
    time.sleep(0.3)
    launches0 = ctx.launch_count()
    lat = []

    def device_steps():
        out = None
        for _ in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            out = plain_prove(ctx, inputs, n, rho)
            b.record(stream)
            lat.append((a, b))
        return out

    elapsed, out = H.timed(stream, device_steps)
    launches = ctx.launch_count() - launches0
    assert out == ref_proof
    lat = sorted(a.elapsed_time(b) for a, b in lat)

    def host_steps():
        o = None
        for _ in range(args.steps):
            o = plain_prove(ctx, inputs, n, rho, "host")
        return o

    e2e_ms, out = H.timed(stream, host_steps)
    h2d, d2h = ctx.last_io_bytes()
    clk = clocks.stop()
    assert out == ref_proof
    roof, fams, extra = family_roofline(ctx, inputs, [(n, rho)] * args.steps)
    total = args.steps * H.world
    line = {
        "value": total / (elapsed / 1000.0), "ms_per_step": elapsed / args.steps,
        "prove_ms": elapsed / args.steps, "p50_ms": pct(lat, 0.5), "p99_ms": pct(lat, 0.99),
        "e2e": {"value": total / (e2e_ms / 1000.0), "unit": "proofs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches, "roofline": roof, "families_ms_per_proof": fams, "clocks": clk,
    }
    line.update(extra)
    if H.world == 1 and H.rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample([(n, rho)] * args.steps, 1, inputs)
    inputs.close()
    return line


def zk_algorithmic_bytes(cfg):
    """Per-family algorithmic bytes of one ZK proof: the two inner
    Config<Identity<Goldilocks>> proofs with 8-byte elements (the formulas of
    algorithmic_bytes, base field throughout)."""
    out = {"ntt": 0, "leaf_hash": 0, "merkle": 0, "sumcheck": 0}
    for inner, nvec in ((cfg.raw.blinded, cfg.num_polynomials), (cfg.raw.blinding, int(cfg.raw.blinding.batch_size))):
        ic = inner.initial_committer
        commits = [(int(ic.vector_size) * nvec, int(ic.codeword_length), int(ic.interleaving_depth) * nvec)]
        for r in range(inner.num_rounds):
            rc = inner.round_configs[r].irs_committer
            commits.append((int(rc.vector_size), int(rc.codeword_length), int(rc.interleaving_depth)))
        out["ntt"] += sum(8 * (v + N * d) for v, N, d in commits)
        out["leaf_hash"] += sum(8 * d * N + 32 * N for v, N, d in commits)
        out["merkle"] += sum(3 * 32 * N for v, N, d in commits)
        size = int(ic.vector_size)
        rounds = [int(inner.initial_sumcheck.num_rounds)] + \
                 [int(inner.round_configs[r].sumcheck.num_rounds) for r in range(inner.num_rounds)] + \
                 [int(inner.final_sumcheck.num_rounds)]
        for k in rounds:  # read a and b, write both folded halves (a: the combined vector)
            for _ in range(k):
                out["sumcheck"] += 8 * size + 8 * size + 2 * 8 * (size // 2)
                size //= 2
    return out


def run_zk(args, H, ctx, w):
    import hashlib

    from whirplonk_b200 import MultilinearExtension, ProverState, cli_domain_separator
    from whirplonk_b200.zk import DeterministicRng, ZkConfig

    torch = H.torch
    n, rho = w["n"], w["rho"]
    params = params_for(rho)
    cfg = ZkConfig.from_params(1 << n, params, 1).disable_pow()
    coeffs, point = zk_inputs(n, gpu_sampler)
    ev = ctx.mle_evaluate(coeffs, point)
    dev = torch.from_numpy(coeffs.view(np.int64)).to(H.device)
    ptr = ctx._L.whirgpu_host_alloc(coeffs.nbytes)
    pinned = np.ctypeslib.as_array((ctypes.c_uint64 * coeffs.size).from_address(ptr))
    pinned[:] = coeffs
    ds = cli_domain_separator(params)
    forms = [MultilinearExtension(point)]
    stream = torch.cuda.ExternalStream(ctx.stream, device=H.device)

    def one(where):
        ps = ProverState.from_ds(ds, b"", ctx)
        rng = DeterministicRng(ZK_SEED)
        if where == "device":
            wit = cfg.commit(ps, None, rng, on_device_ptr=dev.data_ptr())
        else:
            wit = cfg.commit(ps, pinned, rng)
        cfg.prove(ps, None, wit, forms, [ev], rng)
        out = ps.proof()
        del wit
        return out

    ref_proof = one("device")
    for _ in range(max(args.warmup, 3) - 1):
        one("device")
    assert one("host") == ref_proof, "host and device inputs differ"
    clocks = ClockSampler(H.local_rank)
    clocks.start()
    time.sleep(0.3)
    launches0 = ctx.launch_count()
    lat = []

    def device_steps():
        out = None
        for _ in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            out = one("device")
            b.record(stream)
            lat.append((a, b))
        return out

    elapsed, out = H.timed(stream, device_steps)
    launches = ctx.launch_count() - launches0
    assert out == ref_proof
    lat = sorted(a.elapsed_time(b) for a, b in lat)

    def host_steps():
        o = None
        for _ in range(args.steps):
            o = one("host")
        return o

    e2e_ms, out = H.timed(stream, host_steps)
    h2d, d2h = ctx.last_io_bytes()
    clk = clocks.stop()
    assert out == ref_proof
    # per-family device time over steps proofs against the inner proofs' algorithmic bytes
    ctx.set_timing(True)
    ctx.kernel_stats(reset=True)
    for _ in range(args.steps):
        one("device")
    fam = {f: v[1] / args.steps for f, v in ctx.kernel_stats(reset=True).items()}
    ctx.set_timing(False)
    alg = zk_algorithmic_bytes(cfg)
    dominant = max(alg.keys(), key=lambda f: fam.get(f, 0.0))
    peak, peak_kind = read_peaks()
    achieved = alg[dominant] / (fam[dominant] / 1000.0) / 1e9
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": read_traffic(dominant, alg[dominant]), "kernel": dominant, "peak_source": peak_kind,
            "algorithmic_bytes_per_proof": alg[dominant], "ms_per_proof": fam[dominant],
            "traffic_unit": "DRAM bytes per proof of the family (ratio of the plain-proof capture)",
            "binding_limit": ALU_BOUND.get(dominant, "HBM")}
    total = args.steps * H.world
    line = {
        "value": total / (elapsed / 1000.0), "ms_per_step": elapsed / args.steps, "prove_ms": elapsed / args.steps,
        "p50_ms": pct(lat, 0.5), "p99_ms": pct(lat, 0.99),
        "e2e": {"value": total / (e2e_ms / 1000.0), "unit": "proofs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches, "roofline": roof, "families_ms_per_proof": {f: round(v, 4) for f, v in fam.items()},
        "clocks": clk, "proof_bytes": len(ref_proof[0]) + len(ref_proof[1]),
    }
    if H.world == 1 and H.rank == 0 and not args.no_cpu_baseline:
        from oracle.refio import REF_ZK_DRIVER

        if os.path.exists(REF_ZK_DRIVER):
            threads = os.cpu_count() or 1
            r = zk_reference(n, rho, coeffs, point, threads)
            same = (r.narg, r.hints) == ref_proof
            assert same, "GPU zero-knowledge proof differs from the reference's"
            line["cpu_baseline"] = {"value": 1000.0 / r.prove_ms, "unit": "proofs/s", "cores": threads,
                                    "kind": "reference",
                                    "sample": f"one zero-knowledge proof of the same input by the reference C++ "
                                              f"prover (oracle/_ref/ref_zk_driver), {r.prove_ms / 1000.0:.2f} s; "
                                              f"its proof bytes equal the GPU's: {same}"}
    ctx._L.whirgpu_host_free(ptr)
    return line


def batch_vs_plain(H, ctx, inputs, shapes, reps):
    """The batch of `shapes` in one captured graph (device-resident inputs)
    against the plain path on the same proofs, both with CUDA events around
    the whole pass; every batched proof is checked against its plain twin."""
    from whirplonk_b200.batch import Batch

    stream = H.torch.cuda.ExternalStream(ctx.stream, device=H.device)
    expected = [plain_prove(ctx, inputs, n, rho) for n, rho in shapes]
    plain_ms, _ = H.timed(stream, lambda: [plain_prove(ctx, inputs, n, rho) for n, rho in shapes])
    b = Batch(ctx, [inputs.request(n, rho, "device") for n, rho in shapes], Batch.GRAPH)
    for _ in range(2):
        b.run()
    batch_ms, _ = H.timed(stream, lambda: [b.run() for _ in range(reps)])
    same = all(b.proof(i) == expected[i] for i in range(len(shapes)))
    b.close()
    assert same, "a batched proof differs from the plain path's"
    plain_rate = len(shapes) / (plain_ms / 1000.0)
    batch_rate = reps * len(shapes) / (batch_ms / 1000.0)
    return {"batched_proofs_per_s": batch_rate, "plain_proofs_per_s": plain_rate, "ratio": batch_rate / plain_rate,
            "identical_to_plain": same, "proofs": len(shapes), "runs": reps}


def run_batch(args, H, ctx, w):
    from whirplonk_b200.batch import Batch

    torch = H.torch
    shapes = workload_shapes(w, 1, gpu_sampler)
    inputs = Inputs(ctx, shapes, H.rank, H.device)
    stream = torch.cuda.ExternalStream(ctx.stream, device=H.device)
    # plain path: one proof at a time, device-resident inputs
    expected = [plain_prove(ctx, inputs, n, rho) for n, rho in shapes]
    plain_ms, _ = H.timed(stream, lambda: [plain_prove(ctx, inputs, n, rho) for n, rho in shapes])
    dev_batch = Batch(ctx, [inputs.request(n, rho, "device") for n, rho in shapes], Batch.GRAPH)
    host_batch = Batch(ctx, [inputs.request(n, rho, "host") for n, rho in shapes], Batch.GRAPH)
    for _ in range(max(args.warmup, 3)):
        dev_batch.run()
    host_batch.run()
    for i in range(len(shapes)):
        assert dev_batch.proof(i) == expected[i] and host_batch.proof(i) == expected[i], f"batched proof {i} differs"

    clocks = ClockSampler(H.local_rank)
    clocks.start()
    time.sleep(0.3)
    launches0 = ctx.launch_count()
    lat = []

    def steps(b):
        for _ in range(args.steps):
            t0 = time.perf_counter()
            b.run()
            lat.append(1000.0 * (time.perf_counter() - t0))

    elapsed, _ = H.timed(stream, lambda: steps(dev_batch))
    launches = ctx.launch_count() - launches0
    lat_dev = list(lat)
    lat.clear()

    def host_steps():
        steps(host_batch)
        return [host_batch.proof(i) for i in range(len(shapes))]

    e2e_ms, proofs = H.timed(stream, host_steps)
    clk = clocks.stop()
    assert proofs == expected
    for i in range(len(shapes)):
        assert dev_batch.proof(i) == expected[i]
    h2d = sum(inputs.coeff_bytes(n) + 96 + n * 24 + 24 for n, _ in shapes)
    d2h = sum(len(a) + len(b) for a, b in expected)
    dev_batch.close()
    host_batch.close()
    roof, fams, extra = family_roofline(ctx, inputs, shapes)
    count = len(shapes)
    total = count * args.steps * H.world
    plain_rate = H.sum_over_ranks(count / (plain_ms / 1000.0))
    line = {
        "value": total / (elapsed / 1000.0), "ms_per_step": elapsed / args.steps,
        "p50_ms": pct(lat_dev, 0.5), "p99_ms": pct(lat_dev, 0.99), "latency_note": "per batch run (64 proofs)",
        "plain_proofs_per_s": plain_rate, "batched_vs_plain": (total / (elapsed / 1000.0)) / plain_rate,
        "identical_to_plain": True,
        "e2e": {"value": total / (e2e_ms / 1000.0), "unit": "proofs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches, "roofline": roof, "families_ms_per_proof_plain": fams, "clocks": clk,
    }
    line.update(extra)
    if H.world == 1 and H.rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample(shapes, args.steps, inputs)
    inputs.close()
    return line


def serve(srv, reqs, arrivals=None):
    """Submits `reqs` (all at once, or at the given offsets in seconds) and
    returns the served results in request order."""
    tickets = []
    t0 = time.perf_counter()
    for i, r in enumerate(reqs):
        if arrivals is not None:
            wait = t0 + arrivals[i] - time.perf_counter()
            if wait > 0:
                time.sleep(wait)
        tickets.append(srv.submit(r))
    return [srv.poll(t, timeout_ms=300_000) for t in tickets]


def run_served(args, H, ctx, w):
    from whirplonk_b200.batch import Server

    torch = H.torch
    shapes = workload_shapes(w, args.steps, gpu_sampler)
    inputs = Inputs(ctx, shapes, H.rank, H.device)
    stream = torch.cuda.ExternalStream(ctx.stream, device=H.device)
    free, _ = torch.cuda.mem_get_info()
    budget = int(0.6 * free)
    max_inflight = 24  # throughput flat from 16 to 96 in flight; p99 grows with it (46.7 ms at 16, 58.7 at 24, 67.5 at 32)

    # plain path: one proof at a time through the single-proof API (warm first)
    for n, rho in sorted(set(shapes)):
        plain_prove(ctx, inputs, n, rho)
    plain_lat = []

    def plain_all():
        out = []
        for n, rho in shapes:
            t0 = time.perf_counter()
            out.append(plain_prove(ctx, inputs, n, rho))
            plain_lat.append(1000.0 * (time.perf_counter() - t0))
        return out

    plain_ms, expected = H.timed(stream, plain_all)

    srv = Server(ctx, hbm_budget=budget, max_inflight=max_inflight)
    dev_reqs = [inputs.request(n, rho, "device") for n, rho in shapes]
    host_reqs = [inputs.request(n, rho, "host") for n, rho in shapes]
    for _ in range(max(args.warmup, 3) - 1):  # captures the per-workspace programs
        serve(srv, dev_reqs)
    # A workspace is allocated when a shape has more requests in flight than it
    # has idle workspaces cached; how many a pass needs depends on admission
    # timing.  Warm until a pass allocates none (a long-running server's
    # settled cache), at most 8 more passes.
    settle = 0
    for settle in range(1, 9):
        a0 = ctx.workspace_stats()["allocations"]
        serve(srv, dev_reqs)
        if ctx.workspace_stats()["allocations"] == a0:
            break
    res = serve(srv, host_reqs)
    for i, r in enumerate(res):
        assert r.status == 0 and (r.narg, r.hints) == expected[i], f"served request {i} differs from plain"
    serve(srv, dev_reqs)  # the timed pass starts from the state a device pass leaves

    clocks = ClockSampler(H.local_rank)
    clocks.start()
    time.sleep(0.3)
    launches0 = ctx.launch_count()
    ws0 = ctx.workspace_stats()
    elapsed, res = H.timed(stream, lambda: serve(srv, dev_reqs))
    ws1 = ctx.workspace_stats()
    launches = ctx.launch_count() - launches0
    assert all(r.status == 0 and (r.narg, r.hints) == expected[i] for i, r in enumerate(res))
    e2e_ms, res = H.timed(stream, lambda: serve(srv, host_reqs))
    clk = clocks.stop()
    assert all(r.status == 0 and (r.narg, r.hints) == expected[i] for i, r in enumerate(res))

    count = len(shapes)
    served_rate = count / (elapsed / 1000.0)
    plain_rate = count / (plain_ms / 1000.0)
    # latency under seeded Poisson arrivals
    rng = np.random.Generator(np.random.PCG64(w["seed"] + H.rank))
    sweep = []
    for frac in (0.5, 0.8):
        lam = frac * served_rate
        arrivals = np.cumsum(rng.exponential(1.0 / lam, count))
        arrivals -= arrivals[0]
        res = serve(srv, dev_reqs, arrivals)
        assert all(r.status == 0 and (r.narg, r.hints) == expected[i] for i, r in enumerate(res))
        tot = [r.total_ms for r in res]
        sweep.append({"offered_proofs_per_s": lam, "p50_ms": pct(tot, 0.5), "p99_ms": pct(tot, 0.99),
                      "mean_queue_ms": statistics.mean(r.queue_ms for r in res)})
    # the plain path under the same arrivals as the 80% point: one proof at a time, FIFO
    plain_tot = []
    t0 = time.perf_counter()
    for i, (n, rho) in enumerate(shapes):
        wait = t0 + arrivals[i] - time.perf_counter()
        if wait > 0:
            time.sleep(wait)
        plain_prove(ctx, inputs, n, rho)
        plain_tot.append(1000.0 * (time.perf_counter() - (t0 + arrivals[i])))
    st = srv.stats()
    srv.close()

    # the plain path's 2^24 prove time (config 3 shape: n=24, rate 1/4)
    if (24, 2) not in inputs.pts:
        _, point = make_inputs(24, point_seed(H.rank, 24, 2), gpu_sampler)
        if 24 not in inputs.host:
            inputs.host[24], _ = make_inputs(24, coeff_seed(H.rank, 24), gpu_sampler)
            inputs.dev[24] = torch.from_numpy(inputs.host[24].view(np.int64)).to(H.device)
        inputs.pts[(24, 2)] = point
        inputs.evs[(24, 2)] = np.array(ctx.mle_evaluate(inputs.host[24], point), dtype=np.uint64).reshape(1, 3)
    plain_prove(ctx, inputs, 24, 2)
    n24_ms, _ = H.timed(stream, lambda: [plain_prove(ctx, inputs, 24, 2) for _ in range(5)])

    # served / plain by size class on the same stream: each class's requests
    # served alone, against the plain path's time on those requests.
    classes = {}
    srv = Server(ctx, hbm_budget=budget, max_inflight=max_inflight)
    for name, lo, hi in (("n12_18", 12, 18), ("n19_21", 19, 21), ("n22_24", 22, 24)):
        idx = [i for i, (n, _) in enumerate(shapes) if lo <= n <= hi]
        if not idx:
            continue
        sub = [dev_reqs[i] for i in idx]
        serve(srv, sub)  # programs of this class captured, state as in the timed pass
        passes = []
        for _ in range(3):  # a class is a fraction of a second of work: median of three passes
            ms, res = H.timed(stream, lambda: serve(srv, sub))
            assert all(r.status == 0 and (r.narg, r.hints) == expected[i] for i, r in zip(idx, res))
            passes.append(ms)
        ms = statistics.median(passes)
        p_ms = sum(plain_lat[i] for i in idx)
        classes[name] = {"requests": len(idx), "served_proofs_per_s": len(idx) / (ms / 1000.0),
                         "plain_proofs_per_s": len(idx) / (p_ms / 1000.0), "served_vs_plain": p_ms / ms,
                         "plain_share_of_time": p_ms / sum(plain_lat)}
    srv.close()
    # the 64-proof batch (n uniform on {14..22}) in one graph launch, against the plain path
    bshapes = workload_shapes(WORKLOADS["whir_batch64_n14_22"], 1, gpu_sampler)
    inputs.extend(bshapes)
    b64 = batch_vs_plain(H, ctx, inputs, bshapes, reps=3)

    roof, fams, extra = family_roofline(ctx, inputs, shapes[: w["per_step"]])
    h2d = sum(inputs.coeff_bytes(n) + 96 + n * 24 + 24 for n, _ in shapes) / args.steps
    d2h = sum(len(a) + len(b) for a, b in expected) / args.steps
    total_value = H.sum_over_ranks(served_rate)
    line = {
        "value": total_value, "ms_per_step": elapsed / args.steps,
        "p50_ms": sweep[1]["p50_ms"], "p99_ms": sweep[1]["p99_ms"],
        "latency_note": "submit -> result under seeded Poisson arrivals at 80% of the saturated served rate",
        "plain_proofs_per_s": H.sum_over_ranks(plain_rate), "served_vs_plain": served_rate / plain_rate,
        "plain_p50_ms_same_arrivals": pct(plain_tot, 0.5), "plain_p99_ms_same_arrivals": pct(plain_tot, 0.99),
        "plain_p50_ms_alone": pct(plain_lat, 0.5), "plain_p99_ms_alone": pct(plain_lat, 0.99),
        "served_vs_plain_by_size": classes,
        "batch64_vs_plain": b64["ratio"], "batch64": b64,
        "latency_sweep": sweep, "identical_to_plain": True, "prove_ms_n24_rate4": n24_ms / 5,
        "server": {"hbm_budget_bytes": budget, "max_inflight": max_inflight, "peak_inflight": st["peak_inflight"],
                   "peak_bytes": st["peak_bytes"], "workspace_cache_bytes": ws1["cached_bytes"],
                   "workspaces_allocated_in_timed_pass": ws1["allocations"] - ws0["allocations"],
                   "workspaces_evicted_in_timed_pass": ws1["evictions"] - ws0["evictions"],
                   "warm_passes_to_settle": settle},
        "e2e": {"value": H.sum_over_ranks(count / (e2e_ms / 1000.0)), "unit": "proofs/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": launches, "roofline": roof, "families_ms_per_proof_plain": fams, "clocks": clk,
    }
    line.update(extra)
    if H.world == 1 and H.rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample(shapes, args.steps, inputs)
    inputs.close()
    return line


KERNEL_METRIC = "kernel-level RS commitment (NTT/LDE + BLAKE3 leaves + Merkle root) per vector"


def kernel_config(name, w):
    return {"workload": name, "vectors": w["count"], "log_len": w["log_len"], "expansion": 1 << w["log_exp"],
            "row_elements": 1 << w["log_depth"], "hash": "BLAKE3", "seed": w["seed"],
            "l2": "codewords of 4 x 2^24 words (512 MiB) far above the 126 MB L2; no flush"}


def run_kernel(args, H, ctx, w):
    """Kernel-level commitment of `count` vectors per step (rs_commit_batch):
    device-resident inputs for `value`, pinned host inputs for `e2e`; the
    reference's CUDA side-car on the same vectors beside it, roots compared."""
    from whirplonk_b200.rs import rs_commit_batch

    torch = H.torch
    vectors = kernel_vectors(w, gpu_sampler)
    count, log_len, log_exp, log_depth = w["count"], w["log_len"], w["log_exp"], w["log_depth"]
    dev = torch.from_numpy(vectors.reshape(-1).view(np.int64)).to(H.device)
    ptr = ctx._L.whirgpu_host_alloc(vectors.nbytes)
    pinned = np.ctypeslib.as_array((ctypes.c_uint64 * vectors.size).from_address(ptr)).reshape(count, -1)
    pinned[:] = vectors
    stream = torch.cuda.ExternalStream(ctx.stream, device=H.device)

    def dev_step():
        return rs_commit_batch(ctx, None, log_exp, log_depth, on_device_ptr=dev.data_ptr(), count=count,
                               log_len=log_len)

    roots = dev_step()
    assert rs_commit_batch(ctx, pinned, log_exp, log_depth) == roots
    for _ in range(max(args.warmup, 3)):
        dev_step()
    clocks = ClockSampler(H.local_rank)
    clocks.start()
    time.sleep(0.3)
    launches0 = ctx.launch_count()
    elapsed, out = H.timed(stream, lambda: [dev_step() for _ in range(args.steps)][-1])
    launches = ctx.launch_count() - launches0
    assert out == roots
    e2e_ms, out = H.timed(stream, lambda: [rs_commit_batch(ctx, pinned, log_exp, log_depth)
                                           for _ in range(args.steps)][-1])
    clk = clocks.stop()
    assert out == roots
    N = ((1 << log_len) >> log_depth) << log_exp
    d = 1 << log_depth
    alg = count * (8 * ((1 << log_len) + N * d) + (8 * d * N + 32 * N) + 3 * 32 * N)
    bfly = count * d * (N // 2) * (log_len - log_depth)
    comps = count * (N * -(-(8 * d) // 64) + N - 1)
    step_s = elapsed / 1000.0 / args.steps
    peak, peak_kind = read_peaks()
    line = {
        "value": count * args.steps * H.world / (elapsed / 1000.0), "ms_per_step": elapsed / args.steps,
        "e2e": {"value": count * args.steps * H.world / (e2e_ms / 1000.0), "unit": "commitments/s",
                "h2d_bytes_per_step": int(vectors.nbytes), "d2h_bytes_per_step": 32 * count},
        "gpu_launches": launches, "clocks": clk,
        "roofline": {"bound": "hbm", "kernel": "rs_commit (LDE + leaves + Merkle, one call)",
                     "achieved": alg / step_s / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / step_s / 1e9 / peak, "traffic": None, "peak_source": peak_kind,
                     "algorithmic_bytes_per_step": alg},
    }
    pk = measure_int_peaks(ctx.device)
    if pk:
        line["roofline_int"] = {"whole_call": {"butterflies_per_s": bfly / step_s, "compressions_per_s": comps / step_s,
                                               "butterfly_peak": pk["butterflies_per_s"],
                                               "compression_peak": pk["blake3_compressions_per_s"],
                                               "note": "the whole call's time against each unit count: lower bounds "
                                                       "on each family's own rate"}}
        line["int_peaks_measured"] = pk
    if H.world == 1 and H.rank == 0 and not args.no_cpu_baseline:
        from oracle.refio import Oracle

        O = Oracle()
        t0 = time.perf_counter()
        oroots = [O.rs_commit_root(vectors[k], N, d) for k in range(count)]
        cpu_s = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": count / cpu_s, "unit": "commitments/s", "cores": os.cpu_count() or 1,
                                "kind": "port", "sample": f"the same {count} vectors through the oracle's matrix "
                                                          f"commitment (OpenMP), {cpu_s:.1f} s; roots equal the GPU's: "
                                                          f"{oroots == roots}"}
        assert oroots == roots, "kernel-level roots differ from the oracle's"
        r = reference_gpu_commit(w, vectors)
        if r is not None:
            rroots, rms = r
            ours = count / (e2e_ms / 1000.0 / args.steps)
            theirs = count / (rms / 1000.0)
            line["reference_gpu"] = {"value": theirs, "unit": "commitments/s", "ms_per_step": rms,
                                     "roots_equal": rroots == roots,
                                     "sample": "the reference's CUDA side-car (oracle/_ref/ref_gpu_driver, built "
                                               "unmodified for sm_100a) on the same vectors, host in / host out, "
                                               "median of 3 passes after a warm-up"}
            line["vs_reference_gpu"] = ours / theirs
    ctx._L.whirgpu_host_free(ptr)
    return line


def run_gpu_arm(args, rank, world, local_rank):
    from whirplonk_b200 import Context

    H = Harness(rank, world, local_rank)
    w = WORKLOADS[args.workload]
    ctx = Context(local_rank)
    body = {"single": run_single, "batch": run_batch, "served": run_served, "zk": run_zk,
            "kernel": run_kernel}[w["kind"]](args, H, ctx, w)
    kernel = w["kind"] == "kernel"
    line = {"metric": KERNEL_METRIC if kernel else METRIC, "value": body.pop("value"),
            "unit": "commitments/s" if kernel else "proofs/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": body.pop("ms_per_step"), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": DTYPE, "data": DATA,
            "config": kernel_config(args.workload, w) if kernel else config_of(args.workload, w),
            "parallelism": f"replicas x{world} (one independent request stream per GPU)" if world > 1 else "1 GPU"}
    line.update(body)
    ctx.close()
    if rank == 0:
        print(json.dumps(line))
    H.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["gpu", "reference"], default="gpu")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    rank, world, local_rank = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    return run_gpu_arm(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
