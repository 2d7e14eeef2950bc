#!/usr/bin/env python3
"""Benchmark of the B200 WHIR prover (one JSON line on rank 0).

Workload (default): the plain WHIR commit + prove of config 3 -- one
multilinear polynomial of 2^24 Goldilocks coefficients (seeded ChaCha20,
uniform in [0, p)), folding factor 4, starting rate 1/4, 100-bit security,
20 PoW bits, BLAKE3, one MLE statement at a seeded random Ext3 point, the
reference CLI domain separator.  One step = one complete proof.

  value  : proofs/s with the coefficients already resident in HBM
  e2e    : proofs/s through the public API with the coefficients in pinned
           host memory (H2D copy and proof read-back inside every step)
  p50/p99: per-proof latency of the device-resident steps
The working set of a step (~3.4 GB) is far above the 126 MB L2, so no flush is
needed between steps.  Multi-GPU: independent replicas (one proof stream per
rank, no collective on the data path), weak scaling.

--impl reference times the reference C++ CPU prover (oracle/_ref/ref_driver,
built from the reference sources) on the same workload with all host threads.
"""
from __future__ import annotations

import argparse
import ctypes
import json
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
WORKLOADS = {
    # name: (num_variables, folding, log_inv_rate, security, pow_bits)
    "whir_prove_n24_rate4": (24, 4, 2, 100, 20),
    "whir_prove_n22_rate4": (22, 4, 2, 100, 20),
    "whir_prove_n18_rate2": (18, 4, 1, 100, 20),
}
DEFAULT_WORKLOAD = "whir_prove_n24_rate4"
FALLBACK_HBM_GBS = 6650.0


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


def read_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def read_traffic(family):
    path = os.path.join(ROOT, "profiles", "dram_traffic.json")
    try:
        with open(path) as f:
            t = json.load(f)
        return t.get(family)
    except (OSError, ValueError):
        return None


# ---------------------------------------------------------------------------
# reference CPU prover
# ---------------------------------------------------------------------------
def make_inputs(n, seed):
    from whirplonk_b200 import sample_goldilocks

    coeffs = sample_goldilocks(seed, 1 << n)
    point = sample_goldilocks(seed + 7919, 3 * n).reshape(1, n, 3)
    return coeffs, point


def time_reference(n, k, rho, sec, pb, coeffs, point, reps):
    from oracle.refio import ref_available, run_reference

    if not ref_available():
        return None
    threads = os.cpu_count() or 1
    times = []
    for _ in range(reps):
        r = run_reference(n, k, rho, sec, pb, point, coeffs, threads=threads)
        times.append((r.commit_ms + r.prove_ms) / 1000.0)
    return times, threads


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    n, k, rho, sec, pb = WORKLOADS[args.workload]
    coeffs, point = make_inputs(n, 1)
    warm = min(args.warmup, 1)
    res = time_reference(n, k, rho, sec, pb, coeffs, point, warm + args.steps)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_driver not built"}))
        return 0
    times, threads = res
    timed = times[warm:]
    total = sum(timed)
    value = len(timed) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "proofs/s", "n_gpus": world,
        "steps": args.steps, "warmup": warm, "ms_per_step": 1000.0 * total / len(timed),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64 (Goldilocks)",
        "data": "synthetic (seeded ChaCha20 coefficients, seeded Ext3 point)",
        "config": {"workload": args.workload, "num_variables": n, "folding_factor": k, "log_inv_rate": rho,
                   "security_level": sec, "pow_bits": pb, "hash": "BLAKE3", "field": "Goldilocks3",
                   "parallelism": "host OpenMP (reference C++ prover)"},
        "p50_ms": 1000.0 * statistics.median(timed), "p99_ms": 1000.0 * max(timed),
        "cpu_baseline": {"value": value, "unit": "proofs/s", "cores": threads, "kind": "reference",
                         "sample": f"{len(timed)} full proofs of the workload (commit+prove, prover clock)"},
        "e2e": {"value": value, "unit": "proofs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_gpu_arm(args, rank, world, local_rank):
    import torch

    from whirplonk_b200 import Context, ProtocolParameters, prove_once
    from whirplonk_b200.whir import Config

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local_rank)
    n, k, rho, sec, pb = WORKLOADS[args.workload]
    params = ProtocolParameters.cli(security_level=sec, pow_bits=pb, folding_factor=k, log_inv_rate=rho)
    ctx = Context(local_rank)
    coeffs, point = make_inputs(n, 1 + rank)
    ev = np.array(ctx.mle_evaluate(coeffs, point), dtype=np.uint64).reshape(1, 3)

    # device-resident copy of the coefficients (plumbing: torch owns the buffer)
    dcoeffs = torch.from_numpy(coeffs.view(np.int64)).to(f"cuda:{local_rank}")
    torch.cuda.synchronize()
    dptr = dcoeffs.data_ptr()
    # pinned host copy for the end-to-end path
    L = ctx._L
    hbuf = L.whirgpu_host_alloc(coeffs.nbytes)
    if not hbuf:
        raise MemoryError("pinned allocation failed")
    hview = np.ctypeslib.as_array((ctypes.c_uint64 * coeffs.size).from_address(hbuf))
    hview[:] = coeffs

    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local_rank}")

    def step_device():
        return prove_once(n, params, None, point, ev, ctx=ctx, on_device_ptr=dptr)

    def step_e2e():
        return prove_once(n, params, hview, point, ev, ctx=ctx)

    ref_proof = step_device()
    for _ in range(max(args.warmup, 3) - 1):
        step_device()
    for _ in range(2):
        step_e2e()
    assert step_e2e()[0] == ref_proof[0], "host and device inputs gave different proofs"

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local_rank}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- timed region 1: device-resident inputs --------------------------------
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    ctx.set_timing(True)
    ctx.kernel_stats(reset=True)
    launches0 = ctx.launch_count()
    barrier()
    ev_start = torch.cuda.Event(enable_timing=True)
    ev_end = torch.cuda.Event(enable_timing=True)
    step_events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(args.steps)]
    ev_start.record(stream)
    for i in range(args.steps):
        step_events[i][0].record(stream)
        out = step_device()
        step_events[i][1].record(stream)
    ev_end.record(stream)
    barrier()
    launches = ctx.launch_count() - launches0
    fam = ctx.kernel_stats(reset=True)
    ctx.set_timing(False)
    elapsed_ms = max_over_ranks(ev_start.elapsed_time(ev_end))
    lat = sorted(a.elapsed_time(b) for a, b in step_events)
    assert out[0] == ref_proof[0]

    # ---- timed region 2: end to end through the public API, host inputs ---------
    barrier()
    e_start = torch.cuda.Event(enable_timing=True)
    e_end = torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    for _ in range(args.steps):
        out = step_e2e()
    e_end.record(stream)
    barrier()
    h2d, d2h = ctx.last_io_bytes()
    e2e_ms = max_over_ranks(e_start.elapsed_time(e_end))
    clk = clocks.stop()
    assert out[0] == ref_proof[0]

    total_proofs = args.steps * world
    value = total_proofs / (elapsed_ms / 1000.0)
    e2e_value = total_proofs / (e2e_ms / 1000.0)

    # roofline of the dominant family (algorithmic bytes / measured family time)
    sched = Config.from_params(1 << n, params).schedule
    alg = algorithmic_bytes(sched, n, k)
    fam_ms = {f: v[1] / args.steps for f, v in fam.items()}
    dominant = max(alg.keys(), key=lambda f: fam_ms.get(f, 0.0))
    peak, peak_kind = read_peaks()
    achieved = alg[dominant] / (fam_ms[dominant] / 1000.0) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": read_traffic(dominant), "kernel": dominant, "peak_source": peak_kind,
                "algorithmic_bytes_per_proof": alg[dominant], "ms_per_proof": fam_ms[dominant]}

    line = {
        "metric": METRIC, "value": value, "unit": "proofs/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 (Goldilocks; Ext3 challenges)",
        "data": "synthetic (seeded ChaCha20 coefficients, seeded Ext3 point)",
        "config": {"workload": args.workload, "num_variables": n, "folding_factor": k, "log_inv_rate": rho,
                   "security_level": sec, "pow_bits": pb, "hash": "BLAKE3", "field": "Goldilocks3",
                   "parallelism": f"replicas x{world}", "l2": "working set ~3.4 GB per step > 126 MB L2 (no flush)"},
        "prove_ms": elapsed_ms / args.steps, "p50_ms": lat[len(lat) // 2],
        "p99_ms": lat[min(len(lat) - 1, int(0.99 * len(lat)))],
        "e2e": {"value": e2e_value, "unit": "proofs/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": roofline,
        "families_ms_per_proof": {f: round(v, 4) for f, v in fam_ms.items()},
        "clocks": clk,
    }
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        res = time_reference(n, k, rho, sec, pb, coeffs, point, 1)
        if res is not None:
            times, threads = res
            line["cpu_baseline"] = {"value": 1.0 / times[0], "unit": "proofs/s", "cores": threads,
                                    "kind": "reference",
                                    "sample": "1 full proof of the workload by the reference C++ prover "
                                              "(oracle/_ref, commit+prove clock)"}
        else:
            line["cpu_baseline"] = None
    L.whirgpu_host_free(hbuf)
    del dcoeffs
    ctx.close()
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
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
