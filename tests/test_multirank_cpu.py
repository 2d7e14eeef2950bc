"""The bench's multi-GPU path (one process per GPU, replicas with no
data-path collective) on the host: two gloo ranks check the harness's
barrier, max-over-ranks timing and sum-over-ranks throughput, and that each
rank draws its own inputs (weak scaling)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench

    H = bench.Harness(rank, world, rank, backend="gloo")
    elapsed = H.max_over_ranks(10.0 * (rank + 1))   # the slowest rank's time
    rate = H.sum_over_ranks(100.0 + rank)          # whole-job throughput
    coeffs, point = bench.make_inputs(10, bench.coeff_seed(rank, 10), bench.gpu_sampler)
    shapes = bench.workload_shapes(bench.WORKLOADS["whir_served_mixed_n12_24"], 2, bench.gpu_sampler)
    H.barrier()
    H.close()
    q.put((rank, elapsed, rate, int(coeffs[0]), int(point[0, 0, 0]), shapes[:4]))


def test_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    for rank, elapsed, rate, _, _, _ in out:
        assert elapsed == 20.0 and rate == 201.0
    assert out[0][3] != out[1][3] and out[0][4] != out[1][4]  # per-rank coefficients and points
    assert out[0][5] == out[1][5]  # the same request mix on every rank
