"""Many proofs at once: batches (one CUDA graph per batch) and the serving loop.

    reqs = [ProofRequest(n, params, coeffs, points, evaluations) ...]
    with Batch(ctx, reqs, mode=Batch.GRAPH) as b:
        b.run()
        narg, hints = b.proof(0)

    srv = Server(ctx, hbm_budget=40 << 30, max_inflight=32)
    t = srv.submit(req); res = srv.poll(t, timeout_ms=10_000)
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _lib
from .whir import Context, DomainSeparator, ProtocolParameters, cli_domain_separator


@dataclass
class ProofRequest:
    """One complete commit + prove of params.batch_size vectors of
    2^num_variables coefficients."""

    num_variables: int
    params: ProtocolParameters
    coeffs: object  # numpy uint64 array (batch_size rows), or a device pointer (int) with on_device=True
    points: np.ndarray  # (num_points, n, 3) uint64
    evaluations: np.ndarray  # (num_points * batch_size, 3) uint64, form-major
    ds: Optional[DomainSeparator] = None
    on_device: bool = False
    _keep: list = field(default_factory=list, repr=False)

    def to_c(self) -> _lib.Request:
        r = _lib.Request()
        r.num_variables = self.num_variables
        r.params = self.params.to_c()
        if self.on_device:
            r.coeffs, r.coeffs_location = int(self.coeffs), 1
        else:
            c = np.ascontiguousarray(self.coeffs, dtype=np.uint64)
            assert c.size == self.params.batch_size << self.num_variables
            self._keep.append(c)
            r.coeffs, r.coeffs_location = c.ctypes.data, 0
        pts = np.ascontiguousarray(self.points, dtype=np.uint64).reshape(-1, self.num_variables, 3)
        ev = np.ascontiguousarray(self.evaluations, dtype=np.uint64).reshape(-1, 3)
        self._keep += [pts, ev]
        r.points, r.evaluations, r.num_points = pts.ctypes.data, ev.ctypes.data, pts.shape[0]
        ds = self.ds or cli_domain_separator(self.params)
        for i, b in enumerate(ds.protocol_id):
            r.protocol_id[i] = b
        for i, b in enumerate(ds.session_id):
            r.session_id[i] = b
        return r


class Batch:
    GRAPH, STREAMS, PLAIN = 0, 1, 2

    def __init__(self, ctx: Context, requests: List[ProofRequest], mode: int = GRAPH):
        self.ctx = ctx
        self._L = ctx._L
        self._reqs = requests
        arr = (_lib.Request * len(requests))(*[r.to_c() for r in requests])
        self._arr = arr
        h = ctypes.c_void_p()
        _lib.check(self._L.whirgpu_batch_create(ctx.handle, arr, len(requests), mode, ctypes.byref(h)), ctx.handle)
        self.handle = h.value
        ctx.adopt(self)

    def run(self):
        _lib.check(self._L.whirgpu_batch_run(self.handle), self.ctx.handle)

    def proof(self, i: int):
        narg, hints = ctypes.c_void_p(), ctypes.c_void_p()
        ln, lh = ctypes.c_size_t(), ctypes.c_size_t()
        _lib.check(self._L.whirgpu_batch_proof(self.handle, i, ctypes.byref(narg), ctypes.byref(ln),
                                               ctypes.byref(hints), ctypes.byref(lh)), self.ctx.handle)
        return ctypes.string_at(narg, ln.value), ctypes.string_at(hints, lh.value)

    def close(self):
        if self.handle:
            self._L.whirgpu_batch_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class ServedProof:
    status: int
    narg: bytes
    hints: bytes
    queue_ms: float
    total_ms: float


class Server:
    """Continuous-batching prover: requests are admitted as HBM budget and
    stream slots free up; results are polled by ticket."""

    def __init__(self, ctx: Context, hbm_budget: int = 0, max_inflight: int = 32):
        self.ctx = ctx
        self._L = ctx._L
        h = ctypes.c_void_p()
        _lib.check(self._L.whirgpu_server_create(ctx.handle, hbm_budget, max_inflight, ctypes.byref(h)), ctx.handle)
        self.handle = h.value
        ctx.adopt(self)
        self._live = {}

    def submit(self, req: ProofRequest) -> int:
        """Queues a request; its arrays are borrowed until poll() returns it."""
        t = ctypes.c_uint64()
        creq = req.to_c()
        _lib.check(self._L.whirgpu_server_submit(self.handle, ctypes.byref(creq), ctypes.byref(t)))
        self._live[t.value] = req
        return t.value

    def poll(self, ticket: int, timeout_ms: int = 60_000) -> Optional[ServedProof]:
        r = _lib.Result()
        st = self._L.whirgpu_server_poll(self.handle, ticket, timeout_ms, ctypes.byref(r))
        if st == _lib.E_TIMEOUT:
            return None
        _lib.check(st)
        out = ServedProof(r.status, ctypes.string_at(r.narg, r.narg_len) if r.narg_len else b"",
                          ctypes.string_at(r.hints, r.hints_len) if r.hints_len else b"", r.queue_ms, r.total_ms)
        self._L.whirgpu_server_release(self.handle, ticket)
        self._live.pop(ticket, None)
        return out

    def stats(self):
        a, pi, pb, q = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        self._L.whirgpu_server_stats(self.handle, ctypes.byref(a), ctypes.byref(pi), ctypes.byref(pb), ctypes.byref(q))
        return {"admitted": a.value, "peak_inflight": pi.value, "peak_bytes": pb.value, "queued": q.value}

    def close(self):
        if self.handle:
            self._L.whirgpu_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
