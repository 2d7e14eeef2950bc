"""The allocation-free MLE evaluation (whirgpu_mle_evaluate_noalloc).

It exists for callers that cannot call cudaMalloc where they need the value
(host callbacks, callers with their own device-memory pool, latency-critical
loops): its working memory is a fixed device array inside the library and the
caller passes device buffers for the inputs and the output.

Each size is checked against the CPU oracle and against the allocating entry
point (whirgpu_mle_evaluate), on calls in a row of different sizes, so every
call after the first runs on the array the previous call left behind.  The
sizes include n = 24, the documented maximum, where the working memory nearly
fills the array, and n = 0, a one-entry table.  This file is collected last so
that a stop-at-first-failure run has already run every other test; it also
passes alone in a fresh process.
"""
import numpy as np
import pytest

from oracle.refio import Oracle
from whirplonk_b200 import Context, _lib, sample_goldilocks

pytestmark = pytest.mark.gpu


def _call(L, dcoeffs, n, dpoint, dout, stream):
    return L.whirgpu_mle_evaluate_noalloc(dcoeffs.data_ptr(), n, dpoint.data_ptr(), dout.data_ptr(), stream)


def test_noalloc_mle_matches_oracle_and_allocating_entry_point():
    torch = pytest.importorskip("torch")
    L = _lib.load()
    O = Oracle()
    ctx = Context(0)
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    try:
        for call, n in enumerate((20, 24, 13, 0, 24)):
            coeffs = sample_goldilocks(500 + call, 1 << n)
            point = sample_goldilocks(600 + call, 3 * n)
            expected = tuple(int(x) for x in O.mle_eval_base(coeffs, point))
            assert ctx.mle_evaluate(coeffs, point) == expected, f"allocating entry point differs at n={n}"
            dcoeffs = torch.from_numpy(coeffs.view(np.int64)).cuda()
            # n = 0 has no coordinates; the entry point still wants a device pointer
            dpoint = torch.from_numpy(point.view(np.int64)).cuda() if n else torch.zeros(3, dtype=torch.int64,
                                                                                         device="cuda")
            dout = torch.full((3,), -1, dtype=torch.int64, device="cuda")
            assert _call(L, dcoeffs, n, dpoint, dout, stream.cuda_stream) == _lib.OK
            stream.synchronize()
            got = tuple(int(x) for x in dout.cpu().numpy().view(np.uint64))
            assert got == expected, f"call {call} (n={n}): {got} != {expected}"
            del dcoeffs
    finally:
        ctx.close()


def test_noalloc_mle_rejects_sizes_above_capacity():
    torch = pytest.importorskip("torch")
    L = _lib.load()
    dummy = torch.zeros(8, dtype=torch.int64, device="cuda")
    n = _lib.NOALLOC_MLE_MAX_VARS + 1
    assert _call(L, dummy, n, dummy, dummy, torch.cuda.current_stream().cuda_stream) == _lib.E_TOO_LARGE
