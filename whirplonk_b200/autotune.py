"""NTT pass-plan autotuner.

For every LDE shape a set of proofs uses -- (log N, log expansion, planes) of
the initial commitment and of every round commitment -- times all valid pass
plans on the device, keeps the fastest and writes the table as JSON.  The
library installs ``ntt_plans.json`` beside ``libwhirgpu.so`` (or the file named
by ``WHIRGPU_NTT_PLANS``) when the first context is created.

    python -m whirplonk_b200.autotune --out whirplonk_b200/ntt_plans.json
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import time
from typing import Iterable, List, Tuple

from . import _lib
from .whir import Config, Context, ProtocolParameters

DEFAULT_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ntt_plans.json")


def lde_shapes(n: int, params: ProtocolParameters) -> List[Tuple[int, int, int]]:
    """(log N, log expansion, planes) of every RS encoding in one proof."""
    sched = Config.from_params(1 << n, params).schedule
    d_log = params.initial_folding_factor
    out = []
    N0 = sched[1]
    m0 = (1 << n) >> d_log
    out.append((N0.bit_length() - 1, (N0 // m0).bit_length() - 1, 1 << d_log))
    fd = params.folding_factor
    for r in range(sched[0]):
        vsize, N = sched[6 + 6 * r], sched[7 + 6 * r]
        m = max(1, vsize >> fd)
        out.append((N.bit_length() - 1, max(0, (N // m).bit_length() - 1), 3 << fd))
    return out


def workload_shapes(ns: Iterable[int], rates: Iterable[int], fold: int = 4) -> List[Tuple[int, int, int]]:
    shapes = set()
    for n in ns:
        for rho in rates:
            p = ProtocolParameters.cli(folding_factor=fold, log_inv_rate=rho)
            shapes.update(lde_shapes(n, p))
    return sorted(shapes)


def tune(ctx: Context, shapes, reps: int = 5, log=print) -> list:
    L = _lib.load()
    # several plane counts can share (log N, log expansion): tune on the largest
    best_planes = {}
    for ln, lx, planes in shapes:
        best_planes[(ln, lx)] = max(planes, best_planes.get((ln, lx), 0))
    out = []
    for (ln, lx), planes in sorted(best_planes.items()):
        plan = _lib.NttPlan()
        us, tried = ctypes.c_double(), ctypes.c_uint32()
        t0 = time.perf_counter()
        st = L.whirgpu_ntt_autotune(ctx.handle, ln, lx, planes, reps, ctypes.byref(plan), ctypes.byref(us),
                                    ctypes.byref(tried))
        note = ""
        if st == _lib.E_DEVICE:  # fastest agreeing plan installed; some candidates disagreed
            note = L.whirgpu_last_error(ctx.handle).decode()
        else:
            _lib.check(st, ctx.handle)
        d = plan.as_dict()
        d.update(planes=planes, us=round(us.value, 2), candidates=tried.value)
        if note:
            d["rejected"] = note
        out.append(d)
        log(f"log_n={ln:2d} log_exp={lx:2d} planes={planes:3d}: {d['npass']} passes {d['log_radix'][:d['npass']]} "
            f"cols {d['log_cols'][:d['npass']]} minb {d['min_blocks']} pipe {d['pipelined']}  {us.value:9.1f} us  ({tried.value} plans, "
            f"{time.perf_counter() - t0:.1f} s) {note}")
    return out


def save(path: str, results: list, device: str = "") -> None:
    with open(path, "w") as f:
        json.dump({"device": device, "plans": results}, f, indent=1)


def load(path: str = DEFAULT_PATH) -> int:
    n = ctypes.c_size_t()
    _lib.check(_lib.load().whirgpu_ntt_load_plans(path.encode(), ctypes.byref(n)))
    return n.value


def current_plan(log_n: int, log_expansion: int) -> dict:
    plan = _lib.NttPlan()
    _lib.check(_lib.load().whirgpu_ntt_get_plan(log_n, log_expansion, ctypes.byref(plan)))
    return plan.as_dict()


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--out", default=DEFAULT_PATH)
    ap.add_argument("--n-min", type=int, default=12)
    ap.add_argument("--n-max", type=int, default=24)
    ap.add_argument("--rates", default="1,2,3")
    ap.add_argument("--reps", type=int, default=5)
    args = ap.parse_args()
    ctx = Context(0)
    L = _lib.load()
    L.whirgpu_ntt_clear_plans()  # time every candidate against the built-in plan
    shapes = workload_shapes(range(args.n_min, args.n_max + 1), [int(r) for r in args.rates.split(",")])
    res = tune(ctx, shapes, args.reps)
    try:
        import torch

        dev = torch.cuda.get_device_name(0)
    except Exception:
        dev = ""
    save(args.out, res, dev)
    print(f"wrote {len(res)} plans to {args.out}")
    ctx.close()


if __name__ == "__main__":
    main()
