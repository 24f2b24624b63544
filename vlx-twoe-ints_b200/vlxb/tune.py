"""Autotuner: pick the kernel variant of every J and K class by timing.

For each class and each compiled variant (J: thread-per-quartet, column,
McMurchie-Davidson, thread-per-quartet with TMA-staged kets;
K: thread-per-quartet, column with bra or ket lanes, contracted column,
packed column) the class
entry point is timed with CUDA events on a given system's lists (best of
`reps`), and the fastest variant is kept.  The result is a JSON schedule
({"J": {class: variant}, "K": {...}}) that `apply_schedule` loads into the
library's table (vlxb_setSchedule).  Every variant computes the same J/K to
rounding, so the choice only changes speed.

    python -m vlxb.tune [--out vlxb/schedule_b200.json]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_SCHEDULE = os.path.join(HERE, "schedule_b200.json")


# Thread-per-quartet kernels whose code does not fit in registers (ptxas
# keeps them at 32 registers with 15-87 KB of local memory per thread); they
# are 5-10x slower than the column kernels and are not timed.
SPILLING_THREAD_KERNELS = {
    "J": {"dddd"},
    "K": {"ddds", "dpdp", "ppdd", "pddp", "sddd", "pdpd", "dpdd", "dddp", "pddd", "dddd"},
}


def compiled_variants(kind: str, cls: str):
    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "csrc"))
    from gen_column import k_variants

    if kind == "J":
        return [1, 2] if cls in SPILLING_THREAD_KERNELS["J"] else [0, 1, 2, 3]
    l = [{"s": 0, "p": 1, "d": 2}[x] for x in cls]
    return k_variants(*l, spilling=cls in SPILLING_THREAD_KERNELS["K"])


def apply_schedule(path: str = DEFAULT_SCHEDULE) -> bool:
    """Load a tuned schedule into the library (returns False if absent)."""
    from ._lib import lib

    if not os.path.exists(path):
        return False
    sched = json.load(open(path))
    L = lib()
    for kind in ("J", "K"):
        for cls, v in sched.get(kind, {}).items():
            L.set_schedule(kind, cls, int(v))
    return True


def tune(dl, reps: int = 2, log=print):
    import torch

    from . import fock, lists
    from ._lib import lib

    L = lib()
    matJ, matK = fock.alloc_outputs(dl)
    stream = torch.cuda.current_stream(dl.device)
    result = {"J": {}, "K": {}}
    timings = {"J": {}, "K": {}}
    for kind, classes in (("J", lists.j_classes()), ("K", lists.k_classes())):
        for cls in classes:
            if kind == "J" and not (cls[:2] in dl.j and cls[2:] in dl.j):
                continue
            if kind == "K" and not (cls[0] + cls[2] in dl.kpair and cls[:2] in dl.kpart and cls[2:] in dl.kpart):
                continue
            saved = L.get_schedule(kind, cls)
            best = None
            timings[kind][cls] = {}
            variants = compiled_variants(kind, cls)
            variants.sort(key=lambda v: v != saved)  # current choice first
            for v in variants:
                L.set_schedule(kind, cls, v)
                ts = []
                for rep in range(reps):
                    if rep > 0 and best is not None and ts[0] > 4.0 * best[0]:
                        break  # far slower than the best so far: one timing is enough
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    torch.cuda.synchronize()
                    e0.record(stream)
                    if kind == "J":
                        fock.build_jk(dl, matJ=matJ, matK=matK, j_only=[cls], do_k=False)
                    else:
                        fock.build_jk(dl, matJ=matJ, matK=matK, k_only=[cls], do_j=False)
                    e1.record(stream)
                    e1.synchronize()
                    ts.append(e0.elapsed_time(e1))
                t = float(np.min(ts))
                timings[kind][cls][v] = t
                if best is None or t < best[0]:
                    best = (t, v)
            L.set_schedule(kind, cls, saved)
            result[kind][cls] = best[1]
            log(f"{kind} {cls}: " + ", ".join(f"v{v}={t:.2f}ms" for v, t in timings[kind][cls].items())
                + f" -> v{best[1]}")
    return result, timings


def main():
    import torch

    from . import basis, fock, lists
    from ._lib import lib

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_SCHEDULE)
    ap.add_argument("--config", choices=["medium", "small"], default="medium")
    ap.add_argument("--reps", type=int, default=2)
    args = ap.parse_args()
    lib().init(0)
    wl = basis.config_medium(0) if args.config == "medium" else basis.config_small(0)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    dl = fock.to_device(rl)
    res, timings = tune(dl, reps=args.reps)
    with open(args.out, "w") as fh:
        json.dump({"J": res["J"], "K": res["K"], "device": torch.cuda.get_device_name(0),
                   "timings_ms": timings}, fh, indent=1, sort_keys=True)
    print(f"wrote {args.out}")


if __name__ == "__main__":
    main()
