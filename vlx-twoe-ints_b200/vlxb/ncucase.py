"""One class entry point on a small s/p/d system: the case for ncu captures.

    python -m vlxb.ncucase --kind K --cls pddd [--atoms 12] [--reps 2] [--variant V]

Builds a seeded 4s+3p+2d cluster (degree 3, the benchmark's shell recipe and
density), uploads the lists, loads the tuned schedule, then calls the one
class `reps` times (the first call is the warm-up) and prints the time of the
last call.  A handful of device allocations of a few hundred MB at most.
"""
from __future__ import annotations

import argparse
import time

import torch

from . import basis, fock, lists
from ._lib import lib
from .tune import apply_schedule


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kind", choices=["J", "K"], default="K")
    ap.add_argument("--cls", default="pddd")
    ap.add_argument("--atoms", type=int, default=12)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--fp32-cut", type=float, default=0.0)
    ap.add_argument("--variant", type=int, default=None, help="kernel variant for the class (default: tuned)")
    args = ap.parse_args()
    L = lib()
    L.init(0)
    apply_schedule()
    L.set_fp32_cut(args.fp32_cut)
    if args.variant is not None:
        L.set_schedule(args.kind, args.cls, args.variant)
    side = 14.0 * (args.atoms / 40.0) ** (1.0 / 3.0)
    wl = basis.config_custom(args.atoms, side, {0: 4, 1: 3, 2: 2}, 3, 0.05, 2.5, max(2, 2 * args.atoms),
                             1e-12, 0)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    dl = fock.to_device(rl)
    matJ, matK = fock.alloc_outputs(dl)
    dt = 0.0
    for _ in range(args.reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if args.kind == "J":
            fock.build_jk(dl, j_only=[args.cls], do_k=False, matJ=matJ, matK=matK)
        else:
            fock.build_jk(dl, k_only=[args.cls], do_j=False, matJ=matJ, matK=matK)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
    q = L.quartet_counters(reset=True)
    print(f"{args.kind} {args.cls} variant {L.get_schedule(args.kind, args.cls)}: {dt * 1e3:.2f} ms, {q} quartets "
          f"(all reps), {rl.naos} AOs")


if __name__ == "__main__":
    main()
