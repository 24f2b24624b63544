"""Per-class device time of one J+K build through the C ABI.

    python -m vlxb.classprof [medium|small] [--schedule PATH] [--fp32-cut X] [--out FILE]

Each of the 36 Coulomb and 54 exchange entry points is called once on the
workload's lists and timed with CUDA events on the calling stream (the time
includes the call's device-side list regrouping); the kernels' own counters
give the screened-in shell quartets of the class.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import torch

from . import basis, fock, lists
from ._lib import lib
from .tune import apply_schedule


def profile(dl, fp32_cut=None):
    L = lib()
    matJ, matK = fock.alloc_outputs(dl)
    res = {}
    for kind, cl in (("J", lists.j_classes()), ("K", lists.k_classes())):
        for cls in cl:
            L.reset_counters()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            if kind == "J":
                fock.build_jk(dl, j_only=[cls], do_k=False, matJ=matJ, matK=matK)
            else:
                fock.build_jk(dl, k_only=[cls], do_j=False, matJ=matJ, matK=matK)
            e1.record()
            torch.cuda.synchronize()
            q = L.quartet_counters(reset=True)
            res[kind + cls] = (e0.elapsed_time(e1), q[0] if kind == "J" else q[1])
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("config", nargs="?", default="medium", choices=["medium", "small"])
    ap.add_argument("--schedule", default=None)
    ap.add_argument("--fp32-cut", type=float, default=None)
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    L = lib()
    L.init(0)
    if args.schedule:
        apply_schedule(args.schedule)
    if args.fp32_cut is not None:
        L.set_fp32_cut(args.fp32_cut)
    t = time.time()
    wl = basis.config_medium(0) if args.config == "medium" else basis.config_small(0)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    print("lists built", round(time.time() - t, 1), "s", flush=True)
    dl = fock.to_device(rl)
    profile(dl)  # warm-up
    res = profile(dl)
    for k, (ms, q) in res.items():
        print(k[0], k[1:], f"{ms:.2f} ms", q, flush=True)
    print("total ms", sum(v[0] for v in res.values()))
    if args.out:
        os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
        json.dump(res, open(args.out, "w"), indent=1)


if __name__ == "__main__":
    main()
