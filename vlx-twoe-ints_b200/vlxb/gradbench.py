"""Timing of the nuclear-gradient entry points against the J / K builds.

    python -m vlxb.gradbench [--atoms 10] [--density 30] [--seed 7] [--reps 2]

Builds one seeded 4s+3p+2d molecule (`basis.molecule_at_density`, the
served / batched workloads' recipe), uploads its lists, loads the tuned
schedule, and times on the device (CUDA events, after one untimed call each):
the FP64 J build and K build (all 36 / 54 classes), dE_J/dR and dE_K/dR
(all classes plus the per-atom fold), then each exchange-gradient class alone.
Prints one JSON line: times in ms, the largest gradient component and the
largest |sum over atoms| (translational invariance, to the screening error).
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import torch

from . import basis, fock, gradient, lists
from ._lib import lib
from .tune import apply_schedule


def _timed(fn, reps: int):
    fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        out.append(round(e0.elapsed_time(e1), 2))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--atoms", type=int, default=10)
    ap.add_argument("--density", type=float, default=30.0, help="bohr^3 per atom")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--reps", type=int, default=2)
    args = ap.parse_args()
    L = lib()
    L.init(0)
    apply_schedule()
    wl = basis.molecule_at_density(args.atoms, args.density, args.seed)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    dl = fock.to_device(rl)
    cg = gradient.CoulombGradient(dl, wl.mol)
    kg = gradient.ExchangeGradient(dl, wl.mol)
    res = {"workload": wl.name, "naos": wl.mol.naos}
    res["J_build_ms"] = _timed(lambda: fock.build_jk(dl, do_k=False), args.reps)
    res["K_build_ms"] = _timed(lambda: fock.build_jk(dl, do_j=False), args.reps)
    res["dEJ_dR_ms"] = _timed(cg.compute, args.reps)
    res["dEK_dR_ms"] = _timed(kg.compute, args.reps)
    gj = cg.compute().cpu().numpy()
    gk = kg.compute().cpu().numpy()
    res["max_dEJ_dR"] = float(np.abs(gj).max())
    res["max_dEK_dR"] = float(np.abs(gk).max())
    res["max_sum_dEJ_dR"] = float(np.abs(gj.sum(axis=0)).max())
    res["max_sum_dEK_dR"] = float(np.abs(gk.sum(axis=0)).max())
    s = torch.cuda.current_stream().cuda_stream
    G = torch.zeros((6, max(kg.map.total, 1)), dtype=torch.float64, device="cuda")
    per = {}
    for cls in lists.k_classes():
        ac = cls[0] + cls[2]
        if ac not in dl.kpair:
            continue
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        L.exchange_grad(cls, gradient.kgrad_args(dl, cls, G, kg.map.offsets[ac], G.shape[1], s))
        e1.record()
        torch.cuda.synchronize()
        per[cls] = round(e0.elapsed_time(e1), 2)
    res["dEK_dR_class_ms"] = per
    print(json.dumps(res))


if __name__ == "__main__":
    main()
