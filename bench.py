#!/usr/bin/env python
"""Benchmark: J+K Fock builds through the drop-in C ABI on B200.

Workload: 40 atoms in a 14-bohr cube, 4s+3p+2d contracted Cartesian shells of
degree 3, even-tempered exponents 0.05 * 2.5^k, density from 80 occupied
orbitals, Schwarz threshold 1e-12, FP64 (1000 Cartesian AOs; seeded
synthetic molecule and density, no dataset involved).

One step = one complete J+K build: all 36 Coulomb and 54 exchange entry points
of the C ABI, with the reference's list formats as input (the drop-in path).

  value  screened-in primitive shell quartets per second (J and K quartets of
         one build / device time of one build), inputs resident in HBM
  e2e    the same metric with host (pinned) input buffers copied to the device
         and mat_J / mat_K copied back inside every timed step

    python bench.py [--steps K] [--warmup W] [--gpus N] [--impl reference]

Multi-GPU: the path is a single-GPU build; N GPUs run N independent replicas
(one process per GPU) and value is the aggregate over the replicas.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "vlx-twoe-ints_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

METRIC = "quartets/s & J+K builds/s, mixed vs FP64 at 1e-6 Eh; serve p50/p99 ms"
UNIT = "quartets/s"
L2_BYTES = 126 * 1024 * 1024


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["medium", "small"], default="medium")
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="CPU-baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--fp32-cut", type=float, default=1e-6,
                    help="mixed-precision leg: quartets with bound below this run in FP32 (0 skips the leg)")
    ap.add_argument("--schedule", default=None, help="kernel schedule JSON (default: vlxb/schedule_b200.json)")
    return ap.parse_args()


def workload(name):
    from vlxb import basis

    return basis.config_medium(0) if name == "medium" else basis.config_small(0)


def workload_desc(name, wl, rl):
    nj = sum(len(v.first) for v in rl.jlists.values())
    nk = sum(len(v.pair_i) for v in rl.kpairs.values())
    return {"workload": ("40 atoms 14-bohr cube 4s3p2d deg 3 Cartesian (1000 AOs), nocc 80, thr 1e-12"
                         if name == "medium" else "5 atoms 6-bohr cube 3s2p deg 3 (45 AOs), nocc 10, thr 1e-12"),
            "precision": "fp64", "path": "C ABI: 36 Coulomb + 54 exchange entry points per build",
            "j_pairs": nj, "k_ik_pairs": nk, "naos": rl.naos}


# ----------------------------------------------------------------- clocks
class Clocks:
    def __init__(self, index=0):
        self.index = index
        self.path = tempfile.mktemp(suffix=".csv")
        self.proc = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------- distributed
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        import datetime

        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def dist_max(x):
    import torch
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        t = torch.tensor([float(x)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())
    return float(x)


def dist_barrier():
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.barrier()


# ----------------------------------------------------------------- CPU reference
def cpu_reference(rl, budget_s, seed=0):
    """Time the reference's emitted expressions (oracle/_ref) on a bounded
    sample of this build and extrapolate the full-build time.

    Per class: a seeded random sample of bra rows (J) or (i, k) rows (K); each
    sampled row evaluates at most `max_eval` of its passing component quartets;
    the full-build time is (machine throughput in component quartets/s) divided
    into the sampled rows' exact passing counts scaled to all rows."""
    from oracle import ref
    from vlxb import lists

    threads = os.cpu_count() or 1
    try:
        import ctypes.util  # noqa: F401

        threads = int(os.environ.get("OMP_NUM_THREADS", threads))
    except ValueError:
        pass
    rng = np.random.default_rng(seed)
    classes = [("J", c) for c in lists.j_classes() if c[:2] in rl.jlists and c[2:] in rl.jlists]
    classes += [("K", c) for c in lists.k_classes()
                if c[0] + c[2] in rl.kpairs and c[:2] in rl.kpartners and c[2:] in rl.kpartners]
    per = budget_s / len(classes)
    est_total = 0.0
    cq_eval_total = 0
    rows_total = 0
    for kind, cls in classes:
        n = len(rl.jlists[cls[:2]].first) if kind == "J" else len(rl.kpairs[cls[0] + cls[2]].pair_i)
        nrow = min(n, max(threads, 1))
        rows = np.sort(rng.choice(n, size=nrow, replace=False)).astype(np.uint32)
        # pilot to size the per-row evaluation cap
        f = ref.coulomb if kind == "J" else ref.exchange
        t0 = time.perf_counter()
        _, p_pass, p_eval = f(rl, cls, rows=rows, max_eval=8)
        dt = max(time.perf_counter() - t0, 1e-6)
        rate = max(p_eval, 1) / dt
        cap = int(max(8, min(2**40, rate * per / max(nrow, 1))))
        t0 = time.perf_counter()
        _, c_pass, c_eval = f(rl, cls, rows=rows, max_eval=cap)
        dt = max(time.perf_counter() - t0, 1e-6)
        thr = max(c_eval, 1) / dt  # component quartets per second, whole machine
        est_total += (c_pass / nrow) * n / thr
        cq_eval_total += c_eval
        rows_total += nrow
    return est_total, threads, {"classes": len(classes), "rows": rows_total, "component_quartets": cq_eval_total}


def quartets_per_build_ref(rl):
    from oracle import ref
    from vlxb import lists

    n = 0
    for c in lists.j_classes():
        if c[:2] in rl.jlists and c[2:] in rl.jlists:
            n += ref.count_j(rl, c)
    for c in lists.k_classes():
        if c[0] + c[2] in rl.kpairs and c[:2] in rl.kpartners and c[2:] in rl.kpartners:
            n += ref.count_k(rl, c)
    return n


# ----------------------------------------------------------------- reference arm
def run_reference(args):
    ws, rank, local = dist_setup()
    if rank != 0:
        return 0
    from oracle import ref
    from vlxb import lists

    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref/libvlxref.so not built (built from the reference tree by oracle/make_ref.py)"}))
        return 0
    wl = workload(args.config)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, ref.schwarz_fn)
    qpb = quartets_per_build_ref(rl)
    per_step = max(5.0, min(20.0, 150.0 / max(args.steps + args.warmup, 1)))
    for w in range(args.warmup):
        cpu_reference(rl, per_step, seed=100 + w)
    ests = []
    t0 = time.perf_counter()
    for s in range(args.steps):
        est, threads, sample = cpu_reference(rl, per_step, seed=s)
        ests.append(est)
    wall = time.perf_counter() - t0
    build_s = float(np.mean(ests))
    value = qpb / build_s
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": build_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded molecule and density)",
        "config": workload_desc(args.config, wl, rl) | {"extrapolated": True, "cpu_wall_s": wall},
        "builds_per_s": 1.0 / build_s, "quartets_per_build": qpb,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": (f"per step: {sample['rows']} random rows over {sample['classes']} classes, "
                                    f"{sample['component_quartets']} component quartets evaluated with the "
                                    "reference's emitted expressions; full-build time extrapolated from exact "
                                    "per-row passing counts")},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# ----------------------------------------------------------------- our arm
def fp64_peak(L, device, stream):
    import torch

    blocks = 148 * 16
    out = torch.empty(blocks * 256, dtype=torch.float64, device=device)
    iters = 2048
    for _ in range(2):
        L.check(L.cdll.vlxb_fp64Probe(out.data_ptr(), iters, blocks, stream.cuda_stream), "fp64 probe")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(3):
        L.check(L.cdll.vlxb_fp64Probe(out.data_ptr(), iters, blocks, stream.cuda_stream), "fp64 probe")
    e1.record(stream)
    torch.cuda.synchronize()
    s = e0.elapsed_time(e1) / 1e3 / 3
    return 2.0 * 8 * iters * blocks * 256 / s / 1e12


def run_ours(args):
    import torch

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from vlxb import fock, lists
    from vlxb._lib import lib

    L = lib()
    L.init(local)
    from vlxb.tune import DEFAULT_SCHEDULE, apply_schedule

    sched_loaded = apply_schedule(args.schedule or DEFAULT_SCHEDULE)
    L.set_fp32_cut(0.0)
    stream = torch.cuda.Stream(device=dev)
    wl = workload(args.config)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn(dev))
    host = fock.host_arrays(rl)
    pinned = fock.pinned_copy(host)
    dl = fock.upload(rl, pinned, dev)
    matJ, matK = fock.alloc_outputs(dl)
    flush = torch.empty(L2_BYTES * 2 // 8, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    def zero_outputs():
        for t in matJ.values():
            t.zero_()
        for t in matK.values():
            t.zero_()

    def one_build():
        zero_outputs()
        fock.build_jk(dl, stream=stream, matJ=matJ, matK=matK)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            one_build()
        torch.cuda.synchronize()
        L.reset_counters(stream.cuda_stream)
        L.launch_count(reset=True)
        dist_barrier()
        clocks = Clocks(local)
        clocks.start()
        times = []
        for _ in range(args.steps):
            flush.zero_()  # L2 flush between steps (outside the timed events)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            one_build()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
        torch.cuda.synchronize()
        clk = clocks.stop()
        launches = L.launch_count(reset=True) / args.steps
        qj, qk = L.quartet_counters(reset=True, stream=stream.cuda_stream)
        qpb = (qj + qk) / args.steps
        t_build = dist_max(sum(times)) / args.steps
        dist_barrier()

        # ---- end to end: host buffers in, results out, every step
        e2e_steps = args.e2e_steps or args.steps
        hJ = {k: torch.empty(v.numel(), dtype=torch.float64).pin_memory() for k, v in matJ.items()}
        hK = {k: torch.empty(v.numel(), dtype=torch.float64).pin_memory() for k, v in matK.items()}
        h2d = sum(t.numel() * t.element_size() for t in pinned.values())
        d2h = sum(t.numel() * 8 for t in hJ.values()) + sum(t.numel() * 8 for t in hK.values())
        e2e_times = []
        for it in range(e2e_steps + 1):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            dl2 = fock.upload(rl, pinned, dev, non_blocking=True)
            mJ, mK = fock.alloc_outputs(dl2)
            fock.build_jk(dl2, stream=stream, matJ=mJ, matK=mK)
            for k in mJ:
                hJ[k].copy_(mJ[k], non_blocking=True)
            for k in mK:
                hK[k].copy_(mK[k], non_blocking=True)
            e1.record(stream)
            e1.synchronize()
            if it > 0:  # first pass warms the caching allocator
                e2e_times.append(e0.elapsed_time(e1) / 1e3)
            del dl2, mJ, mK
        t_e2e = dist_max(sum(e2e_times)) / len(e2e_times)

        # ---- roofline: per-class calls timed on the stream (prep + integral kernel)
        fl = json.load(open(os.path.join(PKG, "vlxb", "flops_per_class.json")))["classes"]
        per_class = []
        for kind, clist in (("J", lists.j_classes()), ("K", lists.k_classes())):
            for cls in clist:
                zero_outputs()
                L.reset_counters(stream.cuda_stream)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(stream)
                if kind == "J":
                    fock.build_jk(dl, stream=stream, matJ=matJ, matK=matK, j_only=[cls], do_k=False)
                else:
                    fock.build_jk(dl, stream=stream, matJ=matJ, matK=matK, k_only=[cls], do_j=False)
                e1.record(stream)
                e1.synchronize()
                q = L.quartet_counters(reset=True, stream=stream.cuda_stream)
                nq = q[0] if kind == "J" else q[1]
                per_class.append((kind, cls, e0.elapsed_time(e1) / 1e3, nq, nq * fl[cls][kind]))
        peak = fp64_peak(L, dev, stream)

        # ---- mixed precision leg: same build with FP32 below the cutoff,
        # errors of AO J, K and E against this GPU's FP64 build
        mixed = None
        if args.fp32_cut > 0:
            zero_outputs()
            fock.build_jk(dl, stream=stream, matJ=matJ, matK=matK)
            torch.cuda.synchronize()
            J64 = lists.contract_J(rl, {k: v.cpu().numpy() for k, v in matJ.items()})
            K64 = lists.contract_K(rl, {k: v.cpu().numpy() for k, v in matK.items()})
            L.set_fp32_cut(args.fp32_cut)
            one_build()
            torch.cuda.synchronize()
            mt = []
            for _ in range(args.steps):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                one_build()
                e1.record(stream)
                e1.synchronize()
                mt.append(e0.elapsed_time(e1) / 1e3)
            L.set_fp32_cut(0.0)
            J32 = lists.contract_J(rl, {k: v.cpu().numpy() for k, v in matJ.items()})
            K32 = lists.contract_K(rl, {k: v.cpu().numpy() for k, v in matK.items()})
            t_mix = dist_max(sum(mt)) / len(mt)
            mixed = {"fp32_below_bound": args.fp32_cut, "value": qpb / t_mix * ws, "unit": UNIT,
                     "ms_per_step": t_mix * 1e3, "builds_per_s": ws / t_mix,
                     "speedup_vs_fp64": t_build / t_mix,
                     "max_abs_dJ": float(np.abs(J32 - J64).max()), "max_abs_dK": float(np.abs(K32 - K64).max()),
                     "abs_dE_Eh": abs(lists.energy(wl.D, J32, K32) - lists.energy(wl.D, J64, K64)),
                     "reference": "this GPU's FP64 build (parity-tested against the FP64 oracle at 1e-10)"}

    dom = max(per_class, key=lambda r: r[2])
    total_flops = sum(r[4] for r in per_class)
    total_t = sum(r[2] for r in per_class)
    ach_dom = dom[4] / dom[2] / 1e12
    roofline = {"bound": "fp64", "achieved": ach_dom, "peak": peak, "unit": "TFLOP/s", "frac": ach_dom / peak,
                "traffic": None,
                "kernel": f"{dom[0]} class {dom[1].upper()} (prep + integral kernel)",
                "build_achieved": total_flops / total_t / 1e12, "build_frac": total_flops / total_t / 1e12 / peak,
                "peak_source": "measured: FP64 FMA probe kernel on this GPU (MEASURED_PEAKS.json has no FP64 figure)"}
    value = qpb / t_build * ws
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_build * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded molecule and density)",
        "config": workload_desc(args.config, wl, rl) | {"parallelism": f"replicas x{ws}",
                                                        "l2": "flushed (256 MB write) between timed steps"},
        "builds_per_s": ws / t_build, "quartets_per_build": qpb, "gpu_launches": launches,
        "e2e": {"value": qpb / t_e2e * ws, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": t_e2e * 1e3},
        "roofline": roofline, "clocks": clk, "mixed": mixed,
        "schedule": "autotuned (vlxb/schedule_b200.json)" if sched_loaded else "generator defaults",
        "top_classes": [{"class": f"{k} {c.upper()}", "ms": round(t * 1e3, 2), "quartets": n,
                         "tflops": round(f / t / 1e12, 3)} for k, c, t, n, f in
                        sorted(per_class, key=lambda r: -r[2])[:8]],
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            from oracle import ref

            if ref.available():
                est, threads, sample = cpu_reference(rl, args.cpu_seconds, seed=7)
                line["cpu_baseline"] = {
                    "value": qpb / est, "unit": UNIT, "cores": threads, "kind": "reference",
                    "sample": (f"{sample['rows']} random rows over {sample['classes']} classes, "
                               f"{sample['component_quartets']} component quartets with the reference's emitted "
                               "expressions (oracle/_ref); full-build time extrapolated"),
                    "est_build_s": est}
            else:
                line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                        "sample": "oracle/_ref not built"}
        except Exception as ex:  # the baseline must not sink the GPU measurement
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                    "sample": f"failed: {ex}"}
    if rank == 0:
        print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
