#!/usr/bin/env python
"""Benchmark: J+K Fock builds through the drop-in C ABI on B200.

Workload (the headline): 40 atoms in a 14-bohr cube, 4s+3p+2d contracted
Cartesian shells of degree 3, even-tempered exponents 0.05 * 2.5^k, density
from 80 occupied orbitals, Schwarz threshold 1e-12, FP64 (1000 Cartesian AOs;
seeded synthetic molecule and density, no dataset involved).

One step = one complete J+K build: all 36 Coulomb and 54 exchange entry points
of the C ABI, with the reference's list formats as input (the drop-in path).

  value  screened-in primitive shell quartets per second (J and K quartets of
         one build / device time of one build), inputs resident in HBM
  e2e    the same metric with host (pinned) input buffers copied to the device
         and mat_J / mat_K copied back inside every timed step

    python bench.py [--steps K] [--warmup W] [--gpus N] [--impl reference]

After the timed steps the same line carries the other legs (all on this GPU):
  parity   seeded rows of every J and K list of the headline build against the
           reference's own emitted expressions compiled for the host
           (oracle/_ref, FP64), absolute errors
  mixed    the headline build with FP32 below a Schwarz bound of 1e-6 and an
           FP32 error budget; errors against the FP64 build (whole AO
           matrices) and against oracle/_ref on the parity rows
  small    5 atoms 3s2p (45 AOs): timed in full on the GPU and on the host
           cores (reference expressions), every value checked
  large    the large sparse recipe (25 bohr^3 per atom, 4s3p2d) at 48 atoms
           (1200 AOs; --large-atoms 200 runs the 5000-AO cluster, whose
           incremental build is 6.409e12 quartets, about 48 min of one B200
           in mixed precision): incremental build on
           dD of norm 1e-3, density-weighted screening at 1e-11, mixed
           precision with FP64 accumulation
  batched / served   the batching and serving patterns (served: one rate
           below the plain server's capacity and one far above it)
  cpu_baseline       the reference's emitted expressions with OpenMP on the
           host cores, a bounded sample of the headline build extrapolated

Tool modes (no driver line; used by the profiles under profiles/):
    python bench.py --mode case --kind K --cls pddd [--atoms 12] [--reps 2]
        one class entry point on a small cluster (the case for ncu captures)
    python bench.py --mode classes [--config medium|small]
        device time and quartets of every class entry point
    python bench.py --mode gradient [--atoms 10]
        nuclear-gradient entry points against the J / K builds
    python bench.py --mode gradient-cpu [--atoms 10]
        CPU baseline of the nuclear gradients (oracle port, no GPU)
    python bench.py --mode large|batched|served [leg options]
        one leg alone at the sizes given (e.g. --large-atoms 200 --large-no-fp64,
        --batch-mols 256 --batch-atoms 3 30), one JSON line

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
    ap.add_argument("--mode", choices=["bench", "case", "classes", "gradient", "gradient-cpu", "large", "batched",
                                       "served"], default="bench")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["medium", "small"], default="medium")
    ap.add_argument("--cpu-seconds", type=float, default=20.0, help="CPU-baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--parity-rows", type=int, default=6, help="rows per list checked against oracle/_ref (0: none)")
    ap.add_argument("--e2e-steps", type=int, default=None, help="end-to-end steps (default min(steps, 2))")
    ap.add_argument("--mixed-steps", type=int, default=None, help="mixed-precision steps (default min(steps, 2))")
    ap.add_argument("--fp32-cut", type=float, default=1e-6,
                    help="mixed-precision leg: quartets with bound below this may run in FP32 (0 skips the leg)")
    ap.add_argument("--fp32-budget", type=float, default=None,
                    help="mixed-precision leg: FP32 error budget (default: the library's recommended value)")
    ap.add_argument("--schedule", default=None, help="kernel schedule JSON (default: vlxb/schedule_b200.json)")
    ap.add_argument("--small-steps", type=int, default=5, help="5-atom leg: timed builds (0 skips the leg)")
    ap.add_argument("--large-atoms", type=int, default=48,
                    help="large sparse leg: atoms at 25 bohr^3/atom (0 skips the leg; 200 is the full cluster, "
                         "6.4e12 quartets per incremental build, ~48 min)")
    ap.add_argument("--pattern-fp32-cut", type=float, default=1e-6,
                    help="batched / served legs: FP32 below this bound, inside the FP32 error budget")
    ap.add_argument("--large-no-fp64", action="store_true",
                    help="large leg: skip the FP64 reference build (errors against oracle/_ref rows only)")
    ap.add_argument("--batch-mols", type=int, default=32, help="batched leg: molecules (0 skips the leg)")
    ap.add_argument("--batch-atoms", type=int, nargs=2, default=(3, 8), help="batched leg: atom count range")
    ap.add_argument("--fuse-group", type=int, default=64,
                    help="batched leg: molecules per fused union (the fused regrouping's dense tables grow with "
                         "the square of a union's primitive count)")
    ap.add_argument("--serve-reqs", type=int, default=12, help="served leg: requests per rate (0 skips the leg)")
    ap.add_argument("--serve-atoms", type=int, nargs=2, default=(5, 12), help="served leg: atom count range")
    ap.add_argument("--serve-iters", type=int, default=10, help="served leg: densities per request")
    ap.add_argument("--serve-rates", type=float, nargs="+", default=(0.25, 50.0),
                    help="served leg: Poisson arrival rates (req/s), one run of plain and served per rate")
    # tool modes
    ap.add_argument("--kind", choices=["J", "K"], default="K", help="--mode case: entry-point kind")
    ap.add_argument("--cls", default="pddd", help="--mode case: class")
    ap.add_argument("--atoms", type=int, default=None, help="--mode case / gradient / gradient-cpu: atoms")
    ap.add_argument("--density", type=float, default=30.0, help="--mode gradient: bohr^3 per atom")
    ap.add_argument("--seed", type=int, default=7, help="--mode gradient: molecule seed")
    ap.add_argument("--reps", type=int, default=2, help="--mode case / gradient: repetitions")
    ap.add_argument("--variant", type=int, default=None, help="--mode case: kernel variant (default: tuned)")
    ap.add_argument("--case-fp32-cut", type=float, default=0.0, help="--mode case: mixed-precision cutoff")
    ap.add_argument("--out", default=None, help="--mode classes: JSON output file")
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

        if not dist.is_initialized():
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


# ----------------------------------------------------------------- CPU side (checker and baseline)
def _host_threads():
    try:
        return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    except ValueError:
        return os.cpu_count() or 1


def _ref_classes(rl):
    from vlxb import lists

    classes = [("J", c) for c in lists.j_classes() if c[:2] in rl.jlists and c[2:] in rl.jlists]
    classes += [("K", c) for c in lists.k_classes()
                if c[0] + c[2] in rl.kpairs and c[:2] in rl.kpartners and c[2:] in rl.kpartners]
    return classes


def cpu_reference(rl, budget_s, seed=0):
    """Time the reference's emitted expressions (oracle/_ref) on a bounded
    sample of this build and extrapolate the full-build time.

    Per class: a seeded random sample of bra rows (J) or (i, k) rows (K); each
    sampled row evaluates at most `max_eval` of its passing component quartets;
    the full-build time is (machine throughput in component quartets/s) divided
    into the sampled rows' exact passing counts scaled to all rows."""
    from oracle import ref

    threads = _host_threads()
    rng = np.random.default_rng(seed)
    classes = _ref_classes(rl)
    per = budget_s / len(classes)
    est_total = 0.0
    cq_eval_total = 0
    rows_total = 0
    for kind, cls in classes:
        n = len(rl.jlists[cls[:2]].first) if kind == "J" else len(rl.kpairs[cls[0] + cls[2]].pair_i)
        nrow = min(n, max(threads, 1))
        rows = np.sort(rng.choice(n, size=nrow, replace=False)).astype(np.uint32)
        # grow the per-row evaluation cap until the sample takes a fair share
        # of the class's time budget (or every passing quartet is evaluated),
        # so per-call overhead does not bias the measured throughput
        f = ref.coulomb if kind == "J" else ref.exchange
        cap = 64
        while True:
            t0 = time.perf_counter()
            _, c_pass, c_eval = f(rl, cls, rows=rows, max_eval=cap)
            dt = max(time.perf_counter() - t0, 1e-6)
            if dt >= 0.25 * per or c_eval < cap * nrow or cap >= 2**40:
                break
            cap = int(min(2**40, cap * max(2.0, min(64.0, 0.5 * per / dt))))
        thr = max(c_eval, 1) / dt  # component quartets per second, whole machine
        est_total += (c_pass / nrow) * n / thr
        cq_eval_total += c_eval
        rows_total += nrow
    return est_total, threads, {"classes": len(classes), "rows": rows_total, "component_quartets": cq_eval_total}


def cpu_reference_full(rl):
    """The whole build with the reference's emitted expressions (oracle/_ref,
    OpenMP over the host cores): (mat_J, mat_K, seconds)."""
    from oracle import ref

    matJ = {k: np.zeros(len(v.first)) for k, v in rl.jlists.items()}
    matK = {k: np.zeros(len(v.pair_i)) for k, v in rl.kpairs.items()}
    t0 = time.perf_counter()
    for kind, cls in _ref_classes(rl):
        if kind == "J":
            ref.coulomb(rl, cls, mat_J=matJ[cls[:2]])
        else:
            ref.exchange(rl, cls, mat_K=matK[cls[0] + cls[2]])
    return matJ, matK, time.perf_counter() - t0


def quartets_per_build_ref(rl):
    from oracle import ref

    n = 0
    for kind, cls in _ref_classes(rl):
        n += ref.count_j(rl, cls) if kind == "J" else ref.count_k(rl, cls)
    return n


def ref_rows(rl, per_list, seed=0):
    """FP64 values of seeded rows of every J list (mat_J summed over its 6
    classes) and every K (i, k) list (mat_K over its 9 classes), from the
    reference's emitted expressions (oracle/_ref)."""
    from oracle import ref
    from vlxb import lists

    rng = np.random.default_rng(seed)
    out = {}
    t0 = time.perf_counter()
    for ab, jl in rl.jlists.items():
        n = len(jl.first)
        rows = np.sort(rng.choice(n, size=min(per_list, n), replace=False)).astype(np.uint32)
        acc = np.zeros(n)
        for cd in rl.jlists:
            if lists.LV[cd[0]] <= lists.LV[cd[1]]:
                ref.coulomb(rl, ab + cd, rows=rows, mat_J=acc)
        out[("J", ab)] = (rows.astype(np.int64), acc[rows])
    for ac, kq in rl.kpairs.items():
        n = len(kq.pair_i)
        rows = np.sort(rng.choice(n, size=min(per_list, n), replace=False)).astype(np.uint32)
        acc = np.zeros(n)
        for b in "spd":
            for d in "spd":
                cls = ac[0] + b + ac[1] + d
                if cls[:2] in rl.kpartners and cls[2:] in rl.kpartners:
                    ref.exchange(rl, cls, rows=rows, mat_K=acc)
        out[("K", ac)] = (rows.astype(np.int64), acc[rows])
    return out, time.perf_counter() - t0


def row_errors(expected, matJ, matK):
    """Absolute errors of GPU prim-pair outputs (numpy dicts) on the expected rows."""
    res = {"max_abs_dJ": 0.0, "max_abs_dK": 0.0, "max_abs_J": 0.0, "max_abs_K": 0.0, "rows": 0}
    for (kind, key), (rows, vals) in expected.items():
        got = (matJ if kind == "J" else matK)[key][rows]
        err = float(np.abs(got - vals).max()) if len(rows) else 0.0
        mag = float(np.abs(vals).max()) if len(rows) else 0.0
        res[f"max_abs_d{kind}"] = max(res[f"max_abs_d{kind}"], err)
        res[f"max_abs_{kind}"] = max(res[f"max_abs_{kind}"], mag)
        res["rows"] += len(rows)
    return res


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


# ----------------------------------------------------------------- timing helpers
def timed_device(fn, reps, stream=None, flush=None):
    """Device time (s) of each of `reps` calls of fn, CUDA events on `stream`
    (the current stream when None), with an L2 flush before each when given."""
    import torch

    out = []
    for _ in range(reps):
        if flush is not None:
            flush.zero_()
        s = stream or torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        fn()
        e1.record(s)
        e1.synchronize()
        out.append(e0.elapsed_time(e1) / 1e3)
    return out


def ao_matrices(rl, matJ, matK):
    from vlxb import lists

    J = lists.contract_J(rl, {k: v.cpu().numpy() for k, v in matJ.items()})
    K = lists.contract_K(rl, {k: v.cpu().numpy() for k, v in matK.items()})
    return J, K


# ----------------------------------------------------------------- legs
def run_small(args, L, dev, stream, flush):
    """5-atom 3s2p workload (45 AOs), timed in full: GPU builds through the
    C ABI, the whole build of the reference's emitted expressions on the host
    cores, and every value of every list compared."""
    import torch
    from vlxb import basis, fock, lists

    wl = basis.config_small(0)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn(dev))
    dl = fock.to_device(rl, dev)
    matJ, matK = fock.alloc_outputs(dl)

    def build():
        for t in list(matJ.values()) + list(matK.values()):
            t.zero_()
        fock.build_jk(dl, stream=stream, matJ=matJ, matK=matK)

    with torch.cuda.stream(stream):
        for _ in range(2):
            build()
        torch.cuda.synchronize()
        L.reset_counters(stream.cuda_stream)
        ts = timed_device(build, args.small_steps, stream, flush)
        qj, qk = L.quartet_counters(reset=True, stream=stream.cuda_stream)
    q = (qj + qk) / args.small_steps
    t = float(np.median(ts))
    res = {"workload": "5 atoms 6-bohr cube 3s2p deg 3 (45 AOs), nocc 10, thr 1e-12, FP64",
           "steps": args.small_steps, "ms_per_step": t * 1e3, "quartets_per_build": q, "value": q / t,
           "unit": UNIT, "builds_per_s": 1.0 / t}
    from oracle import ref

    if ref.available():
        rJ, rK, cpu_s = cpu_reference_full(rl)
        gJ = {k: v.cpu().numpy() for k, v in matJ.items()}
        gK = {k: v.cpu().numpy() for k, v in matK.items()}
        dJ = max(float(np.abs(gJ[k] - rJ[k]).max()) for k in rJ)
        dK = max(float(np.abs(gK[k] - rK[k]).max()) for k in rK)
        J, K = lists.contract_J(rl, gJ), lists.contract_K(rl, gK)
        Jr, Kr = lists.contract_J(rl, rJ), lists.contract_K(rl, rK)
        res["parity"] = {"reference": "the reference's emitted expressions (oracle/_ref), every list entry",
                         "max_abs_dJ_pairs": dJ, "max_abs_dK_pairs": dK,
                         "max_abs_dJ_ao": float(np.abs(J - Jr).max()), "max_abs_dK_ao": float(np.abs(K - Kr).max()),
                         "abs_dE_Eh": abs(lists.energy(wl.D, J, K) - lists.energy(wl.D, Jr, Kr)),
                         "max_abs_J": float(np.abs(Jr).max()), "max_abs_K": float(np.abs(Kr).max())}
        res["cpu_reference"] = {"value": q / cpu_s, "unit": UNIT, "build_s": cpu_s, "cores": _host_threads(),
                                "kind": "reference", "sample": "the whole build (not extrapolated)"}
    return res


def run_large(args, L, dev, stream, cut, budget):
    """Large sparse workload: `args.large_atoms` atoms at 25 bohr^3 per atom,
    4s3p2d (5000 Cartesian AOs at 200 atoms).  Lists of the density difference
    dD (seeded, Frobenius norm 1e-3) are built on the device with Schwarz and
    density-weighted screening at 1e-11; the build on dD runs with FP32 below
    `cut` inside the error budget and FP64 accumulation, and is added to the
    previous J/K.  Reported: its device time, quartets, screened fraction
    against the full-density lists, errors against the FP64 build of the same
    dD (AO matrices) and against oracle/_ref on seeded rows, and the quartet
    counts of the reference's screening loops for dD and for the full density."""
    import torch
    from vlxb import basis, devlists, fock, lists

    n = args.large_atoms
    wl = basis.molecule_at_density(n, 25.0, 0, threshold=1e-11)
    rng = np.random.default_rng(3)
    P = rng.standard_normal(wl.D.shape)
    P = 0.5 * (P + P.T)
    dD = P * (1e-3 / np.linalg.norm(P))
    res = {"workload": f"{n} atoms at 25 bohr^3/atom 4s3p2d ({wl.mol.naos} AOs), incremental build on dD "
                       "(|dD|_F = 1e-3), Schwarz + density screening at 1e-11",
           "naos": wl.mol.naos}
    with torch.cuda.stream(stream):
        t0 = time.perf_counter()
        dl = devlists.build_device_lists(wl.mol, dD, 1e-11, dev)
        torch.cuda.synchronize()
        res["list_build_s"] = time.perf_counter() - t0
        res["j_pairs"] = int(sum(v["first"].numel() for v in dl.j.values()))
        res["k_ik_pairs"] = int(sum(v["i"].numel() for v in dl.kpair.values()))
        matJ, matK = fock.alloc_outputs(dl)

        def build():
            for t in list(matJ.values()) + list(matK.values()):
                t.zero_()
            fock.build_jk(dl, stream=stream, matJ=matJ, matK=matK)

        # the kernels are loaded by the builds before this leg (or by the
        # first class calls here), so each build is timed once, cold
        J64 = K64 = None
        t64 = None
        if not args.large_no_fp64:
            L.set_fp32_cut(0.0)
            t64 = timed_device(build, 1, stream)[0]
            J64 = {k: v.cpu().numpy() for k, v in matJ.items()}
            K64 = {k: v.cpu().numpy() for k, v in matK.items()}
        L.set_fp32_cut(cut)
        L.set_fp32_budget(budget)
        L.reset_counters(stream.cuda_stream)
        tmx = timed_device(build, 1, stream)[0]
        qj, qk = L.quartet_counters(reset=True, stream=stream.cuda_stream)
        L.set_fp32_cut(0.0)
        J32 = {k: v.cpu().numpy() for k, v in matJ.items()}
        K32 = {k: v.cpu().numpy() for k, v in matK.items()}
    q = qj + qk
    res.update({"fp64_ms": t64 * 1e3 if t64 else None, "mixed_ms": tmx * 1e3, "quartets": q, "value": q / tmx,
                "unit": UNIT, "builds_per_s": 1.0 / tmx, "speedup_mixed_vs_fp64": t64 / tmx if t64 else None,
                "fp32_below_bound": cut, "fp32_budget": budget})
    host = devlists.to_host(dl, wl.mol)
    if J64 is not None:
        J64a, K64a = lists.contract_J(host, J64), lists.contract_K(host, K64)
        J32a, K32a = lists.contract_J(host, J32), lists.contract_K(host, K32)
        res["mixed_vs_fp64"] = {"max_abs_dJ": float(np.abs(J32a - J64a).max()),
                                "max_abs_dK": float(np.abs(K32a - K64a).max()),
                                "abs_dE_Eh": abs(lists.energy(dD, J32a, K32a) - lists.energy(dD, J64a, K64a))}
    from oracle import ref

    if ref.available() and wl.mol.naos <= 2400:
        # the reference's own screening loops: the quartet count of the dD
        # build (must equal the kernels' counters) and of a full-density build
        # of the same molecule, whose ratio is the screened fraction (host
        # counting time grows past minutes beyond ~2400 AOs, so larger
        # clusters skip it)
        q_ref = quartets_per_build_ref(host)
        with torch.cuda.stream(stream):
            dl0 = devlists.build_device_lists(wl.mol, wl.D, 1e-11, dev)
            torch.cuda.synchronize()
        host0 = devlists.to_host(dl0, wl.mol)
        del dl0
        q_full = quartets_per_build_ref(host0)
        res["screening"] = {"quartets_dD_reference_count": q_ref, "counts_equal": q_ref == q,
                            "quartets_full_density": q_full, "fraction_kept": q / q_full if q_full else None}
    if ref.available() and args.parity_rows > 0:
        exp, secs = ref_rows(host, max(2, args.parity_rows // 2), seed=11)
        if J64 is not None:
            res["parity_fp64"] = row_errors(exp, J64, K64) | {"oracle_s": secs}
        res["parity_mixed"] = row_errors(exp, J32, K32) | {"oracle_s": secs}
    return res


def run_batched(args, L, dev, cut):
    """Batched leg: many small molecules (1 atom per 30 bohr^3, the 4s3p2d
    recipe), all resident.  plain = the molecules' FP64 builds one after the
    other through the C ABI; batched = one CUDA graph replay per iteration (all
    molecules' class calls on 8 capture streams), FP64 and with FP32 below
    `cut`.  Device time with CUDA events; builds/s = molecules/s."""
    import torch
    from vlxb import basis, fock, lists
    from vlxb.batch import BatchedBuilder

    wls = basis.config_batch(args.batch_mols, tuple(args.batch_atoms), 30.0, seed=3)
    L.set_fp32_cut(0.0)
    bb = BatchedBuilder([w.mol for w in wls], [w.D for w in wls], 1e-12, device=dev, streams=8)

    def plain():
        # on the current stream, like the graph replay, so the events below see it
        s = torch.cuda.current_stream(dev)
        for m in bb.members:
            for t in list(m.matJ.values()) + list(m.matK.values()):
                t.zero_()
            fock.build_jk(m.dl, stream=s, matJ=m.matJ, matK=m.matK)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        return min(timed_device(fn, reps))

    def energies():
        out = []
        for t, m in enumerate(bb.members):
            J = lists.contract_J(m.rl, {k: v.cpu().numpy() for k, v in m.matJ.items()})
            K = lists.contract_K(m.rl, {k: v.cpu().numpy() for k, v in m.matK.items()})
            out.append((J, K, lists.energy(wls[t].D, J, K)))
        return out

    t_plain = timed(plain, 2)
    bb.capture()
    q = bb.quartets_per_iteration
    t_b64 = timed(bb.run, 3)
    ref = energies()
    L.set_fp32_cut(cut)
    bb.capture()
    t_bmx = timed(bb.run, 3)
    L.set_fp32_cut(0.0)
    got = energies()
    # fused: one class call per class for each union of up to --fuse-group
    # molecules, one graph per iteration
    from vlxb.batchfuse import FusedBatchGroups

    # the per-molecule graph's memory is no longer needed
    bb.graph = None
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    fb = FusedBatchGroups([w.mol for w in wls], [w.D for w in wls], 1e-12, device=dev, group=args.fuse_group)
    fb.capture()
    t_f64 = timed(fb.run, 3)
    fused_dE = 0.0
    for t, m in enumerate(bb.members):
        fJ, fK = fb.results(t)
        J = lists.contract_J(m.rl, fJ)
        K = lists.contract_K(m.rl, fK)
        fused_dE = max(fused_dE, abs(lists.energy(wls[t].D, J, K) - ref[t][2]))
    L.set_fp32_cut(cut)
    fb.graph = None
    torch.cuda.empty_cache()
    fb.capture()
    t_fmx = timed(fb.run, 3)
    L.set_fp32_cut(0.0)
    n = len(wls)
    atoms = [len(w.mol.coords) for w in wls]
    return {"molecules": n, "atoms": [min(atoms), max(atoms)], "quartets_per_iteration": q,
            "plain_fp64_builds_per_s": n / t_plain, "batched_fp64_builds_per_s": n / t_b64,
            "batched_mixed_builds_per_s": n / t_bmx, "fp32_below_bound": cut,
            "speedup_batched_fp64": t_plain / t_b64, "speedup_batched_mixed": t_plain / t_bmx,
            "fused_fp64_builds_per_s": n / t_f64, "fused_mixed_builds_per_s": n / t_fmx,
            "speedup_fused_fp64": t_plain / t_f64, "speedup_fused_mixed": t_plain / t_fmx,
            "fused_vs_batched_max_abs_dE_Eh": fused_dE, "fused_unions": len(fb.parts),
            "max_abs_dJ": max(float(np.abs(a[0] - b[0]).max()) for a, b in zip(got, ref)),
            "max_abs_dK": max(float(np.abs(a[1] - b[1]).max()) for a, b in zip(got, ref)),
            "max_abs_dE_Eh": max(abs(a[2] - b[2]) for a, b in zip(got, ref)),
            "timing": ("device (CUDA events), best of 2-3 iterations; plain = sequential per-molecule builds; "
                       "batched = every molecule's class calls in one graph on 8 streams; fused = one class "
                       "call per class per union of up to --fuse-group molecules (vlxb_coulombBatch / "
                       "vlxb_exchangeBatch), one graph")}


def run_served(args, L, dev, cut):
    """Served leg: Poisson arrivals, atom counts log-uniform, each request a
    sequence of densities (D0 then D0 + seeded perturbations of norm 1e-2 ..
    1e-6).  Per arrival rate: plain = one request at a time, full FP64
    builds; served = continuous admission of up to 8 concurrent requests on
    their own streams, FP32 below `cut` inside the FP32 error budget,
    incremental dD builds.  Wall-clock (host) timing of the whole request
    stream; p50/p99 = request latency from arrival to result.  One rate sits
    below the plain server's capacity (latency = service time) and one far
    above it (latency dominated by queueing)."""
    from vlxb import basis
    from vlxb.serve import Request, Server, perturbed_densities

    counts = basis.serve_atom_counts(args.serve_reqs, args.serve_atoms[0], args.serve_atoms[1], seed=5)
    wls = [basis.molecule_at_density(int(n), 30.0, 1000 + t) for t, n in enumerate(counts)]

    def reqs(arr):
        out = []
        for t, w in enumerate(wls):
            Ds = perturbed_densities(w.D, args.serve_iters, np.random.default_rng(200 + t))
            out.append(Request(t, w.mol, Ds, w.threshold, arrival=float(arr[t])))
        return out

    Server(device=dev, max_active=1).run(reqs(np.zeros(len(wls)))[:1])  # warm-up (kernel loading)
    keys = ("builds_per_s", "p50_ms", "p99_ms", "wall_s")
    per_rate = []
    err = None
    for rate in args.serve_rates:
        rng = np.random.default_rng(11)
        gaps = rng.exponential(1.0 / rate, size=len(wls))
        arr = np.cumsum(gaps) - gaps[0]
        plain = Server(device=dev, max_active=1).run(reqs(arr))
        fast_reqs = reqs(arr)
        fast = Server(device=dev, max_active=8, fp32_cut=cut, incremental=True).run(fast_reqs)
        per_rate.append({"rate_req_per_s": rate, "plain_fp64": {k: plain[k] for k in keys},
                         "served_mixed_incremental": {k: fast[k] for k in keys},
                         "speedup_builds_per_s": fast["builds_per_s"] / plain["builds_per_s"]})
        if err is None:
            ref_reqs = reqs(arr)
            Server(device=dev, max_active=8).run(ref_reqs)
            err = {"max_abs_dJ_last": max(float(np.abs(a.J - b.J).max()) for a, b in zip(fast_reqs, ref_reqs)),
                   "max_abs_dK_last": max(float(np.abs(a.K - b.K).max()) for a, b in zip(fast_reqs, ref_reqs)),
                   "abs_dE_last_Eh": max(abs(a.energies[-1] - b.energies[-1])
                                         for a, b in zip(fast_reqs, ref_reqs))}
    return {"requests_per_rate": len(wls), "atoms": [int(counts.min()), int(counts.max())],
            "densities_per_request": args.serve_iters, "fp32_below_bound": cut,
            "fp32_budget": L.get_fp32_budget(), "rates": per_rate, **(err or {}),
            "reference": "the same request stream served with full FP64 builds (errors: first rate)",
            "timing": "wall clock of the whole request stream (host-side serving loop included)"}


def run_leg(args):
    """One leg alone (--mode large / batched / served) at the sizes given."""
    import torch
    from vlxb._lib import lib
    from vlxb.tune import DEFAULT_SCHEDULE, apply_schedule

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    L = lib()
    L.init(0)
    apply_schedule(args.schedule or DEFAULT_SCHEDULE)
    if args.fp32_budget is not None:
        L.set_fp32_budget(args.fp32_budget)
    stream = torch.cuda.Stream(device=dev)
    t0 = time.perf_counter()
    if args.mode == "large":
        res = run_large(args, L, dev, stream, args.fp32_cut, L.get_fp32_budget())
    elif args.mode == "batched":
        res = run_batched(args, L, dev, args.pattern_fp32_cut)
    else:
        res = run_served(args, L, dev, args.pattern_fp32_cut)
    res["leg"] = args.mode
    res["wall_s_total"] = time.perf_counter() - t0
    print(json.dumps(res))
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
    budget = args.fp32_budget if args.fp32_budget is not None else L.get_fp32_budget()
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

    # end-to-end step: upload of the step's inputs from pinned host memory,
    # the build, read-back of mat_J / mat_K into pinned host buffers
    hJ = {k: torch.empty(v.numel(), dtype=torch.float64).pin_memory() for k, v in matJ.items()}
    hK = {k: torch.empty(v.numel(), dtype=torch.float64).pin_memory() for k, v in matK.items()}
    h2d = sum(t.numel() * t.element_size() for t in pinned.values())
    d2h = sum(t.numel() * 8 for t in hJ.values()) + sum(t.numel() * 8 for t in hK.values())

    def e2e_build():
        dl2 = fock.upload(rl, pinned, dev, non_blocking=True)
        mJ, mK = fock.alloc_outputs(dl2)
        fock.build_jk(dl2, stream=stream, matJ=mJ, matK=mK)
        for k in mJ:
            hJ[k].copy_(mJ[k], non_blocking=True)
        for k in mK:
            hK[k].copy_(mK[k], non_blocking=True)
        return dl2, mJ, mK

    with torch.cuda.stream(stream):
        # warm-up through the end-to-end path: loads every kernel and warms the
        # caching allocator for the end-to-end leg; the last warm-up step runs
        # with the mixed-precision cutoff, which loads the FP32 pass kernels
        for w in range(args.warmup):
            if w == args.warmup - 1 and args.fp32_cut > 0:
                L.set_fp32_cut(args.fp32_cut)
                L.set_fp32_budget(budget)
            keep = e2e_build()
            torch.cuda.synchronize()
            del keep
            L.set_fp32_cut(0.0)
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
            torch.cuda.nvtx.range_push("timed_step")  # lets ncu capture exactly the timed launches
            one_build()
            torch.cuda.nvtx.range_pop()
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

        # FP64 results of the last timed build: the parity rows and the mixed leg's reference
        G64 = ({k: v.cpu().numpy() for k, v in matJ.items()}, {k: v.cpu().numpy() for k, v in matK.items()})
        J64 = lists.contract_J(rl, G64[0])
        K64 = lists.contract_K(rl, G64[1])

        # ---- end to end: host buffers in, results out, every step
        e2e_steps = args.e2e_steps or min(args.steps, 2)
        e2e_times = []
        for it in range(e2e_steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            keep = e2e_build()
            e1.record(stream)
            e1.synchronize()
            e2e_times.append(e0.elapsed_time(e1) / 1e3)
            del keep
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

        # ---- mixed precision leg: same build with FP32 below the cutoff inside
        # the error budget; errors of AO J, K and E against this GPU's FP64 build
        mixed = None
        G32 = None
        if args.fp32_cut > 0:
            L.set_fp32_cut(args.fp32_cut)
            L.set_fp32_budget(budget)
            mt = []
            for _ in range(args.mixed_steps or min(args.steps, 2)):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                one_build()
                e1.record(stream)
                e1.synchronize()
                mt.append(e0.elapsed_time(e1) / 1e3)
            L.set_fp32_cut(0.0)
            G32 = ({k: v.cpu().numpy() for k, v in matJ.items()}, {k: v.cpu().numpy() for k, v in matK.items()})
            J32 = lists.contract_J(rl, G32[0])
            K32 = lists.contract_K(rl, G32[1])
            t_mix = dist_max(sum(mt)) / len(mt)
            mixed = {"fp32_below_bound": args.fp32_cut, "fp32_budget": budget, "value": qpb / t_mix * ws,
                     "unit": UNIT, "ms_per_step": t_mix * 1e3, "builds_per_s": ws / t_mix,
                     "speedup_vs_fp64": t_build / t_mix,
                     "max_abs_dJ": float(np.abs(J32 - J64).max()), "max_abs_dK": float(np.abs(K32 - K64).max()),
                     "abs_dE_Eh": abs(lists.energy(wl.D, J32, K32) - lists.energy(wl.D, J64, K64)),
                     "reference": ("this GPU's FP64 build, whole AO matrices (its rows are checked against "
                                   "oracle/_ref in `parity`)")}

        # ---- other workloads (rank 0 of a replica run does them alone)
        small = large = batched = served = None
        if rank == 0 and args.small_steps > 0:
            small = run_small(args, L, dev, stream, flush)
        if rank == 0 and args.large_atoms > 0 and args.fp32_cut > 0:
            large = run_large(args, L, dev, stream, args.fp32_cut, budget)
        if rank == 0 and args.batch_mols > 0:
            batched = run_batched(args, L, dev, args.pattern_fp32_cut)
        if rank == 0 and args.serve_reqs > 0:
            served = run_served(args, L, dev, args.pattern_fp32_cut)
        dist_barrier()

    dom = max(per_class, key=lambda r: r[2])
    total_flops = sum(r[4] for r in per_class)
    total_t = sum(r[2] for r in per_class)
    ach_dom = dom[4] / dom[2] / 1e12
    # DRAM bytes of the dominant launch from one ncu capture of this workload
    # (profiles/*_40atom_traffic.md), when the dominant class and its kernel
    # variant are the captured ones
    traffic = None
    tpath = os.path.join(PKG, "vlxb", "traffic_b200.json")
    if os.path.exists(tpath) and args.config == "medium":
        tr = json.load(open(tpath)).get(f"{dom[0]} {dom[1]}")
        if tr and tr.get("variant") == L.get_schedule(dom[0], dom[1]):
            traffic = tr["dram_bytes_read"] + tr["dram_bytes_write"]
    roofline = {"bound": "fp64", "achieved": ach_dom, "peak": peak, "unit": "TFLOP/s", "frac": ach_dom / peak,
                "traffic": traffic, "traffic_unit": "bytes per launch (DRAM read + write, one ncu capture)",
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
        "roofline": roofline, "clocks": clk, "mixed": mixed, "small": small, "large": large,
        "batched": batched, "served": served,
        "schedule": "autotuned (vlxb/schedule_b200.json)" if sched_loaded else "generator defaults",
        "top_classes": [{"class": f"{k} {c.upper()}", "ms": round(t * 1e3, 2), "quartets": n,
                         "tflops": round(f / t / 1e12, 3)} for k, c, t, n, f in
                        sorted(per_class, key=lambda r: -r[2])[:8]],
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        # CPU leg, after every GPU measurement: the reference's emitted
        # expressions as the timed baseline, and as the FP64 checker of seeded
        # rows of the headline build (FP64 and mixed)
        try:
            from oracle import ref

            if ref.available():
                if args.parity_rows > 0:
                    exp, secs = ref_rows(rl, args.parity_rows, seed=5)
                    par = row_errors(exp, *G64)
                    par.update({"reference": "oracle/_ref (the reference's emitted expressions, FP64)",
                                "rows_per_list": args.parity_rows, "oracle_s": secs,
                                "bar_abs": 1e-10})
                    line["parity"] = par
                    if G32 is not None:
                        pm = row_errors(exp, *G32)
                        line["mixed"]["vs_oracle_rows"] = {k: pm[k] for k in ("max_abs_dJ", "max_abs_dK", "rows")}
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


# ----------------------------------------------------------------- tool modes
def _tool_setup():
    import torch
    from vlxb._lib import lib
    from vlxb.tune import apply_schedule

    L = lib()
    L.init(0)
    apply_schedule()
    return torch, L


def mode_case(args):
    """One class entry point on a seeded 4s3p2d cluster (the benchmark's
    recipe and density, side scaled with the atom count): `reps` calls, the
    first a warm-up; prints the time of the last.  A few hundred MB of device
    memory at most: the case for ncu captures."""
    torch, L = _tool_setup()
    from vlxb import basis, fock, lists

    L.set_fp32_cut(args.case_fp32_cut)
    if args.variant is not None:
        L.set_schedule(args.kind, args.cls, args.variant)
    n = args.atoms or 12
    side = 14.0 * (n / 40.0) ** (1.0 / 3.0)
    wl = basis.config_custom(n, side, {0: 4, 1: 3, 2: 2}, 3, 0.05, 2.5, max(2, 2 * n), 1e-12, 0)
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
    return 0


def mode_classes(args):
    """Device time (CUDA events on the calling stream, list regrouping
    included) and screened-in quartets of every class entry point, after one
    warm-up pass."""
    torch, L = _tool_setup()
    from vlxb import fock, lists

    if args.schedule:
        from vlxb.tune import apply_schedule

        apply_schedule(args.schedule)
    wl = workload(args.config)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    dl = fock.to_device(rl)
    matJ, matK = fock.alloc_outputs(dl)
    res = {}
    for rep in range(2):
        for kind, cl in (("J", lists.j_classes()), ("K", lists.k_classes())):
            for cls in cl:
                L.reset_counters()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
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
    for k, (ms, q) in res.items():
        print(k[0], k[1:], f"{ms:.2f} ms", q, flush=True)
    print("total ms", sum(v[0] for v in res.values()))
    if args.out:
        os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
        json.dump(res, open(args.out, "w"), indent=1)
    return 0


def mode_gradient(args):
    """Device time (CUDA events, after one untimed call each) of the FP64 J
    and K builds, dE_J/dR and dE_K/dR (all classes plus the per-atom fold) and
    each exchange-gradient class alone, on one seeded 4s3p2d molecule; one
    JSON line with the times in ms and the translational-invariance residues."""
    torch, L = _tool_setup()
    from vlxb import basis, fock, gradient, lists

    wl = basis.molecule_at_density(args.atoms or 10, args.density, args.seed)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    dl = fock.to_device(rl)
    cg = gradient.CoulombGradient(dl, wl.mol)
    kg = gradient.ExchangeGradient(dl, wl.mol)

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        return [round(t * 1e3, 2) for t in timed_device(fn, args.reps)]

    res = {"workload": wl.name, "naos": wl.mol.naos}
    res["J_build_ms"] = timed(lambda: fock.build_jk(dl, do_k=False))
    res["K_build_ms"] = timed(lambda: fock.build_jk(dl, do_j=False))
    res["dEJ_dR_ms"] = timed(cg.compute)
    res["dEK_dR_ms"] = timed(kg.compute)
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
    return 0


def run_gradient_cpu(args):
    """CPU baseline of the nuclear gradients dE_J/dR and dE_K/dR.  The
    reference has no gradient code, so this times the oracle's derivative
    routines (a port: the Obara-Saika derivative relation on the oracle's
    integrals, all host threads) on the molecule `--mode gradient` times on
    the GPU: per class a seeded sample of bra rows (J) or (i, k) rows (K).
    The sample's time is scaled by the class's screened-in component quartets
    over the sample's (counted with the reference's screening loops in
    oracle/_ref when it is built, else by row count), since screening makes
    the per-row cost very uneven.  Needs no GPU.  Prints one JSON line."""
    from oracle import oracle, ref
    from vlxb import basis, lists

    threads = _host_threads()
    wl = basis.molecule_at_density(args.atoms or 10, 30.0, 7)
    have_ref = ref.available()

    def schwarz(la, lb, pd, P, Q):
        out = np.zeros(len(P))
        ia, ib = pd.info[la], pd.info[lb]
        for t, (p, q) in enumerate(zip(P, Q)):
            A, B = ia[2:5, p], ib[2:5, q]
            I = oracle.eri_shell_quartet(la, lb, la, lb, ia[0, p], A, ib[0, q], B, ia[0, p], A, ib[0, q], B)
            n = I.shape[0] * I.shape[1]
            out[t] = np.sqrt(np.abs(np.diag(I.reshape(n, n))).max())
        return out

    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, ref.schwarz_fn if have_ref else schwarz)
    LVv = lists.LV
    est = {"J": 0.0, "K": 0.0}
    rows_total = {"J": 0, "K": 0}
    spread = {"J": [], "K": []}
    for seed in (11, 12):
        rng = np.random.default_rng(seed)
        tot = {"J": 0.0, "K": 0.0}
        for kind, cls in _ref_classes(rl):
            a, b, c, d = cls
            n = len(rl.jlists[a + b].first) if kind == "J" else len(rl.kpairs[a + c].pair_i)
            rows = np.sort(rng.choice(n, size=min(n, 2 * threads), replace=False)).astype(np.uint32)
            t0 = time.perf_counter()
            if kind == "J":
                jab, jcd = rl.jlists[a + b], rl.jlists[c + d]
                oracle.coulomb_grad(LVv[a], LVv[b], LVv[c], LVv[d], rl.pd.info, rl.pd.count, jcd.D, jab.Q, jcd.Q,
                                    jab.first, jab.second, jab.pdata, jcd.first, jcd.second, jcd.pdata,
                                    rl.threshold, rows=rows)
            else:
                kq, p1, p2 = rl.kpairs[a + c], rl.kpartners[a + b], rl.kpartners[c + d]
                oracle.exchange_grad(LVv[a], LVv[b], LVv[c], LVv[d], kq.pair_i, kq.pair_k, rl.pd.info,
                                     rl.pd.aoinds, rl.pd.count, rl.maxD[b + d], rl.D_AO, p1.Q, p2.Q, p1.Dinds,
                                     p2.Dinds, p1.displs, p2.displs, p1.counts, p2.counts, p1.pdata, p2.pdata,
                                     0.0, rl.threshold, rows=rows)
            dt = time.perf_counter() - t0
            scale = n / len(rows)
            if have_ref:
                f = ref.coulomb if kind == "J" else ref.exchange
                _, c_rows, _ = f(rl, cls, rows=rows, max_eval=0)
                _, c_all, _ = f(rl, cls, max_eval=0)
                scale = c_all / c_rows if c_rows else scale
            tot[kind] += dt * scale
            if seed == 11:
                rows_total[kind] += len(rows)
        for k in ("J", "K"):
            spread[k].append(tot[k])
    for k in ("J", "K"):
        est[k] = float(np.mean(spread[k]))
    print(json.dumps({"metric": "nuclear-gradient time, CPU port (oracle)", "unit": "s",
                      "workload": wl.name, "naos": wl.mol.naos, "dEJ_dR_s": round(est["J"], 2),
                      "dEK_dR_s": round(est["K"], 2),
                      "two_seeds_s": {k: [round(v, 1) for v in spread[k]] for k in spread},
                      "cores": threads, "kind": "port",
                      "sample": (f"{rows_total['J']} J bra rows and {rows_total['K']} K (i, k) rows per seed "
                                 "(2 x threads per class), scaled per class by screened-in component quartets "
                                 f"({'oracle/_ref counts' if have_ref else 'row count'}); mean of two seeds")}))
    return 0


def main():
    args = parse()
    if args.mode == "gradient-cpu":
        return run_gradient_cpu(args)
    if args.mode == "case":
        return mode_case(args)
    if args.mode == "classes":
        return mode_classes(args)
    if args.mode == "gradient":
        return mode_gradient(args)
    if args.mode in ("large", "batched", "served"):
        return run_leg(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
