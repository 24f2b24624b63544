"""Fock-build serving loop with continuous admission.

A request is one molecule plus a sequence of densities (SCF-like updates).
The server admits queued requests whenever a slot and device memory are free
(budgeted on the request's resident lists and outputs), keeps each admitted
request's lists resident for all of its iterations, and runs every admitted
request on its own CUDA stream, so requests that arrive while others are on
the GPU are started as soon as capacity frees up and their kernels overlap on
the device.  Host-side list building of newly admitted requests runs on a
worker thread while the GPU works.

Iterations after the first can be incremental: the build runs on
dD = D_i - D_{i-1} (J and K are linear in D; small dD screens away part of
the quartets) and is added to the previous J/K in FP64.

J and K stay on the device: the prim-pair outputs are contracted to AO
matrices by vlxb_pairsToAO, incremental updates are added there, and only
the energy terms (vlxb_fockEnergy, three doubles) are read back per build;
the AO J and K of a request are copied to the host once, when it finishes.
With device_lists (the default) the lists themselves are built on the GPU at
admission (vlxb.devlists) and refreshed there for every new density, so the
host only uploads each density and reads back three doubles per build.

Results are deterministic: the kernels have no atomics on J/K, so a request
gives the same J/K alone and in any mix (tested).
"""
from __future__ import annotations

import concurrent.futures as cf
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import aomap, devlists, fock, lists
from ._lib import lib


@dataclass
class Request:
    rid: int
    mol: object
    densities: list                   # AO densities, one build per entry
    threshold: float = 1e-12
    arrival: float = 0.0              # seconds after the server start
    # filled by the server
    admitted: float = None
    finished: float = None
    energies: list = field(default_factory=list)
    J: np.ndarray = None
    K: np.ndarray = None


def perturbed_densities(D0: np.ndarray, n: int, rng: np.random.Generator, hi: float = 1e-2, lo: float = 1e-6):
    """D0 followed by n-1 densities D0 + P_i with seeded symmetric P_i of
    Frobenius norm log-spaced from hi down to lo."""
    out = [D0]
    for eps in np.logspace(math.log10(hi), math.log10(lo), n - 1):
        P = rng.standard_normal(D0.shape)
        P = 0.5 * (P + P.T)
        out.append(D0 + P * (eps / np.linalg.norm(P)))
    return out


class _Active:
    def __init__(self, req, rl, dl, stream, incremental):
        self.req = req
        self.rl = rl          # host lists, or None when the lists live on the device only
        self.dl = dl
        self.stream = stream
        self.incremental = incremental
        self.it = 0
        self.prevD = None
        n = dl.naos
        with torch.cuda.stream(stream):
            self.am = aomap.AOMap(rl, dl.device) if rl is not None else aomap.AOMap.from_device(dl)
            self.prevDdev = torch.zeros((n, n), dtype=torch.float64, device=dl.device)
            self.useDdev = torch.empty_like(self.prevDdev)
            self.flatJ, self.matJ, self.flatK, self.matK = self.am.alloc_outputs()
            self.J = torch.zeros((n, n), dtype=torch.float64, device=dl.device)   # running AO J
            self.K = torch.zeros((n, n), dtype=torch.float64, device=dl.device)
            self.dJ = torch.empty_like(self.J)
            self.dK = torch.empty_like(self.K)
            self.Ddev = torch.empty_like(self.J)
            self.e_dev = torch.empty(3, dtype=torch.float64, device=dl.device)
        self.e_host = torch.empty(3, dtype=torch.float64).pin_memory()
        self.pending = None  # (event, density used)
        self.bytes = dl.nbytes() + self.am.nbytes() + 6 * n * n * 8


class Server:
    def __init__(self, budget_bytes: float = 120e9, max_active: int = 16, device="cuda", fp32_cut: float = 0.0,
                 incremental: bool = False, prep_workers: int = 2, device_lists: bool = True):
        self.budget = float(budget_bytes)
        self.max_active = max_active
        self.device = torch.device(device)
        self.L = lib()
        self.L.init(self.device.index or 0)
        self.fp32_cut = fp32_cut
        self.incremental = incremental
        self.device_lists = device_lists
        self.pool = cf.ThreadPoolExecutor(max_workers=prep_workers)
        self.schwarz = fock.gpu_schwarz_fn(self.device)

    def _prepare(self, req):
        if self.device_lists:
            return None  # built on the GPU at admission
        return lists.build_lists(req.mol, req.densities[0], req.threshold, self.schwarz)

    @staticmethod
    def _set_density(rl, dl, D):
        rl.D_AO = np.ascontiguousarray(D)
        for key in list(rl.maxD):
            b, d = key
            blk = D[np.ix_(rl.pd.aoinds[lists.LV[b]].ravel(), rl.pd.aoinds[lists.LV[d]].ravel())]
            rl.maxD[key] = float(np.abs(blk).max())
        dl.maxD = dict(rl.maxD)
        for key, jl in rl.jlists.items():
            la, lb = lists.LV[key[0]], lists.LV[key[1]]
            na, nb = lists.NCART[la], lists.NCART[lb]
            ai = rl.pd.aoinds[la][jl.first % na, jl.first // na]
            bj = rl.pd.aoinds[lb][jl.second % nb, jl.second // nb]
            jl.D = D[ai, bj].copy()
            dl.j[key]["D"].copy_(torch.from_numpy(jl.D), non_blocking=False)
        dl.D_AO.copy_(torch.from_numpy(rl.D_AO))

    def _launch(self, a: _Active):
        """Queue iteration a.it of an active request on its stream: the build
        (on D, or on dD after the first iteration in incremental mode), the AO
        contraction on the device, the energy of the running J/K with D, and
        its read-back."""
        D = a.req.densities[a.it]
        inc = a.incremental and a.prevD is not None
        with torch.cuda.stream(a.stream):
            a.Ddev.copy_(torch.from_numpy(np.ascontiguousarray(D)))
            if a.rl is None:
                if inc:
                    torch.sub(a.Ddev, a.prevDdev, out=a.useDdev)
                    devlists.set_density(a.dl, a.useDdev, stream=a.stream)
                else:
                    devlists.set_density(a.dl, a.Ddev, stream=a.stream)
                a.prevDdev.copy_(a.Ddev)
            else:
                self._set_density(a.rl, a.dl, D - a.prevD if inc else D)
            a.flatJ.zero_()
            a.flatK.zero_()
            fock.build_jk(a.dl, stream=a.stream, matJ=a.matJ, matK=a.matK)
            if inc:
                a.am.to_ao("J", a.flatJ, out=a.dJ, stream=a.stream)
                a.am.to_ao("K", a.flatK, out=a.dK, stream=a.stream)
                a.J.add_(a.dJ)
                a.K.add_(a.dK)
            else:
                a.am.to_ao("J", a.flatJ, out=a.J, stream=a.stream)
                a.am.to_ao("K", a.flatK, out=a.K, stream=a.stream)
            aomap.energy(a.Ddev, a.J, a.K, out=a.e_dev, stream=a.stream)
            a.e_host.copy_(a.e_dev, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(a.stream)
        a.pending = (ev, D)

    def _collect(self, a: _Active):
        _, D = a.pending
        a.req.energies.append(float(a.e_host[0]))
        a.prevD = D
        a.pending = None
        a.it += 1

    def run(self, requests, poll: float = 2e-4):
        """Serve `requests` (arrival times relative to now); returns stats."""
        self.L.set_fp32_cut(self.fp32_cut)
        t0 = time.perf_counter()
        queue = sorted(requests, key=lambda r: r.arrival)
        qi = 0
        preparing = {}
        active = []
        resident = 0.0
        done = []
        builds = 0
        try:
            while len(done) < len(requests):
                now = time.perf_counter() - t0
                # start host preparation of arrived requests (FIFO)
                while qi < len(queue) and queue[qi].arrival <= now:
                    r = queue[qi]
                    preparing[r.rid] = (r, self.pool.submit(self._prepare, r))
                    qi += 1
                # admit prepared requests while slots and memory allow
                for rid in sorted(preparing, key=lambda k: preparing[k][0].arrival):
                    r, fut = preparing[rid]
                    if not fut.done() or len(active) >= self.max_active:
                        continue
                    rl = fut.result()
                    if rl is not None:
                        est = 1.5 * sum(x.nbytes for x in fock.host_arrays(rl).values())
                    else:  # bound on the device lists: all primitive pairs of all type pairs
                        n = r.mol.naos
                        est = 8.0 * 64 * n * n
                    if resident + est > self.budget and active:
                        continue
                    st = torch.cuda.Stream(device=self.device)
                    if rl is not None:
                        dl = fock.to_device(rl, self.device)
                    else:
                        with torch.cuda.stream(st):
                            dl = devlists.build_device_lists(r.mol, r.densities[0], r.threshold, self.device)
                    a = _Active(r, rl, dl, st, self.incremental)
                    r.admitted = time.perf_counter() - t0
                    resident += a.bytes
                    active.append(a)
                    del preparing[rid]
                # progress active requests
                busy = False
                for a in list(active):
                    if a.pending is not None:
                        if a.pending[0].query():
                            self._collect(a)
                            builds += 1
                        else:
                            busy = True
                            continue
                    if a.it < len(a.req.densities):
                        self._launch(a)
                        busy = True
                    else:
                        a.req.finished = time.perf_counter() - t0
                        a.req.J, a.req.K = a.J.cpu().numpy(), a.K.cpu().numpy()
                        resident -= a.bytes
                        active.remove(a)
                        done.append(a.req)
                if not busy and not preparing:
                    time.sleep(poll)
        finally:
            self.L.set_fp32_cut(0.0)
        wall = time.perf_counter() - t0
        lat = np.array([r.finished - r.arrival for r in done])
        return {"requests": len(done), "builds": builds, "wall_s": wall, "builds_per_s": builds / wall,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "max_active": self.max_active, "budget_bytes": self.budget}
