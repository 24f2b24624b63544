"""Batched J/K builds of many independent molecules, one CUDA graph per iteration.

Every molecule keeps its reference-format lists resident on the device
(`DeviceLists`).  One iteration = the 36 Coulomb and 54 exchange class calls of
every molecule.  All of them are captured once into a single CUDA graph: the
molecules are spread round-robin over `streams` capture streams forked from
and joined back into the capture origin, so their kernels are independent
graph branches that run concurrently and fill the GPU (a 3-atom molecule's
class kernel alone would occupy a few SMs).  Each replay is one
cudaGraphLaunch; scratch inside the graph comes from graph memory nodes
(cudaMallocAsync under capture).  The mat_J / mat_K outputs are zeroed inside
the graph, so a replay is a complete build.

Densities are read from the resident list arrays, so a new density is a copy
into those arrays followed by a replay.  The K screen uses each molecule's
max |D| per shell-type block, which the graph holds as a kernel argument: a
new density must not raise it (`set_density` checks this and re-captures when
it does).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import fock, lists
from ._lib import lib


@dataclass
class Member:
    rl: lists.ReferenceLists
    dl: fock.DeviceLists
    matJ: dict
    matK: dict


class BatchedBuilder:
    def __init__(self, molecules, densities, threshold: float, device="cuda", streams: int = 8,
                 omega: float = 0.0, schwarz_fn=None):
        self.device = torch.device(device)
        self.omega = omega
        self.L = lib()
        self.L.init(self.device.index or 0)
        sfn = schwarz_fn or fock.gpu_schwarz_fn(self.device)
        self.members = []
        for mol, D in zip(molecules, densities):
            rl = lists.build_lists(mol, D, threshold, sfn)
            dl = fock.to_device(rl, self.device)
            mJ, mK = fock.alloc_outputs(dl)
            self.members.append(Member(rl, dl, mJ, mK))
        self.nstreams = max(1, streams)
        self.graph = None
        self.quartets_per_iteration = None

    # ------------------------------------------------------------ capture
    def _issue(self, streams):
        for t in range(len(self.members)):
            m = self.members[t]
            s = streams[t % len(streams)]
            with torch.cuda.stream(s):
                for v in m.matJ.values():
                    v.zero_()
                for v in m.matK.values():
                    v.zero_()
                fock.build_jk(m.dl, stream=s, omega=self.omega, matJ=m.matJ, matK=m.matK)

    def capture(self):
        """(Re)capture the iteration graph; an eager run first warms every path."""
        side = [torch.cuda.Stream(device=self.device) for _ in range(self.nstreams)]
        origin = torch.cuda.Stream(device=self.device)
        # eager warm-up (first-use set-up must not happen under capture)
        self._issue(side)
        torch.cuda.synchronize(self.device)
        self.L.reset_counters()
        self._issue(side)
        torch.cuda.synchronize(self.device)
        qj, qk = self.L.quartet_counters(reset=True)
        self.quartets_per_iteration = qj + qk
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=origin):
            fork = torch.cuda.Event()
            fork.record(origin)
            for s in side:
                s.wait_event(fork)
            self._issue(side)
            for s in side:
                ev = torch.cuda.Event()
                ev.record(s)
                origin.wait_event(ev)
        self.graph = g
        self._origin = origin

    def run(self):
        """One batched iteration (asynchronous on the capture origin stream)."""
        if self.graph is None:
            self.capture()
        self.graph.replay()

    def synchronize(self):
        torch.cuda.synchronize(self.device)

    # ------------------------------------------------------------ densities
    def set_density(self, t: int, D: np.ndarray):
        """New AO density of member t: updates its resident pair densities and
        AO density in place; re-captures if a block max |D| grew."""
        m = self.members[t]
        rl, dl = m.rl, m.dl
        rl.D_AO = np.ascontiguousarray(D)
        regrow = False
        for key in list(rl.maxD):
            b, d = key
            lb, ld = lists.LV[b], lists.LV[d]
            blk = D[np.ix_(rl.pd.aoinds[lb].ravel(), rl.pd.aoinds[ld].ravel())]
            new = float(np.abs(blk).max())
            if new > rl.maxD[key]:
                rl.maxD[key] = new
                dl.maxD[key] = new
                regrow = True
        for key, jl in rl.jlists.items():
            la, lb = lists.LV[key[0]], lists.LV[key[1]]
            na, nb = lists.NCART[la], lists.NCART[lb]
            ai = rl.pd.aoinds[la][jl.first % na, jl.first // na]
            bj = rl.pd.aoinds[lb][jl.second % nb, jl.second // nb]
            jl.D = D[ai, bj].copy()
            dl.j[key]["D"].copy_(torch.from_numpy(jl.D))
        dl.D_AO.copy_(torch.from_numpy(rl.D_AO))
        if regrow:
            self.graph = None

    # ------------------------------------------------------------ results
    def results(self, t: int):
        """(mat_J, mat_K) of member t as numpy dicts (synchronises)."""
        m = self.members[t]
        self.synchronize()
        return ({k: v.cpu().numpy() for k, v in m.matJ.items()}, {k: v.cpu().numpy() for k, v in m.matK.items()})

    def resident_bytes(self) -> int:
        return sum(m.dl.nbytes() for m in self.members)
