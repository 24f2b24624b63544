"""Fused batches: one class call per class for many molecules.

`batch.BatchedBuilder` replays every molecule's 90 class calls inside one
CUDA graph.  `FusedBatch` instead concatenates the molecules' reference-format
lists into one union (primitives of each type numbered molecule after
molecule, no pair across two molecules) and runs each class ONCE for the whole
batch through `vlxb_coulombBatch` / `vlxb_exchangeBatch`: one device-side
regrouping and one persistent kernel launch (two with FP32 below a cutoff)
per class per iteration, whatever the number of molecules.

Molecule boundaries reach the kernels as data: a Coulomb bra only meets the
kets of its own molecule (per-molecule ket segments sorted by bound), and an
exchange output block is screened with its own molecule's max |D|.  The
exchange density is a stack of the molecules' AO density blocks (rows in the
union AO numbering, columns local, row stride = the largest molecule), so the
memory is sum(n_m) * max(n_m), not (sum n_m)^2.  Each molecule's J and K are
its slices of the union outputs and equal the molecule's own class calls
(tested).  One iteration can be captured into a CUDA graph (`capture`).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import fock, lists
from ._lib import lib
from .lists import ANG, LV, NCART


class VlxbBatchCall(ctypes.Structure):
    """Mirror of VlxbBatchCall in include/vlxb.h."""
    _fields_ = [
        ("mat", ctypes.c_void_p),
        ("prim_info", ctypes.c_void_p * 3),
        ("prim_aoinds", ctypes.c_void_p * 3),
        ("prim_aocols", ctypes.c_void_p * 3),
        ("prim_count", ctypes.c_uint32 * 3),
        ("prim_mol", ctypes.c_void_p * 3),
        ("n_mol", ctypes.c_int32),
        ("ab_Q", ctypes.c_void_p), ("cd_Q", ctypes.c_void_p), ("cd_D", ctypes.c_void_p),
        ("ab_pdata", ctypes.c_void_p), ("cd_pdata", ctypes.c_void_p),
        ("ab_first", ctypes.c_void_p), ("ab_second", ctypes.c_void_p),
        ("cd_first", ctypes.c_void_p), ("cd_second", ctypes.c_void_p),
        ("n_ab", ctypes.c_uint32), ("n_cd", ctypes.c_uint32),
        ("pair_i", ctypes.c_void_p), ("pair_k", ctypes.c_void_p),
        ("n_ik", ctypes.c_uint32),
        ("D", ctypes.c_void_p),
        ("D_stride", ctypes.c_uint32),
        ("naos", ctypes.c_uint32),
        ("maxD_mol", ctypes.c_void_p),
        ("Q_ab", ctypes.c_void_p), ("Q_cd", ctypes.c_void_p),
        ("pdata_ab", ctypes.c_void_p), ("pdata_cd", ctypes.c_void_p),
        ("Dinds_ab", ctypes.c_void_p), ("Dinds_cd", ctypes.c_void_p),
        ("displs_ab", ctypes.c_void_p), ("displs_cd", ctypes.c_void_p),
        ("counts_ab", ctypes.c_void_p), ("counts_cd", ctypes.c_void_p),
        ("omega", ctypes.c_double),
        ("thr", ctypes.c_double),
    ]


def _i32(a):
    return np.ascontiguousarray(np.asarray(a).astype(np.int64).astype(np.uint32).view(np.int32))


def union_lists(rls) -> dict:
    """The union of per-molecule reference-format lists (pure numpy): primitive
    tables per type concatenated molecule after molecule, list indices shifted
    by the molecule's primitive offsets, the density stack and the
    per-molecule max-|D| bounds.  Returns the arrays (name -> numpy) and the
    layout (per-molecule slices of the J and K output lists)."""
    nm = len(rls)
    naos_m = np.array([rl.naos for rl in rls], dtype=np.int64)
    ao0 = np.concatenate([[0], np.cumsum(naos_m)]).astype(np.int64)
    naos, W = int(ao0[-1]), int(naos_m.max())
    cnt = {l: np.array([rl.pd.count[l] for rl in rls], dtype=np.int64) for l in range(3)}
    poff = {l: np.concatenate([[0], np.cumsum(cnt[l])]).astype(np.int64) for l in range(3)}
    count = {l: int(poff[l][-1]) for l in range(3)}
    h = {}
    for l in range(3):
        if count[l] == 0:
            continue
        h[f"info{l}"] = np.concatenate([rl.pd.info[l] for rl in rls if rl.pd.count[l]], axis=1)
        h[f"row{l}"] = _i32(np.concatenate([rl.pd.aoinds[l].astype(np.int64) + ao0[m]
                                            for m, rl in enumerate(rls) if rl.pd.count[l]], axis=1))
        h[f"col{l}"] = _i32(np.concatenate([rl.pd.aoinds[l] for rl in rls if rl.pd.count[l]], axis=1))
        h[f"mol{l}"] = np.concatenate([np.full(cnt[l][m], m, dtype=np.int32) for m in range(nm)])
    jkeys = sorted({k for rl in rls for k in rl.jlists})
    jslices = {}
    for key in jkeys:
        la, lb = LV[key[0]], LV[key[1]]
        parts = {n: [] for n in ("first", "second", "pdata", "Q", "D")}
        off, sl = 0, []
        for m, rl in enumerate(rls):
            jl = rl.jlists.get(key)
            n = 0 if jl is None else len(jl.first)
            sl.append((off, off + n))
            off += n
            if n:
                parts["first"].append(jl.first.astype(np.int64) + poff[la][m] * NCART[la])
                parts["second"].append(jl.second.astype(np.int64) + poff[lb][m] * NCART[lb])
                for nme in ("pdata", "Q", "D"):
                    parts[nme].append(getattr(jl, nme))
        jslices[key] = sl
        h[f"j_{key}_first"] = _i32(np.concatenate(parts["first"]))
        h[f"j_{key}_second"] = _i32(np.concatenate(parts["second"]))
        for nme in ("pdata", "Q", "D"):
            h[f"j_{key}_{nme}"] = np.concatenate(parts[nme])
    kpkeys = sorted({k for rl in rls for k in rl.kpartners})
    for key in kpkeys:
        la, lb = LV[key[0]], LV[key[1]]
        counts, dinds, Q, pdata = [], [], [], []
        for m, rl in enumerate(rls):
            kp = rl.kpartners.get(key)
            if kp is None:
                counts.append(np.zeros(rl.pd.count[la] * NCART[la], dtype=np.int64))
                continue
            counts.append(kp.counts.astype(np.int64))
            dinds.append(kp.Dinds.astype(np.int64) + poff[lb][m] * NCART[lb])
            Q.append(kp.Q)
            pdata.append(kp.pdata)
        c = np.concatenate(counts)
        d = np.zeros(len(c), dtype=np.int64)
        d[1:] = np.cumsum(c[:-1])
        h[f"kp_{key}_counts"], h[f"kp_{key}_displs"] = _i32(c), _i32(d)
        h[f"kp_{key}_Dinds"] = _i32(np.concatenate(dinds)) if dinds else np.zeros(0, np.int32)
        h[f"kp_{key}_Q"] = np.concatenate(Q) if Q else np.zeros(0)
        h[f"kp_{key}_pdata"] = np.concatenate(pdata) if pdata else np.zeros(0)
    kkeys = sorted({k for rl in rls for k in rl.kpairs})
    kslices = {}
    for key in kkeys:
        la, lc = LV[key[0]], LV[key[1]]
        ii, kk, off, sl = [], [], 0, []
        for m, rl in enumerate(rls):
            kq = rl.kpairs.get(key)
            n = 0 if kq is None else len(kq.pair_i)
            sl.append((off, off + n))
            off += n
            if n:
                ii.append(kq.pair_i.astype(np.int64) + poff[la][m] * NCART[la])
                kk.append(kq.pair_k.astype(np.int64) + poff[lc][m] * NCART[lc])
        kslices[key] = sl
        h[f"kq_{key}_i"] = _i32(np.concatenate(ii)) if ii else np.zeros(0, np.int32)
        h[f"kq_{key}_k"] = _i32(np.concatenate(kk)) if kk else np.zeros(0, np.int32)
    Dst = np.zeros((naos, W))
    for m, rl in enumerate(rls):
        Dst[ao0[m]:ao0[m] + rl.naos, :rl.naos] = rl.D_AO
    h["Dstack"] = Dst
    maxD_keys = sorted({k for rl in rls for k in rl.maxD})
    for key in maxD_keys:
        h[f"maxD_{key}"] = np.array([rl.maxD.get(key, 0.0) for rl in rls])
    return {"naos_m": naos_m, "ao0": ao0, "naos": naos, "W": W, "count": count, "poff": poff,
            "jkeys": jkeys, "jslices": jslices, "kpkeys": kpkeys, "kkeys": kkeys, "kslices": kslices,
            "maxD_keys": maxD_keys, "arrays": h}


class FusedBatch:
    def __init__(self, molecules, densities, threshold: float, device="cuda", schwarz_fn=None, omega: float = 0.0):
        self.device = torch.device(device)
        self.L = lib()
        self.L.init(self.device.index or 0)
        self.threshold = threshold
        self.omega = omega
        sfn = schwarz_fn or fock.gpu_schwarz_fn(self.device)
        self.rls = [lists.build_lists(m, D, threshold, sfn) for m, D in zip(molecules, densities)]
        self.nmol = len(self.rls)
        self._build_union()
        self.graph = None

    # ------------------------------------------------------------ union lists
    def _build_union(self):
        u = union_lists(self.rls)
        for k in ("naos_m", "ao0", "naos", "W", "count", "jkeys", "jslices", "kpkeys", "kkeys", "kslices",
                  "maxD_keys"):
            setattr(self, k, u[k])
        dev = self.device
        self.d = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in u["arrays"].items()}
        self.matJ = {k: torch.zeros(self.d[f"j_{k}_first"].numel(), dtype=torch.float64, device=dev)
                     for k in self.jkeys}
        self.matK = {k: torch.zeros(self.d[f"kq_{k}_i"].numel(), dtype=torch.float64, device=dev)
                     for k in self.kkeys}

    def nbytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in self.d.values())

    # ------------------------------------------------------------ calls
    def _base(self, mat):
        c = VlxbBatchCall()
        c.mat = mat.data_ptr()
        for l in range(3):
            if self.count[l]:
                c.prim_info[l] = self.d[f"info{l}"].data_ptr()
                c.prim_aoinds[l] = self.d[f"row{l}"].data_ptr()
                c.prim_aocols[l] = self.d[f"col{l}"].data_ptr()
                c.prim_count[l] = self.count[l]
                c.prim_mol[l] = self.d[f"mol{l}"].data_ptr()
        c.n_mol = self.nmol
        c.thr = self.threshold
        c.omega = self.omega
        return c

    def _coulomb(self, cls, stream):
        ab, cd = cls[:2], cls[2:]
        if ab not in self.jkeys or cd not in self.jkeys:
            return
        c = self._base(self.matJ[ab])
        d = self.d
        c.ab_Q, c.cd_Q, c.cd_D = d[f"j_{ab}_Q"].data_ptr(), d[f"j_{cd}_Q"].data_ptr(), d[f"j_{cd}_D"].data_ptr()
        c.ab_pdata, c.cd_pdata = d[f"j_{ab}_pdata"].data_ptr(), d[f"j_{cd}_pdata"].data_ptr()
        c.ab_first, c.ab_second = d[f"j_{ab}_first"].data_ptr(), d[f"j_{ab}_second"].data_ptr()
        c.cd_first, c.cd_second = d[f"j_{cd}_first"].data_ptr(), d[f"j_{cd}_second"].data_ptr()
        c.n_ab, c.n_cd = d[f"j_{ab}_first"].numel(), d[f"j_{cd}_first"].numel()
        l4 = [LV[x] for x in cls]
        self.L.check(self.L.cdll.vlxb_coulombBatch(*l4, ctypes.byref(c), stream), f"vlxb_coulombBatch {cls}")

    def _exchange(self, cls, stream):
        a, b, cc, dd = cls
        ac, ab, cd = a + cc, a + b, cc + dd
        if ac not in self.kkeys or ab not in self.kpkeys or cd not in self.kpkeys:
            return
        c = self._base(self.matK[ac])
        d = self.d
        c.pair_i, c.pair_k = d[f"kq_{ac}_i"].data_ptr(), d[f"kq_{ac}_k"].data_ptr()
        c.n_ik = d[f"kq_{ac}_i"].numel()
        c.D, c.D_stride, c.naos = d["Dstack"].data_ptr(), self.W, self.naos
        c.maxD_mol = d[f"maxD_{b}{dd}"].data_ptr()
        for side, key in (("ab", ab), ("cd", cd)):
            setattr(c, f"Q_{side}", d[f"kp_{key}_Q"].data_ptr())
            setattr(c, f"pdata_{side}", d[f"kp_{key}_pdata"].data_ptr())
            setattr(c, f"Dinds_{side}", d[f"kp_{key}_Dinds"].data_ptr())
            setattr(c, f"displs_{side}", d[f"kp_{key}_displs"].data_ptr())
            setattr(c, f"counts_{side}", d[f"kp_{key}_counts"].data_ptr())
        l4 = [LV[x] for x in cls]
        self.L.check(self.L.cdll.vlxb_exchangeBatch(*l4, ctypes.byref(c), stream), f"vlxb_exchangeBatch {cls}")

    def issue(self, stream=None):
        """Zero the outputs and queue one batched iteration (90 class calls)."""
        st = stream or torch.cuda.current_stream(self.device)
        with torch.cuda.stream(st):
            for t in list(self.matJ.values()) + list(self.matK.values()):
                t.zero_()
            for cls in lists.j_classes():
                self._coulomb(cls, st.cuda_stream)
            for cls in lists.k_classes():
                self._exchange(cls, st.cuda_stream)

    def capture(self):
        """Capture one iteration into a CUDA graph (after an eager warm-up)."""
        s = torch.cuda.Stream(device=self.device)
        self.issue(s)
        torch.cuda.synchronize(self.device)
        self.L.reset_counters()
        self.issue(s)
        torch.cuda.synchronize(self.device)
        qj, qk = self.L.quartet_counters(reset=True)
        self.quartets_per_iteration = qj + qk
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self.issue(s)
        self.graph = g

    def run(self):
        if self.graph is None:
            self.issue()
        else:
            self.graph.replay()

    # ------------------------------------------------------------ densities / results
    def set_density(self, m: int, D: np.ndarray):
        """New AO density of molecule m: its J lists' densities, its block of
        the density stack and its max-|D| bounds (read by the kernels from
        device memory, so a captured graph stays valid)."""
        rl = self.rls[m]
        rl.D_AO = np.ascontiguousarray(D)
        for key, jl in rl.jlists.items():
            la, lb = LV[key[0]], LV[key[1]]
            ai = rl.pd.aoinds[la][jl.first % NCART[la], jl.first // NCART[la]]
            bj = rl.pd.aoinds[lb][jl.second % NCART[lb], jl.second // NCART[lb]]
            jl.D = D[ai, bj].copy()
            s0, s1 = self.jslices[key][m]
            self.d[f"j_{key}_D"][s0:s1].copy_(torch.from_numpy(jl.D))
        n = rl.naos
        self.d["Dstack"][int(self.ao0[m]):int(self.ao0[m]) + n, :n].copy_(torch.from_numpy(rl.D_AO))
        for key in self.maxD_keys:
            if key in rl.maxD:
                b, d = key
                blk = D[np.ix_(rl.pd.aoinds[LV[b]].ravel(), rl.pd.aoinds[LV[d]].ravel())]
                rl.maxD[key] = float(np.abs(blk).max())
                self.d[f"maxD_{key}"][m] = rl.maxD[key]

    def results(self, m: int):
        """(mat_J, mat_K) of molecule m as numpy dicts in its own list layout."""
        torch.cuda.synchronize(self.device)
        rl = self.rls[m]
        J = {k: self.matJ[k][slice(*self.jslices[k][m])].cpu().numpy() for k in rl.jlists}
        K = {k: self.matK[k][slice(*self.kslices[k][m])].cpu().numpy() for k in rl.kpairs}
        return J, K


class FusedBatchGroups:
    """A large batch as several fused unions of at most `group` molecules,
    issued together (one graph for all of them with `capture`).

    The device-side regrouping of a class call builds dense occupancy tables
    over (first shell, second shell) of the call's primitives, whose size is
    the product of the union's primitive counts: with 256 molecules of 3-8
    atoms one union needs tables of about 1 GB per type pair and per class
    call, and the whole iteration ran out of device memory.  Unions of 64
    molecules keep each table 16 times smaller; the kernels, results and
    quartet counts are those of FusedBatch on each group."""

    def __init__(self, molecules, densities, threshold: float, device="cuda", group: int = 64, **kw):
        if group < 1:
            raise ValueError("group must be at least 1")
        self.device = torch.device(device)
        self.parts, self.where = [], []
        for s in range(0, len(molecules), group):
            fb = FusedBatch(molecules[s:s + group], densities[s:s + group], threshold, device=device, **kw)
            self.where += [(len(self.parts), m) for m in range(fb.nmol)]
            self.parts.append(fb)
        self.nmol = len(self.where)
        self.graph = None

    def nbytes(self) -> int:
        return sum(p.nbytes() for p in self.parts)

    def issue(self, stream=None):
        """Zero the outputs and queue one iteration of every group."""
        for p in self.parts:
            p.issue(stream)

    def capture(self):
        """Capture one iteration of all groups into one CUDA graph."""
        s = torch.cuda.Stream(device=self.device)
        L = self.parts[0].L
        self.issue(s)
        torch.cuda.synchronize(self.device)
        L.reset_counters()
        self.issue(s)
        torch.cuda.synchronize(self.device)
        qj, qk = L.quartet_counters(reset=True)
        self.quartets_per_iteration = qj + qk
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=s):
            self.issue(s)
        self.graph = g

    def run(self):
        if self.graph is None:
            self.issue()
        else:
            self.graph.replay()

    def set_density(self, m: int, D: np.ndarray):
        p, k = self.where[m]
        self.parts[p].set_density(k, D)

    def results(self, m: int):
        p, k = self.where[m]
        return self.parts[p].results(k)
