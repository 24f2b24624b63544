"""Primitive-pair -> AO contraction of J and K, and the energy, on the device.

The class entry points write mat_J / mat_K in primitive Cartesian pair space
(one value per list entry, gen_coulomb.py:296, gen_exchange.py:341).
`lists.contract_J` / `lists.contract_K` turn them into symmetric AO matrices on
the host; `AOMap` does the same on the GPU through `vlxb_pairsToAO`, with the
per-list outputs laid out in one flat buffer so that a single CSR gather
covers every list.  The map is built once per list set and stays resident,
so an SCF loop can keep J, K and D on the device and read back only the
energy (`vlxb_fockEnergy`).
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import lib
from .lists import LV, NCART, ReferenceLists

WEIGHT2 = np.uint32(1 << 31)


def _targets_J(rl: ReferenceLists, key: str):
    jl = rl.jlists[key]
    la, lb = LV[key[0]], LV[key[1]]
    a = rl.pd.aoinds[la][jl.first % NCART[la], jl.first // NCART[la]]
    b = rl.pd.aoinds[lb][jl.second % NCART[lb], jl.second // NCART[lb]]
    diag_entry = (la == lb) & (jl.first == jl.second)
    return a.astype(np.int64), b.astype(np.int64), diag_entry


def _targets_K(rl: ReferenceLists, key: str):
    kp = rl.kpairs[key]
    la, lc = LV[key[0]], LV[key[1]]
    a = rl.pd.aoinds[la][kp.pair_i % NCART[la], kp.pair_i // NCART[la]]
    c = rl.pd.aoinds[lc][kp.pair_k % NCART[lc], kp.pair_k // NCART[lc]]
    diag_entry = (la == lc) & (kp.pair_i == kp.pair_k)
    return a.astype(np.int64), c.astype(np.int64), diag_entry


def build_map(naos: int, parts):
    """CSR over AO pairs (a <= b) from [(offset, a, b, diag_entry), ...].

    Every value v at flat position offset + t lands in AO pair
    (min(a, b), max(a, b)) with weight 2 when a == b and it is not a
    diagonal entry of a same-type list, else 1: the AO matrix is M + M^T of
    the host contraction.  Entries of one row keep ascending flat position.
    Returns numpy (rowptr int64, row_ao int32, src uint32)."""
    rows, srcs = [], []
    for off, a, b, de in parts:
        lo, hi = np.minimum(a, b), np.maximum(a, b)
        pos = off + np.arange(len(a), dtype=np.int64)
        if len(pos) and pos[-1] >= (1 << 31):
            raise ValueError("more than 2^31 pair values")
        w2 = (a == b) & ~de
        rows.append(lo * naos + hi)
        srcs.append(pos.astype(np.uint32) | np.where(w2, WEIGHT2, np.uint32(0)))
    if not rows:
        return np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0, np.uint32)
    row = np.concatenate(rows)
    src = np.concatenate(srcs)
    order = np.lexsort(((src & ~WEIGHT2).astype(np.int64), row))  # by row, then by position
    row, src = row[order], src[order]
    uniq, start = np.unique(row, return_index=True)
    rowptr = np.append(start, len(row)).astype(np.int64)
    return rowptr, uniq.astype(np.int32), src.astype(np.uint32)


def contract_host(naos: int, values: np.ndarray, rowptr, row_ao, src) -> np.ndarray:
    """numpy evaluation of a map (the device kernel's arithmetic, for tests)."""
    M = np.zeros((naos, naos))
    w = np.where(src >> 31, 2.0, 1.0)
    v = values[(src & ~WEIGHT2).astype(np.int64)] * w
    for r in range(len(row_ao)):
        s = 0.0
        for x in v[rowptr[r]:rowptr[r + 1]]:
            s += x
        a, b = divmod(int(row_ao[r]), naos)
        M[a, b] = M[b, a] = s
    return M


def build_map_torch(naos: int, parts):
    """build_map on tensors (same layout and entry order): parts are
    (offset, a, b, diag_entry) with int64 / bool tensors.  Returns tensors
    (rowptr int64, row_ao int32, src int32 holding the uint32 bits)."""
    dev = parts[0][1].device if parts else torch.device("cpu")
    rows, srcs = [], []
    for off, a, b, de in parts:
        lo, hi = torch.minimum(a, b), torch.maximum(a, b)
        pos = off + torch.arange(a.numel(), dtype=torch.int64, device=dev)
        if pos.numel() and int(pos[-1]) >= (1 << 31):
            raise ValueError("more than 2^31 pair values")
        rows.append(lo * naos + hi)
        srcs.append(pos | (((a == b) & ~de).to(torch.int64) << 31))
    if not rows:
        return (torch.zeros(1, dtype=torch.int64, device=dev), torch.zeros(0, dtype=torch.int32, device=dev),
                torch.zeros(0, dtype=torch.int32, device=dev))
    row = torch.cat(rows)
    src = torch.cat(srcs)
    order = torch.sort(row, stable=True).indices  # positions ascend within a row: the concatenation order
    row, src = row[order], src[order]
    uniq, cnt = torch.unique_consecutive(row, return_counts=True)
    rowptr = torch.zeros(uniq.numel() + 1, dtype=torch.int64, device=dev)
    rowptr[1:] = torch.cumsum(cnt, 0)
    src32 = torch.where(src >= (1 << 31), src - (1 << 32), src).to(torch.int32)  # uint32 bits in int32 storage
    return rowptr, uniq.to(torch.int32), src32


class _DeviceMap:
    def __init__(self, keys, sizes, rowptr, row_ao, src, device):
        self.keys = list(keys)
        self.sizes = list(sizes)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        self.total = int(self.offsets[-1])
        if isinstance(rowptr, torch.Tensor):
            self.rowptr, self.row_ao, self.src = rowptr.to(device), row_ao.to(device), src.to(device)
        else:
            self.rowptr = torch.from_numpy(rowptr).to(device)
            self.row_ao = torch.from_numpy(row_ao).to(device)
            self.src = torch.from_numpy(src.view(np.int32)).to(device)
        self.n_rows = int(self.row_ao.numel())

    def alloc(self, device):
        """Zeroed flat value buffer and per-list views into it."""
        flat = torch.zeros(max(self.total, 1), dtype=torch.float64, device=device)
        views = {k: flat[int(o):int(o) + n] for k, o, n in zip(self.keys, self.offsets, self.sizes)}
        return flat, views

    def nbytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in (self.rowptr, self.row_ao, self.src))


class AOMap:
    """Resident J and K AO maps of one list set."""

    def __init__(self, rl: ReferenceLists, device="cuda"):
        self.device = torch.device(device)
        self.naos = rl.naos
        jkeys = sorted(rl.jlists)
        kkeys = sorted(rl.kpairs)
        jsz = [len(rl.jlists[k].first) for k in jkeys]
        ksz = [len(rl.kpairs[k].pair_i) for k in kkeys]
        joff = np.concatenate([[0], np.cumsum(jsz)])
        koff = np.concatenate([[0], np.cumsum(ksz)])
        jmap = build_map(self.naos, [(joff[i], *_targets_J(rl, k)) for i, k in enumerate(jkeys)])
        kmap = build_map(self.naos, [(koff[i], *_targets_K(rl, k)) for i, k in enumerate(kkeys)])
        self.J = _DeviceMap(jkeys, jsz, *jmap, self.device)
        self.K = _DeviceMap(kkeys, ksz, *kmap, self.device)

    @classmethod
    def from_device(cls, dl) -> "AOMap":
        """The map of device-resident lists (fock.DeviceLists), built where they live."""
        self = cls.__new__(cls)
        self.device = dl.device
        self.naos = dl.naos

        def ao(l, idx):
            n = NCART[l]
            idx = idx.long()
            return dl.aoinds[l][idx % n, idx // n].long()

        jkeys, kkeys = sorted(dl.j), sorted(dl.kpair)
        jsz = [dl.j[k]["first"].numel() for k in jkeys]
        ksz = [dl.kpair[k]["i"].numel() for k in kkeys]
        joff = np.concatenate([[0], np.cumsum(jsz)]).astype(np.int64)
        koff = np.concatenate([[0], np.cumsum(ksz)]).astype(np.int64)
        jp, kp = [], []
        for t, k in enumerate(jkeys):
            la, lb = LV[k[0]], LV[k[1]]
            f, s2 = dl.j[k]["first"], dl.j[k]["second"]
            jp.append((int(joff[t]), ao(la, f), ao(lb, s2), (f == s2) & (la == lb)))
        for t, k in enumerate(kkeys):
            la, lc = LV[k[0]], LV[k[1]]
            i, kk = dl.kpair[k]["i"], dl.kpair[k]["k"]
            kp.append((int(koff[t]), ao(la, i), ao(lc, kk), (i == kk) & (la == lc)))
        self.J = _DeviceMap(jkeys, jsz, *build_map_torch(self.naos, jp), self.device)
        self.K = _DeviceMap(kkeys, ksz, *build_map_torch(self.naos, kp), self.device)
        return self

    def alloc_outputs(self):
        """(flatJ, matJ views, flatK, matK views): pass the views to build_jk."""
        fj, vj = self.J.alloc(self.device)
        fk, vk = self.K.alloc(self.device)
        return fj, vj, fk, vk

    def to_ao(self, which: str, flat: torch.Tensor, out: torch.Tensor | None = None, stream=None) -> torch.Tensor:
        m = self.J if which == "J" else self.K
        if out is None:
            out = torch.empty((self.naos, self.naos), dtype=torch.float64, device=self.device)
        s = (stream or torch.cuda.current_stream(self.device)).cuda_stream
        lib().pairs_to_ao(flat.data_ptr(), m.rowptr.data_ptr(), m.row_ao.data_ptr(), m.src.data_ptr(), m.n_rows,
                          out.data_ptr(), self.naos, s)
        return out

    def nbytes(self) -> int:
        return self.J.nbytes() + self.K.nbytes()


def energy(D: torch.Tensor, J: torch.Tensor | None, K: torch.Tensor | None, out: torch.Tensor | None = None,
           stream=None) -> torch.Tensor:
    """Device tensor [Tr D(J - K/2), Tr DJ, Tr DK] (fixed summation order)."""
    dev = D.device
    if out is None:
        out = torch.empty(3, dtype=torch.float64, device=dev)
    s = (stream or torch.cuda.current_stream(dev)).cuda_stream
    lib().fock_energy(D.data_ptr(), J.data_ptr() if J is not None else 0, K.data_ptr() if K is not None else 0,
                      D.shape[0], out.data_ptr(), s)
    return out


__all__ = ["AOMap", "build_map", "build_map_torch", "contract_host", "energy"]
