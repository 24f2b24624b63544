"""Nuclear gradients of the two-electron energy terms on the device:
dE_J/dR for E_J = 1/2 Tr[D J[D]] and dE_K/dR for E_K = 1/2 Tr[D K[D]]
(closed-shell HF: dE_2e/dR = dE_J/dR - 1/2 dE_K/dR with D the total density).

Coulomb.  Over the reference-format J lists E_J = 1/2 sum_o w_o D_o mat_J[o],
o running over the bra entries of every J list, D_o = cd_mat_D of the entry,
w_o = 1 for a diagonal entry of a same-type list, else 2 (the weights that
turn the list values into the AO matrix M + M^T; gen_coulomb.py:296 writes
mat_J[ij]).  The double sum over bra and ket entries is symmetric, so

    dE_J/dR = sum over the 36 J classes of sum_o w_o D_o d mat_J[o] / dR,

with d mat_J[o]/dR the bra-centre derivatives (ket fixed) that
vlxb_computeCoulombGradient<ABCD> writes: rows 0..2 for the entry's first
centre, 3..5 for its second.

Exchange.  E_K = 1/2 sum_{ijkl} D_ik D_jl (ij|kl) is symmetric under
(i <-> j, k <-> l) and (ij) <-> (kl), so only the centres of i and k need
derivatives: vlxb_computeExchangeGradient<ABCD> writes, per primitive shell
block of each K (i, k) list, sum w_ik D_ik sum_jl D_jl d(ij|kl)/d(A, C) at
the block's lowest list position (already weighted).

`vlxb_pairGradientToAtoms` folds either onto atoms through a resident CSR
(entry, side) -> atom, summed in a fixed order.  The derivative terms are the
reference generator's gradient='a'..'c' terms (eri.py:85-152,
eriwriter.py:72-87), which no reference generator emits.

Screening is the entry points' own (J: |Q_ij Q_kl D_kl| > threshold, K:
|Q_ij Q_kl max_D| > threshold), so the symmetries, and with them
translational invariance, hold to the screening error.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import lib
from .fock import DeviceLists, exchange_args
from .lists import ANG, LV, NCART, j_classes, k_classes, prim_data


def grad_args(dl: DeviceLists, cls: str, grad: torch.Tensor, offset: int, stride: int, stream: int) -> dict:
    """Arguments of vlxb_computeCoulombGradient<cls> writing into the columns
    offset.. of a [6][stride] device array."""
    a, b, c, d = cls
    ab, cd = a + b, c + d
    A = {"grad_J": grad.data_ptr() + 8 * offset, "grad_stride": stride}
    for x in ANG:
        if x in cls:
            A[f"{x}_prim_info"] = dl.info[LV[x]].data_ptr()
            A[f"{x}_prim_count"] = dl.count[LV[x]]
    jab, jcd = dl.j[ab], dl.j[cd]
    A.update({
        f"{cd}_mat_D": jcd["D"].data_ptr(), f"{ab}_mat_Q_local": jab["Q"].data_ptr(),
        f"{cd}_mat_Q": jcd["Q"].data_ptr(),
        f"{ab}_first_inds_local": jab["first"].data_ptr(), f"{ab}_second_inds_local": jab["second"].data_ptr(),
        f"{ab}_pair_data_local": jab["pdata"].data_ptr(), f"{ab}_prim_pair_count_local": jab["first"].numel(),
        f"{cd}_first_inds": jcd["first"].data_ptr(), f"{cd}_second_inds": jcd["second"].data_ptr(),
        f"{cd}_pair_data": jcd["pdata"].data_ptr(), f"{cd}_prim_pair_count": jcd["first"].numel(),
        "boys_func_table": None, "boys_func_ft": None, "eri_threshold": dl.threshold, "stream": stream,
    })
    return A


def kgrad_args(dl: DeviceLists, cls: str, grad: torch.Tensor, offset: int, stride: int, stream: int,
               omega: float = 0.0) -> dict:
    """Arguments of vlxb_computeExchangeGradient<cls> writing into the columns
    offset.. of a [6][stride] device array."""
    A = exchange_args(dl, cls, grad, stream, omega)
    del A["mat_K"]
    A["grad_K"] = grad.data_ptr() + 8 * offset
    A["grad_stride"] = stride
    return A


def prim_atoms(mol, device) -> dict:
    """Atom of every primitive of each angular momentum (the prim_info order)."""
    pd = prim_data(mol)
    return {l: torch.from_numpy(pd.atom[l].astype(np.int64)).to(device) for l in range(3) if pd.count[l] > 0}


class GradientMap:
    """Resident layout of one family of lists (the J lists, fields "first" /
    "second", or the K (i, k) lists, fields "i" / "k"): the flat entry space
    (list `key` at columns offsets[key]..), the CSR (entry, side) -> atom, and
    the diagonal flags of same-type lists."""

    def __init__(self, lists: dict, fields, atoms: dict, natoms: int, device):
        if any("f" in k for k in lists):
            raise ValueError("the nuclear-gradient entry points cover s, p and d shells only")
        self.device = torch.device(device)
        self.natoms = int(natoms)
        self.keys = sorted(lists)
        sizes = [lists[k][fields[0]].numel() for k in self.keys]
        offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        self.offsets = {k: int(offs[t]) for t, k in enumerate(self.keys)}
        self.total = int(offs[-1])
        if self.total >= (1 << 31):
            raise ValueError("more than 2^31 list entries")
        dev = self.device
        rows, srcs, diag = [], [], []
        for k in self.keys:
            la, lb = LV[k[0]], LV[k[1]]
            f = lists[k][fields[0]].long()
            s2 = lists[k][fields[1]].long()
            pos = self.offsets[k] + torch.arange(f.numel(), dtype=torch.int64, device=dev)
            rows += [atoms[la][f // NCART[la]], atoms[lb][s2 // NCART[lb]]]
            srcs += [pos, pos | (1 << 31)]
            diag.append((f == s2) & (la == lb))
        if rows:
            row = torch.cat(rows)
            src = torch.cat(srcs)
            order = torch.sort(row, stable=True).indices
            row, src = row[order], src[order]
            cnt = torch.bincount(row, minlength=self.natoms)
            self.diag = torch.cat(diag)
        else:
            src = torch.zeros(0, dtype=torch.int64, device=dev)
            cnt = torch.zeros(self.natoms, dtype=torch.int64, device=dev)
            self.diag = torch.zeros(0, dtype=torch.bool, device=dev)
        self.rowptr = torch.zeros(self.natoms + 1, dtype=torch.int64, device=dev)
        self.rowptr[1:] = torch.cumsum(cnt, 0)
        self.src = torch.where(src >= (1 << 31), src - (1 << 32), src).to(torch.int32)  # uint32 bits

    def nbytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in (self.rowptr, self.src, self.diag))


def coulomb_weights(dl: DeviceLists, gmap: GradientMap) -> torch.Tensor:
    """w_o D_o over the flat J entry space (current densities of the lists)."""
    if not gmap.keys:
        return torch.zeros(0, dtype=torch.float64, device=gmap.device)
    w = torch.where(gmap.diag, 1.0, 2.0).to(torch.float64)
    return w * torch.cat([dl.j[k]["D"] for k in gmap.keys])


def pair_gradients(dl: DeviceLists, gmap: GradientMap, stream=None, classes=None) -> torch.Tensor:
    """[6][total] bra-centre derivatives of every J list entry, summed over
    the J classes (all 36 by default), through the class entry points."""
    L = lib()
    st = stream or torch.cuda.current_stream(dl.device)
    G = torch.zeros((6, max(gmap.total, 1)), dtype=torch.float64, device=dl.device)
    with torch.cuda.stream(st):
        for cls in (classes or j_classes()):
            if cls[:2] in dl.j and cls[2:] in dl.j:
                L.coulomb_grad(cls, grad_args(dl, cls, G, gmap.offsets[cls[:2]], G.shape[1], st.cuda_stream))
    return G


def exchange_pair_gradients(dl: DeviceLists, kmap: GradientMap, stream=None, omega: float = 0.0,
                            classes=None) -> torch.Tensor:
    """[6][total] energy-weighted K derivatives over the flat (i, k) entry
    space, summed over the K classes (all 54 by default)."""
    L = lib()
    st = stream or torch.cuda.current_stream(dl.device)
    G = torch.zeros((6, max(kmap.total, 1)), dtype=torch.float64, device=dl.device)
    with torch.cuda.stream(st):
        for cls in (classes or k_classes()):
            ac = cls[0] + cls[2]
            if ac in dl.kpair and cls[:2] in dl.kpart and cls[2:] in dl.kpart:
                L.exchange_grad(cls, kgrad_args(dl, cls, G, kmap.offsets[ac], G.shape[1], st.cuda_stream, omega))
    return G


def to_atoms(G: torch.Tensor, gmap: GradientMap, weight: torch.Tensor | None = None, stream=None,
             out: torch.Tensor | None = None) -> torch.Tensor:
    """Per-atom gradient [natoms, 3] of pair derivatives G (weights: 1 when
    `weight` is None)."""
    st = stream or torch.cuda.current_stream(gmap.device)
    if out is None:
        out = torch.empty((gmap.natoms, 3), dtype=torch.float64, device=gmap.device)
    wp = weight.data_ptr() if weight is not None and weight.numel() else 0
    stride = G.shape[1] if gmap.total else 0  # no entries: nothing is read
    lib().check(lib().cdll.vlxb_pairGradientToAtoms(G.data_ptr(), stride, wp, gmap.rowptr.data_ptr(),
                                                    gmap.src.data_ptr() if gmap.src.numel() else 0,
                                                    gmap.natoms, out.data_ptr(), st.cuda_stream),
                "vlxb_pairGradientToAtoms")
    return out


class CoulombGradient:
    """Resident Coulomb-gradient state of one system: its device lists and the
    J gradient map; `compute()` is one gradient evaluation on the device."""

    def __init__(self, dl: DeviceLists, mol):
        self.dl = dl
        self.map = GradientMap(dl.j, ("first", "second"), prim_atoms(mol, dl.device), mol.natoms, dl.device)

    def compute(self, stream=None) -> torch.Tensor:
        st = stream or torch.cuda.current_stream(self.dl.device)
        with torch.cuda.stream(st):
            G = pair_gradients(self.dl, self.map, st)
            return to_atoms(G, self.map, coulomb_weights(self.dl, self.map), st)


class ExchangeGradient:
    """Resident exchange-gradient state of one system: dE_K/dR for
    E_K = 1/2 Tr[D K] (omega > 0: the erf-attenuated operator)."""

    def __init__(self, dl: DeviceLists, mol):
        self.dl = dl
        self.map = GradientMap(dl.kpair, ("i", "k"), prim_atoms(mol, dl.device), mol.natoms, dl.device)

    def compute(self, omega: float = 0.0, stream=None) -> torch.Tensor:
        st = stream or torch.cuda.current_stream(self.dl.device)
        with torch.cuda.stream(st):
            G = exchange_pair_gradients(self.dl, self.map, st, omega)
            return to_atoms(G, self.map, None, st)


def coulomb_gradient(mol, D_AO, threshold: float = 1e-12, device="cuda", dl: DeviceLists | None = None):
    """dE_J/dR (natoms x 3, device tensor) for E_J = 1/2 Tr[D J[D]], with the
    lists built on the device when `dl` is not given."""
    if dl is None:
        from .devlists import build_device_lists

        dl = build_device_lists(mol, D_AO, threshold, device)
    return CoulombGradient(dl, mol).compute()


def exchange_gradient(mol, D_AO, threshold: float = 1e-12, device="cuda", dl: DeviceLists | None = None,
                      omega: float = 0.0):
    """dE_K/dR (natoms x 3, device tensor) for E_K = 1/2 Tr[D K[D]]."""
    if dl is None:
        from .devlists import build_device_lists

        dl = build_device_lists(mol, D_AO, threshold, device)
    return ExchangeGradient(dl, mol).compute(omega)


__all__ = ["CoulombGradient", "ExchangeGradient", "GradientMap", "coulomb_gradient", "coulomb_weights",
           "exchange_gradient", "exchange_pair_gradients", "grad_args", "kgrad_args", "pair_gradients",
           "prim_atoms", "to_atoms"]
