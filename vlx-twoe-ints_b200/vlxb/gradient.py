"""Coulomb nuclear gradient on the device: dE_J/dR for E_J = 1/2 Tr[D J[D]].

Over the reference-format J lists, E_J = 1/2 sum_o w_o D_o mat_J[o], o running
over the bra entries of every J list, D_o = cd_mat_D of the entry and w_o = 1
for a diagonal entry of a same-type list, else 2 (the weights that turn the
list values into the AO matrix M + M^T; gen_coulomb.py:296 writes mat_J[ij]).
The double sum over bra and ket entries is symmetric, so the derivative of
the ket side equals that of the bra side and

    dE_J/dR = sum over the 36 J classes of sum_o w_o D_o d mat_J[o] / dR,

with d mat_J[o]/dR the bra-centre derivatives (ket fixed) that
vlxb_computeCoulombGradient<ABCD> writes: rows 0..2 for the entry's first
centre A, 3..5 for its second centre B.  `vlxb_pairGradientToAtoms` then
folds them onto atoms through a resident CSR (entry, side) -> atom, summed in
a fixed order.  The derivative terms are the reference generator's
gradient='a' / 'b' terms (eri.py:85-129, eriwriter.py:72-87), which no
reference generator emits.

Screening is the J entry points' (|Q_ij Q_kl D_kl| > threshold on the ket
sum), so the bra/ket symmetry, and with it translational invariance, holds to
the screening error.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import lib
from .fock import DeviceLists
from .lists import ANG, LV, NCART, j_classes, prim_data


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


def prim_atoms(mol, device) -> dict:
    """Atom of every primitive of each angular momentum (the prim_info order)."""
    pd = prim_data(mol)
    return {l: torch.from_numpy(pd.atom[l].astype(np.int64)).to(device) for l in range(3) if pd.count[l] > 0}


class GradientMap:
    """Resident layout of one list set: the flat bra-entry space of all J
    lists (list "ab" at columns offsets[ab]..), the CSR (entry, side) -> atom
    and the diagonal weights w_o."""

    def __init__(self, dl: DeviceLists, atoms: dict, natoms: int):
        self.device = dl.device
        self.natoms = int(natoms)
        self.keys = sorted(dl.j)
        sizes = [dl.j[k]["first"].numel() for k in self.keys]
        offs = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        self.offsets = {k: int(offs[t]) for t, k in enumerate(self.keys)}
        self.total = int(offs[-1])
        if self.total >= (1 << 31):
            raise ValueError("more than 2^31 J list entries")
        dev = self.device
        rows, srcs, wd = [], [], []
        for k in self.keys:
            la, lb = LV[k[0]], LV[k[1]]
            f = dl.j[k]["first"].long()
            s2 = dl.j[k]["second"].long()
            pos = self.offsets[k] + torch.arange(f.numel(), dtype=torch.int64, device=dev)
            rows += [atoms[la][f // NCART[la]], atoms[lb][s2 // NCART[lb]]]
            srcs += [pos, pos | (1 << 31)]
            diag = (f == s2) & (la == lb)
            wd.append(torch.where(diag, 1.0, 2.0).to(torch.float64))
        if rows:
            row = torch.cat(rows)
            src = torch.cat(srcs)
            order = torch.sort(row, stable=True).indices
            row, src = row[order], src[order]
            cnt = torch.bincount(row, minlength=self.natoms)
            self.wdiag = torch.cat(wd)
        else:
            src = torch.zeros(0, dtype=torch.int64, device=dev)
            cnt = torch.zeros(self.natoms, dtype=torch.int64, device=dev)
            self.wdiag = torch.zeros(0, dtype=torch.float64, device=dev)
        self.rowptr = torch.zeros(self.natoms + 1, dtype=torch.int64, device=dev)
        self.rowptr[1:] = torch.cumsum(cnt, 0)
        self.src = torch.where(src >= (1 << 31), src - (1 << 32), src).to(torch.int32)  # uint32 bits

    def weights(self, dl: DeviceLists) -> torch.Tensor:
        """w_o D_o over the flat entry space (current densities of the lists)."""
        if not self.keys:
            return self.wdiag
        return self.wdiag * torch.cat([dl.j[k]["D"] for k in self.keys])

    def nbytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in (self.rowptr, self.src, self.wdiag))


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


def to_atoms(G: torch.Tensor, gmap: GradientMap, weight: torch.Tensor, stream=None,
             out: torch.Tensor | None = None) -> torch.Tensor:
    """Per-atom gradient [natoms, 3] of pair derivatives G and weights."""
    st = stream or torch.cuda.current_stream(gmap.device)
    if out is None:
        out = torch.empty((gmap.natoms, 3), dtype=torch.float64, device=gmap.device)
    lib().check(lib().cdll.vlxb_pairGradientToAtoms(G.data_ptr(), G.shape[1], weight.data_ptr() if weight.numel() else 0,
                                                    gmap.rowptr.data_ptr(), gmap.src.data_ptr() if gmap.src.numel() else 0,
                                                    gmap.natoms, out.data_ptr(), st.cuda_stream),
                "vlxb_pairGradientToAtoms")
    return out


class CoulombGradient:
    """Resident Coulomb-gradient state of one system: its device lists and the
    gradient map; `compute()` is one gradient evaluation on the device."""

    def __init__(self, dl: DeviceLists, mol):
        self.dl = dl
        self.map = GradientMap(dl, prim_atoms(mol, dl.device), mol.natoms)

    def compute(self, stream=None) -> torch.Tensor:
        st = stream or torch.cuda.current_stream(self.dl.device)
        with torch.cuda.stream(st):
            G = pair_gradients(self.dl, self.map, st)
            w = self.map.weights(self.dl)
            return to_atoms(G, self.map, w, st)


def coulomb_gradient(mol, D_AO, threshold: float = 1e-12, device="cuda", dl: DeviceLists | None = None):
    """dE_J/dR (natoms x 3, device tensor) for E_J = 1/2 Tr[D J[D]], with the
    lists built on the device when `dl` is not given."""
    if dl is None:
        from .devlists import build_device_lists

        dl = build_device_lists(mol, D_AO, threshold, device)
    return CoulombGradient(dl, mol).compute()


__all__ = ["CoulombGradient", "GradientMap", "coulomb_gradient", "grad_args", "pair_gradients", "prim_atoms",
           "to_atoms"]
