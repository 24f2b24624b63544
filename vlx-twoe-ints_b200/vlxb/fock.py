"""J/K builds through the C ABI (the drop-in path).

`DeviceLists` holds the reference-format arrays of one system on the GPU
(torch tensors used as plain device buffers); `build_jk` calls the 36 Coulomb
and 54 exchange entry points exactly as the reference's host would call the
emitted kernels, accumulating mat_J per bra list ("ab") and mat_K per (i, k)
list ("ac").
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from ._lib import lib
from .lists import ANG, LMAX, LV, ReferenceLists, j_classes_all, k_classes_all


def _i32(a: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)


@dataclass
class DeviceLists:
    device: torch.device
    naos: int
    threshold: float
    count: dict
    info: dict = field(default_factory=dict)
    aoinds: dict = field(default_factory=dict)
    D_AO: torch.Tensor = None
    j: dict = field(default_factory=dict)      # "ab" -> dict of tensors
    kpart: dict = field(default_factory=dict)  # "ab" -> dict of tensors
    kpair: dict = field(default_factory=dict)  # "ac" -> dict of tensors
    maxD: dict = field(default_factory=dict)

    def nbytes(self) -> int:
        n = self.D_AO.numel() * 8
        for d in (self.info, self.aoinds):
            n += sum(t.numel() * t.element_size() for t in d.values())
        for grp in (self.j, self.kpart, self.kpair):
            for d in grp.values():
                n += sum(t.numel() * t.element_size() for t in d.values())
        return n


def host_arrays(rl: ReferenceLists) -> dict:
    """Flat dict name -> contiguous numpy array (uint32 viewed as int32)."""
    out = {"D_AO": np.ascontiguousarray(rl.D_AO, dtype=np.float64)}
    for l in range(LMAX + 1):
        if rl.pd.count[l] > 0:
            out[f"info{l}"] = np.ascontiguousarray(rl.pd.info[l])
            out[f"aoinds{l}"] = _i32(rl.pd.aoinds[l])
    for k, jl in rl.jlists.items():
        out[f"j_{k}_first"] = _i32(jl.first)
        out[f"j_{k}_second"] = _i32(jl.second)
        out[f"j_{k}_pdata"] = jl.pdata
        out[f"j_{k}_Q"] = jl.Q
        out[f"j_{k}_D"] = jl.D
    for k, kp in rl.kpartners.items():
        out[f"kp_{k}_displs"] = _i32(kp.displs)
        out[f"kp_{k}_counts"] = _i32(kp.counts)
        out[f"kp_{k}_Dinds"] = _i32(kp.Dinds)
        out[f"kp_{k}_Q"] = kp.Q
        out[f"kp_{k}_pdata"] = kp.pdata
    for k, kq in rl.kpairs.items():
        out[f"kq_{k}_i"] = _i32(kq.pair_i)
        out[f"kq_{k}_k"] = _i32(kq.pair_k)
    return out


def pinned_copy(arrays: dict) -> dict:
    """Page-locked host copies (torch CPU tensors) of the host arrays."""
    return {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in arrays.items()}


def upload(rl: ReferenceLists, tensors: dict, device, non_blocking: bool = False) -> DeviceLists:
    """Device copies of host tensors (torch CPU, ideally pinned) laid out as DeviceLists."""
    dev = torch.device(device)
    g = {k: v.to(dev, non_blocking=non_blocking) for k, v in tensors.items()}
    dl = DeviceLists(device=dev, naos=rl.naos, threshold=rl.threshold, count=dict(rl.pd.count), maxD=dict(rl.maxD))
    dl.D_AO = g["D_AO"]
    for l in range(LMAX + 1):
        if f"info{l}" in g:
            dl.info[l] = g[f"info{l}"]
            dl.aoinds[l] = g[f"aoinds{l}"]
    for k in rl.jlists:
        dl.j[k] = {n: g[f"j_{k}_{n}"] for n in ("first", "second", "pdata", "Q", "D")}
    for k in rl.kpartners:
        dl.kpart[k] = {n: g[f"kp_{k}_{n}"] for n in ("displs", "counts", "Dinds", "Q", "pdata")}
    for k in rl.kpairs:
        dl.kpair[k] = {"i": g[f"kq_{k}_i"], "k": g[f"kq_{k}_k"]}
    return dl


def to_device(rl: ReferenceLists, device="cuda") -> DeviceLists:
    return upload(rl, {k: torch.from_numpy(v) for k, v in host_arrays(rl).items()}, device)


def _p(t: torch.Tensor) -> int:
    return t.data_ptr()


def coulomb_args(dl: DeviceLists, cls: str, matJ: torch.Tensor, stream: int) -> dict:
    a, b, c, d = cls
    ab, cd = a + b, c + d
    A = {"mat_J": _p(matJ)}
    for x in ANG:
        if x in cls:
            A[f"{x}_prim_info"] = _p(dl.info[LV[x]])
            A[f"{x}_prim_count"] = dl.count[LV[x]]
    jab, jcd = dl.j[ab], dl.j[cd]
    A.update({
        f"{cd}_mat_D": _p(jcd["D"]), f"{ab}_mat_Q_local": _p(jab["Q"]), f"{cd}_mat_Q": _p(jcd["Q"]),
        f"{ab}_first_inds_local": _p(jab["first"]), f"{ab}_second_inds_local": _p(jab["second"]),
        f"{ab}_pair_data_local": _p(jab["pdata"]), f"{ab}_prim_pair_count_local": jab["first"].numel(),
        f"{cd}_first_inds": _p(jcd["first"]), f"{cd}_second_inds": _p(jcd["second"]),
        f"{cd}_pair_data": _p(jcd["pdata"]), f"{cd}_prim_pair_count": jcd["first"].numel(),
        "boys_func_table": None, "boys_func_ft": None, "eri_threshold": dl.threshold, "stream": stream,
    })
    return A


def exchange_args(dl: DeviceLists, cls: str, matK: torch.Tensor, stream: int, omega: float) -> dict:
    a, b, c, d = cls
    ac = a + c
    A = {"mat_K": _p(matK), f"pair_inds_i_for_K_{ac}": _p(dl.kpair[ac]["i"]),
         f"pair_inds_k_for_K_{ac}": _p(dl.kpair[ac]["k"]), f"pair_inds_count_for_K_{ac}": dl.kpair[ac]["i"].numel()}
    for x in ANG:
        if x in cls:
            A[f"{x}_prim_info"] = _p(dl.info[LV[x]])
            A[f"{x}_prim_aoinds"] = _p(dl.aoinds[LV[x]])
            A[f"{x}_prim_count"] = dl.count[LV[x]]
    A[f"{b}{d}_max_D"] = dl.maxD[b + d]
    A["mat_D_full_AO"] = _p(dl.D_AO)
    A["naos"] = dl.naos
    for key in {a + b, c + d}:
        kp = dl.kpart[key]
        A[f"Q_K_{key}"] = _p(kp["Q"])
        A[f"D_inds_K_{key}"] = _p(kp["Dinds"])
        A[f"pair_displs_K_{key}"] = _p(kp["displs"])
        A[f"pair_counts_K_{key}"] = _p(kp["counts"])
        A[f"pair_data_K_{key}"] = _p(kp["pdata"])
    A.update({"boys_func_table": None, "boys_func_ft": None, "omega": omega,
              "eri_threshold": dl.threshold, "stream": stream})
    return A


def alloc_outputs(dl: DeviceLists):
    matJ = {k: torch.zeros(v["first"].numel(), dtype=torch.float64, device=dl.device) for k, v in dl.j.items()}
    matK = {k: torch.zeros(v["i"].numel(), dtype=torch.float64, device=dl.device) for k, v in dl.kpair.items()}
    return matJ, matK


def build_jk(dl: DeviceLists, stream: torch.cuda.Stream | None = None, omega: float = 0.0,
             j_only=None, k_only=None, matJ=None, matK=None, do_j=True, do_k=True):
    """Launch every J and K class through the C ABI on `stream` (asynchronous).
    Returns (matJ, matK): device tensors in prim-cart pair space."""
    L = lib()
    if stream is None:
        stream = torch.cuda.current_stream(dl.device)
    s = stream.cuda_stream
    if matJ is None or matK is None:
        matJ, matK = alloc_outputs(dl)
    with torch.cuda.stream(stream):
        if do_j:
            for cls in (j_only or j_classes_all()):
                if cls[:2] in dl.j and cls[2:] in dl.j:
                    L.coulomb(cls, coulomb_args(dl, cls, matJ[cls[:2]], s))
        if do_k:
            for cls in (k_only or k_classes_all()):
                ac = cls[0] + cls[2]
                if ac in dl.kpair and cls[:2] in dl.kpart and cls[2:] in dl.kpart:
                    L.exchange(cls, exchange_args(dl, cls, matK[ac], s, omega))
    return matJ, matK


def gpu_schwarz_fn(device="cuda"):
    """Schwarz helper for lists.build_lists backed by vlxb_schwarzBareMax."""
    L = lib()
    dev = torch.device(device)

    def fn(la, lb, pd, P, Q):
        n = len(P)
        if n == 0:
            return np.zeros(0)
        ia = torch.from_numpy(np.ascontiguousarray(pd.info[la])).to(dev)
        ib = torch.from_numpy(np.ascontiguousarray(pd.info[lb])).to(dev)
        tp = torch.from_numpy(_i32(P)).to(dev)
        tq = torch.from_numpy(_i32(Q)).to(dev)
        out = torch.empty(n, dtype=torch.float64, device=dev)
        s = torch.cuda.current_stream(dev).cuda_stream
        L.check(L.cdll.vlxb_schwarzBareMax(la, lb, ia.data_ptr(), pd.count[la], ib.data_ptr(), pd.count[lb],
                                           tp.data_ptr(), tq.data_ptr(), n, out.data_ptr(), s),
                "vlxb_schwarzBareMax")
        return out.cpu().numpy()

    return fn
