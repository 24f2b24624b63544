"""Reference-format lists built on the GPU (the caller-side step before the
class entry points).

`lists.build_lists` builds the pair data, Schwarz values, density-in-pair-space
and sorted J / K lists on the host with numpy, as the reference's caller does.
`build_device_lists` produces the same lists on the device: the numerics run in
the library's kernels (`vlxb_shellPairData` for S and Q of every primitive
shell pair, `vlxb_gatherPairDensity` for cd_mat_D, `vlxb_blockMaxAbs` for the
bd_max_D bounds), the compaction and the orderings with stable device sorts,
so the result is a `fock.DeviceLists` ready for the entry points.  The orders
are the host builder's: J lists by descending |Q D| (stable), K partner lists
by first index then descending Q, K (i, k) lists row-major.

`set_density` is the per-SCF step: it refreshes the resident lists' density
values and the max-|D| bounds from a device AO density, with no host copy of
any list.
"""
from __future__ import annotations

import numpy as np
import torch

from . import lists
from ._lib import lib
from .fock import DeviceLists
from .lists import ANG, LMAX, LV, NCART


def _u32(t: torch.Tensor) -> torch.Tensor:
    """index tensor -> int32 storage of the uint32 values the ABI reads."""
    return t.to(torch.int32)


def _shell_pairs(L, dl, la, lb, s):
    na, nb = dl.count[la], dl.count[lb]
    dev = dl.device
    if la == lb:
        PQ = torch.triu_indices(na, na, device=dev)
        P, Q = PQ[0], PQ[1]
    else:
        P = torch.arange(na, device=dev).repeat_interleave(nb)
        Q = torch.arange(nb, device=dev).repeat(na)
    n = P.numel()
    S = torch.empty(n, dtype=torch.float64, device=dev)
    q = torch.empty(n, dtype=torch.float64, device=dev)
    P32, Q32 = _u32(P), _u32(Q)
    L.shell_pair_data(la, lb, dl.info[la].data_ptr(), na, dl.info[lb].data_ptr(), nb, P32.data_ptr(),
                      Q32.data_ptr(), n, S.data_ptr(), q.data_ptr(), s)
    return P, Q, S, q


def _expand(P, Q, S, q, la, lb, upper):
    """Shell pairs -> prim-cart pairs (lists._expand on the device)."""
    na, nb = NCART[la], NCART[lb]
    dev = P.device
    ca = torch.arange(na, device=dev).repeat_interleave(nb)
    cb = torch.arange(nb, device=dev).repeat(na)
    i = (P[:, None] * na + ca[None, :]).reshape(-1)
    j = (Q[:, None] * nb + cb[None, :]).reshape(-1)
    Sx = S.repeat_interleave(na * nb)
    qx = q.repeat_interleave(na * nb)
    if upper:
        m = i <= j
        i, j, Sx, qx = i[m], j[m], Sx[m], qx[m]
    return i, j, Sx, qx


def _gather_D(L, dl, D, la, lb, i, j, out, s):
    L.gather_pair_density(D.data_ptr(), dl.naos, i.data_ptr(), j.data_ptr(), dl.aoinds[la].data_ptr(), NCART[la],
                          dl.count[la], dl.aoinds[lb].data_ptr(), NCART[lb], dl.count[lb], i.numel(),
                          out.data_ptr(), s)


def _block_max(L, dl, D, lb, ld, s) -> torch.Tensor:
    out = torch.empty(1, dtype=torch.float64, device=dl.device)
    rows, cols = dl.aoinds[lb].reshape(-1), dl.aoinds[ld].reshape(-1)
    L.block_max_abs(D.data_ptr(), dl.naos, rows.data_ptr(), rows.numel(), cols.data_ptr(), cols.numel(),
                    out.data_ptr(), s)
    return out


def build_device_lists(mol, D_AO, threshold: float, device="cuda") -> DeviceLists:
    """The reference-format J / K lists of `mol` and density `D_AO` (numpy or
    a device tensor), built on `device` (current stream)."""
    L = lib()
    dev = torch.device(device)
    s = torch.cuda.current_stream(dev).cuda_stream
    pd = lists.prim_data(mol)
    dl = DeviceLists(device=dev, naos=mol.naos, threshold=threshold, count=dict(pd.count))
    D = D_AO if isinstance(D_AO, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(D_AO))
    dl.D_AO = D.to(dev, dtype=torch.float64).contiguous()
    ls = [l for l in range(LMAX + 1) if pd.count[l] > 0]
    for l in ls:
        dl.info[l] = torch.from_numpy(np.ascontiguousarray(pd.info[l])).to(dev)
        dl.aoinds[l] = torch.from_numpy(pd.aoinds[l].astype(np.int32)).to(dev)
    sp = {}
    for la in ls:
        for lb in ls:
            if la <= lb:
                sp[(la, lb)] = _shell_pairs(L, dl, la, lb, s)
    qmax = max(float(v[3].max()) for v in sp.values() if v[3].numel())
    dmax = float(dl.D_AO.abs().max())
    bmax = {b + d: _block_max(L, dl, dl.D_AO, LV[b], LV[d], s) for b in ANG for d in ANG
            if LV[b] in ls and LV[d] in ls}
    dl.maxD = {k: float(v) for k, v in bmax.items()}

    # J lists: pairs that can pass with the largest partner, prim-cart pairs
    # (i <= j for same-type lists), sorted by descending |Q D| (stable)
    for (la, lb), (P, Q, S, q) in sp.items():
        keep = q * qmax * dmax > threshold
        i, j, Sx, qx = _expand(P[keep], Q[keep], S[keep], q[keep], la, lb, upper=(la == lb))
        i32, j32 = _u32(i), _u32(j)
        Dv = torch.empty(i.numel(), dtype=torch.float64, device=dev)
        _gather_D(L, dl, dl.D_AO, la, lb, i32, j32, Dv, s)
        order = torch.sort((qx * Dv).abs(), descending=True, stable=True).indices
        dl.j[ANG[la] + ANG[lb]] = {"first": i32[order].contiguous(), "second": j32[order].contiguous(),
                                   "pdata": Sx[order].contiguous(), "Q": qx[order].contiguous(),
                                   "D": Dv[order].contiguous()}

    # K partner lists for every ordered type pair: by first index, then descending Q
    for la in ls:
        for lb in ls:
            if la <= lb:
                P, Q, S, q = sp[(la, lb)]
                if la == lb:  # add the mirrored pairs P > Q
                    off = P != Q
                    P, Q = torch.cat([P, Q[off]]), torch.cat([Q, P[off]])
                    S, q = torch.cat([S, S[off]]), torch.cat([q, q[off]])
            else:
                Q, P, S, q = sp[(lb, la)]
            keep = q * qmax * dmax > threshold
            i, j, Sx, qx = _expand(P[keep], Q[keep], S[keep], q[keep], la, lb, upper=False)
            o1 = torch.sort(qx, descending=True, stable=True).indices
            o2 = torch.sort(i[o1], stable=True).indices
            order = o1[o2]
            i, j, Sx, qx = i[order], j[order], Sx[order], qx[order]
            n_first = dl.count[la] * NCART[la]
            counts = torch.bincount(i, minlength=n_first)
            displs = torch.zeros(n_first, dtype=torch.int64, device=dev)
            if n_first > 1:
                displs[1:] = torch.cumsum(counts[:-1], 0)
            dl.kpart[ANG[la] + ANG[lb]] = {"displs": _u32(displs), "counts": _u32(counts), "Dinds": _u32(j),
                                           "Q": qx.contiguous(), "pdata": Sx.contiguous()}

    # K (i, k) lists: keep (i, k) when the best partner product can pass
    qpart = {}
    for la in ls:
        best = torch.zeros(dl.count[la] * NCART[la], dtype=torch.float64, device=dev)
        for lb in ls:
            kp = dl.kpart[ANG[la] + ANG[lb]]
            has = kp["counts"] > 0
            first_q = torch.zeros_like(best)
            if kp["Q"].numel():
                first_q[has] = kp["Q"][kp["displs"][has].long()]
            best = torch.maximum(best, first_q)
        qpart[la] = best
    for la in ls:
        for lc in ls:
            if la > lc:
                continue
            ii, kk = torch.nonzero(qpart[la][:, None] * qpart[lc][None, :] * dmax > threshold, as_tuple=True)
            if la == lc:
                m = ii <= kk
                ii, kk = ii[m], kk[m]
            dl.kpair[ANG[la] + ANG[lc]] = {"i": _u32(ii), "k": _u32(kk)}
    return dl


def set_density(dl: DeviceLists, D: torch.Tensor, stream=None):
    """Per-SCF update of resident lists: the AO density, every J list's
    cd_mat_D (gathered in list order) and the bd_max_D bounds (read back: the
    entry points take them by value)."""
    L = lib()
    st = stream or torch.cuda.current_stream(dl.device)
    s = st.cuda_stream
    with torch.cuda.stream(st):
        dl.D_AO.copy_(D)
        for key, jl in dl.j.items():
            la, lb = LV[key[0]], LV[key[1]]
            _gather_D(L, dl, dl.D_AO, la, lb, jl["first"], jl["second"], jl["D"], s)
        keys = list(dl.maxD)
        if keys:
            vals = torch.cat([_block_max(L, dl, dl.D_AO, LV[k[0]], LV[k[1]], s) for k in keys]).cpu()
            for t, k in enumerate(keys):
                dl.maxD[k] = float(vals[t])
    return dl


def to_host(dl: DeviceLists, mol) -> lists.ReferenceLists:
    """Host (numpy) copy of device-built lists as a `lists.ReferenceLists`
    (prim tables from `mol`, which the lists were built from): for the AO
    contraction on the host and for checks against the CPU references."""
    pd = lists.prim_data(mol)
    rl = lists.ReferenceLists(pd=pd, naos=dl.naos, D_AO=dl.D_AO.cpu().numpy(), threshold=dl.threshold,
                              maxD=dict(dl.maxD))
    u32 = lambda t: t.cpu().numpy().astype(np.uint32)  # noqa: E731
    for k, v in dl.j.items():
        rl.jlists[k] = lists.JList(u32(v["first"]), u32(v["second"]), v["pdata"].cpu().numpy(),
                                   v["Q"].cpu().numpy(), v["D"].cpu().numpy())
    for k, v in dl.kpart.items():
        rl.kpartners[k] = lists.KPartners(u32(v["displs"]), u32(v["counts"]), u32(v["Dinds"]),
                                          v["Q"].cpu().numpy(), v["pdata"].cpu().numpy())
    for k, v in dl.kpair.items():
        rl.kpairs[k] = lists.KPairs(u32(v["i"]), u32(v["k"]))
    return rl
