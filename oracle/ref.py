"""ctypes front-end of oracle/_ref/libvlxref.so (the reference generator's own
emitted expressions inside a host restatement of the emitted kernels' loops,
built by oracle/make_ref.py).

TEST / BASELINE INFRASTRUCTURE ONLY: used by tests/ to pin the oracle and by
bench.py's CPU-baseline and reference legs.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, "_ref", "libvlxref.so")
LV = {"s": 0, "p": 1, "d": 2}
_vp = ctypes.c_void_p
_u32 = ctypes.c_uint32
_u64 = ctypes.c_uint64
_f64 = ctypes.c_double


def available() -> bool:
    return os.path.exists(LIB)


class RefLib:
    def __init__(self, path: str = LIB):
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run python oracle/make_ref.py where the reference tree is present")
        self.c = ctypes.CDLL(path)
        self.c.vlxref_count_j.restype = _u64
        self.c.vlxref_count_j.argtypes = [ctypes.c_int] * 4 + [_vp, _vp, _vp, _u32, _vp, _vp, _vp, _vp, _u32, _f64]
        self.c.vlxref_count_k.restype = _u64
        self.c.vlxref_count_k.argtypes = ([ctypes.c_int] * 4 + [_u32, _u32, _vp, _vp, _u32]
                                          + [_vp] * 8 + [_f64, _f64])

    def fn(self, name, argtypes):
        f = getattr(self.c, name)
        f.argtypes = argtypes
        f.restype = None
        return f


_REF = None


def lib() -> RefLib:
    global _REF
    if _REF is None:
        _REF = RefLib()
    return _REF


def _p(a):
    return a.ctypes.data_as(_vp) if a is not None else None


def _tables(pd, with_aoinds=False):
    keep = []
    infos = (_vp * 3)()
    aoi = (_vp * 3)()
    counts = np.zeros(3, dtype=np.uint32)
    for l in range(3):
        a = np.ascontiguousarray(pd.info[l] if pd.count[l] else np.zeros((5, 1)))
        keep.append(a)
        infos[l] = a.ctypes.data
        counts[l] = pd.count[l]
        if with_aoinds:
            b = np.ascontiguousarray(pd.aoinds[l] if pd.count[l] else np.zeros((1, 1)), dtype=np.uint32)
            keep.append(b)
            aoi[l] = b.ctypes.data
    keep.append(counts)
    return infos, aoi, counts, keep


def schwarz_fn(la, lb, pd, P, Q):
    """lists.build_lists Schwarz callable from the (ab|ab) expressions."""
    ab = "spd"[la] + "spd"[lb]
    f = lib().fn(f"vlxref_schwarz_{ab}", [_vp, _vp, _vp, _vp, _u32, _vp])
    infos, _, counts, keep = _tables(pd)
    P = np.ascontiguousarray(P, dtype=np.uint32)
    Q = np.ascontiguousarray(Q, dtype=np.uint32)
    out = np.zeros(len(P))
    f(infos, _p(counts), _p(P), _p(Q), len(P), _p(out))
    return out


def coulomb(rl, cls, rows=None, max_eval=2**63, mat_J=None):
    """mat_J (+=) of one class; returns (mat_J, passing cq of the rows, evaluated cq)."""
    a, b, c, d = cls
    jab, jcd = rl.jlists[a + b], rl.jlists[c + d]
    f = lib().fn(f"vlxref_coulomb_{cls}", [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _u32, _vp, _vp, _vp, _u32,
                                          _f64, _vp, _u32, _u64, _vp, _vp])
    infos, _, counts, keep = _tables(rl.pd)
    if mat_J is None:
        mat_J = np.zeros(len(jab.first))
    r = None if rows is None else np.ascontiguousarray(rows, dtype=np.uint32)
    cp, ce = _u64(0), _u64(0)
    f(_p(mat_J), infos, _p(counts), _p(jcd.D), _p(jab.Q), _p(jcd.Q), _p(jab.first), _p(jab.second), _p(jab.pdata),
      len(jab.first), _p(jcd.first), _p(jcd.second), _p(jcd.pdata), len(jcd.first), float(rl.threshold), _p(r),
      0 if r is None else len(r), int(max_eval), ctypes.byref(cp), ctypes.byref(ce))
    return mat_J, cp.value, ce.value


def exchange(rl, cls, omega=0.0, rows=None, max_eval=2**63, mat_K=None):
    a, b, c, d = cls
    kq = rl.kpairs[a + c]
    p1, p2 = rl.kpartners[a + b], rl.kpartners[c + d]
    f = lib().fn(f"vlxref_exchange_{cls}", [_vp, _vp, _vp, _u32, _vp, _vp, _vp, _f64, _vp, _u32] + [_vp] * 10
                 + [_f64, _f64, _vp, _u32, _u64, _vp, _vp])
    infos, aoi, counts, keep = _tables(rl.pd, with_aoinds=True)
    if mat_K is None:
        mat_K = np.zeros(len(kq.pair_i))
    r = None if rows is None else np.ascontiguousarray(rows, dtype=np.uint32)
    D = np.ascontiguousarray(rl.D_AO)
    cp, ce = _u64(0), _u64(0)
    f(_p(mat_K), _p(kq.pair_i), _p(kq.pair_k), len(kq.pair_i), infos, aoi, _p(counts), float(rl.maxD[b + d]), _p(D),
      int(rl.naos), _p(p1.Q), _p(p2.Q), _p(p1.Dinds), _p(p2.Dinds), _p(p1.displs), _p(p2.displs), _p(p1.counts),
      _p(p2.counts), _p(p1.pdata), _p(p2.pdata), float(omega), float(rl.threshold), _p(r),
      0 if r is None else len(r), int(max_eval), ctypes.byref(cp), ctypes.byref(ce))
    return mat_K, cp.value, ce.value


def count_j(rl, cls) -> int:
    a, b, c, d = cls
    jab, jcd = rl.jlists[a + b], rl.jlists[c + d]
    return int(lib().c.vlxref_count_j(LV[a], LV[b], LV[c], LV[d], _p(jab.Q), _p(jab.first), _p(jab.second),
                                      len(jab.first), _p(jcd.Q), _p(jcd.D), _p(jcd.first), _p(jcd.second),
                                      len(jcd.first), float(rl.threshold)))


def count_k(rl, cls) -> int:
    a, b, c, d = cls
    kq = rl.kpairs[a + c]
    p1, p2 = rl.kpartners[a + b], rl.kpartners[c + d]
    return int(lib().c.vlxref_count_k(LV[a], LV[b], LV[c], LV[d], rl.pd.count[LV[a]], rl.pd.count[LV[c]],
                                      _p(kq.pair_i), _p(kq.pair_k), len(kq.pair_i), _p(p1.Q), _p(p1.Dinds),
                                      _p(p1.displs), _p(p1.counts), _p(p2.Q), _p(p2.Dinds), _p(p2.displs),
                                      _p(p2.counts), float(rl.maxD[b + d]), float(rl.threshold)))
