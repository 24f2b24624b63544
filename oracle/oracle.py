"""ctypes front-end of the C oracle (eri_oracle.c) plus an mpmath Boys function.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  The C file restates the
reference's algorithm; each function cites the reference file:line it follows.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "eri_oracle.c")
_LIB = os.path.join(_HERE, "liboracle.so")

_u32p = ctypes.POINTER(ctypes.c_uint32)
_f64p = ctypes.POINTER(ctypes.c_double)


def build(force: bool = False) -> str:
    """Compile eri_oracle.c into oracle/liboracle.so (gcc, OpenMP)."""
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(_SRC):
        cmd = ["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-o", _LIB, _SRC, "-lm"]
        subprocess.run(cmd, check=True)
    return _LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB)
        L.oracle_boys.argtypes = [ctypes.c_int, ctypes.c_double, _f64p]
        L.oracle_eri_shell_quartet.argtypes = (
            [ctypes.c_int] * 4
            + [ctypes.c_double, _f64p] * 4
            + [ctypes.c_double, _f64p]
        )
        L.oracle_eri_shell_quartet_grad.argtypes = (
            [ctypes.c_int] * 5
            + [ctypes.c_double, _f64p] * 4
            + [ctypes.c_double, _f64p]
        )
        L.oracle_coulomb_fock.argtypes = (
            [ctypes.c_int] * 4
            + [_f64p, ctypes.POINTER(_f64p), _u32p, _f64p, _f64p, _f64p,
               _u32p, _u32p, _f64p, ctypes.c_uint32,
               _u32p, _u32p, _f64p, ctypes.c_uint32,
               ctypes.c_double, _u32p, ctypes.c_uint32]
        )
        L.oracle_coulomb_grad.argtypes = (
            [ctypes.c_int] * 4
            + [_f64p, ctypes.c_uint64, ctypes.POINTER(_f64p), _u32p, _f64p, _f64p, _f64p,
               _u32p, _u32p, _f64p, ctypes.c_uint32,
               _u32p, _u32p, _f64p, ctypes.c_uint32,
               ctypes.c_double, _u32p, ctypes.c_uint32]
        )
        L.oracle_exchange_fock.argtypes = (
            [ctypes.c_int] * 4
            + [_f64p, _u32p, _u32p, ctypes.c_uint32,
               ctypes.POINTER(_f64p), ctypes.POINTER(_u32p), _u32p,
               ctypes.c_double, _f64p, ctypes.c_uint32,
               _f64p, _f64p, _u32p, _u32p, _u32p, _u32p, _u32p, _u32p, _f64p, _f64p,
               ctypes.c_double, ctypes.c_double, _u32p, ctypes.c_uint32]
        )
        L.oracle_exchange_grad.argtypes = (
            [ctypes.c_int] * 4
            + [_f64p, ctypes.c_uint64, _u32p, _u32p, ctypes.c_uint32,
               ctypes.POINTER(_f64p), ctypes.POINTER(_u32p), _u32p,
               ctypes.c_double, _f64p, ctypes.c_uint32,
               _f64p, _f64p, _u32p, _u32p, _u32p, _u32p, _u32p, _u32p, _f64p, _f64p,
               ctypes.c_double, ctypes.c_double, _u32p, ctypes.c_uint32]
        )
        L.oracle_num_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _f(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_f64p)


def _u(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, a.ctypes.data_as(_u32p)


def boys(M: int, T: float) -> np.ndarray:
    out = np.zeros(M + 1)
    lib().oracle_boys(int(M), float(T), out.ctypes.data_as(_f64p))
    return out


def boys_mpmath(M: int, T: float, dps: int = 40) -> list:
    """F_m(T) = gamma(m+1/2) * P(m+1/2, T) / (2 T^(m+1/2)), exact to dps digits."""
    import mpmath as mp

    with mp.workdps(dps):
        t = mp.mpf(T)
        out = []
        for m in range(M + 1):
            if t == 0:
                out.append(mp.mpf(1) / (2 * m + 1))
            else:
                a = mp.mpf(m) + mp.mpf(1) / 2
                out.append(mp.gammainc(a, 0, t) / (2 * t ** a))
        return out


def eri_shell_quartet(la, lb, lc, ld, ai, A, aj, B, ak, C, al, D, omega=0.0):
    """Bare (ab|cd)/(S_ab S_cd) for all Cartesian components, shape (na,nb,nc,nd);
    shells up to f."""
    nc = [1, 3, 6, 10]
    out = np.zeros(nc[la] * nc[lb] * nc[lc] * nc[ld])
    args = []
    keep = []
    for al_, R in ((ai, A), (aj, B), (ak, C), (al, D)):
        r, p = _f(R)
        keep.append(r)
        args += [ctypes.c_double(al_), p]
    lib().oracle_eri_shell_quartet(la, lb, lc, ld, *args, ctypes.c_double(omega),
                                   out.ctypes.data_as(_f64p))
    return out.reshape(nc[la], nc[lb], nc[lc], nc[ld])


def eri_shell_quartet_grad(la, lb, lc, ld, center, ai, A, aj, B, ak, C, al, D, omega=0.0):
    """d/dX_g of the bare integrals, X the centre `center` (0..3 = A..D):
    array (3, na, nb, nc, nd)."""
    nc = [1, 3, 6]
    out = np.zeros(3 * nc[la] * nc[lb] * nc[lc] * nc[ld])
    args = []
    keep = []
    for al_, R in ((ai, A), (aj, B), (ak, C), (al, D)):
        r, p = _f(R)
        keep.append(r)
        args += [ctypes.c_double(al_), p]
    lib().oracle_eri_shell_quartet_grad(la, lb, lc, ld, int(center), *args, ctypes.c_double(omega),
                                        out.ctypes.data_as(_f64p))
    return out.reshape(3, nc[la], nc[lb], nc[lc], nc[ld])


def _prim_tables(prim_info, prim_count, prim_aoinds=None):
    """prim_info: dict l -> array (5, count); returns ctypes arrays and keep-alive list."""
    keep = []
    infos = (_f64p * 4)()
    aoinds = (_u32p * 4)()
    counts = np.zeros(4, dtype=np.uint32)
    for l in range(4):
        if l in prim_info and prim_info[l] is not None:
            a, p = _f(prim_info[l])
            keep.append(a)
            infos[l] = p
            counts[l] = prim_count[l]
            if prim_aoinds is not None:
                b, q = _u(prim_aoinds[l])
                keep.append(b)
                aoinds[l] = q
        else:
            dummy = np.zeros(5)
            keep.append(dummy)
            infos[l] = dummy.ctypes.data_as(_f64p)
            if prim_aoinds is not None:
                dz = np.zeros(1, dtype=np.uint32)
                keep.append(dz)
                aoinds[l] = dz.ctypes.data_as(_u32p)
    keep.append(counts)
    return infos, aoinds, counts, keep


def coulomb_fock(la, lb, lc, ld, prim_info, prim_count, cd_D, ab_Q, cd_Q,
                 ab_first, ab_second, ab_pdata, cd_first, cd_second, cd_pdata,
                 thr, rows=None, mat_J=None):
    """Oracle J for one class; returns mat_J (len n_ab, += semantics onto mat_J)."""
    n_ab = len(ab_first)
    n_cd = len(cd_first)
    if mat_J is None:
        mat_J = np.zeros(n_ab)
    mat_J = np.ascontiguousarray(mat_J, dtype=np.float64)
    infos, _, counts, keep = _prim_tables(prim_info, prim_count)
    arrs = [_f(cd_D), _f(ab_Q), _f(cd_Q), _u(ab_first), _u(ab_second), _f(ab_pdata),
            _u(cd_first), _u(cd_second), _f(cd_pdata)]
    if rows is None:
        r, rp, nr = None, None, 0
    else:
        r, rp = _u(rows)
        nr = len(r)
    lib().oracle_coulomb_fock(
        la, lb, lc, ld, mat_J.ctypes.data_as(_f64p), infos, counts.ctypes.data_as(_u32p),
        arrs[0][1], arrs[1][1], arrs[2][1], arrs[3][1], arrs[4][1], arrs[5][1], n_ab,
        arrs[6][1], arrs[7][1], arrs[8][1], n_cd, float(thr), rp, nr)
    del keep, arrs, r
    return mat_J


def coulomb_grad(la, lb, lc, ld, prim_info, prim_count, cd_D, ab_Q, cd_Q,
                 ab_first, ab_second, ab_pdata, cd_first, cd_second, cd_pdata,
                 thr, rows=None, grad=None):
    """Oracle bra-centre derivatives of J for one class: array (6, n_ab),
    rows 0..2 d mat_J / dA, rows 3..5 d mat_J / dB (+= onto grad)."""
    n_ab = len(ab_first)
    n_cd = len(cd_first)
    if grad is None:
        grad = np.zeros((6, n_ab))
    grad = np.ascontiguousarray(grad, dtype=np.float64)
    assert grad.shape == (6, n_ab)
    infos, _, counts, keep = _prim_tables(prim_info, prim_count)
    arrs = [_f(cd_D), _f(ab_Q), _f(cd_Q), _u(ab_first), _u(ab_second), _f(ab_pdata),
            _u(cd_first), _u(cd_second), _f(cd_pdata)]
    if rows is None:
        r, rp, nr = None, None, 0
    else:
        r, rp = _u(rows)
        nr = len(r)
    lib().oracle_coulomb_grad(
        la, lb, lc, ld, grad.ctypes.data_as(_f64p), n_ab, infos, counts.ctypes.data_as(_u32p),
        arrs[0][1], arrs[1][1], arrs[2][1], arrs[3][1], arrs[4][1], arrs[5][1], n_ab,
        arrs[6][1], arrs[7][1], arrs[8][1], n_cd, float(thr), rp, nr)
    del keep, arrs, r
    return grad


def exchange_fock(la, lb, lc, ld, pair_i, pair_k, prim_info, prim_aoinds, prim_count,
                  bd_max_D, D_AO, Q_ab, Q_cd, Dinds_ab, Dinds_cd, displs_ab, displs_cd,
                  counts_ab, counts_cd, pdata_ab, pdata_cd, omega, thr, rows=None, mat_K=None):
    """Oracle K for one class; returns mat_K (len n_ik, += semantics onto mat_K)."""
    n_ik = len(pair_i)
    if mat_K is None:
        mat_K = np.zeros(n_ik)
    mat_K = np.ascontiguousarray(mat_K, dtype=np.float64)
    infos, aoinds, counts, keep = _prim_tables(prim_info, prim_count, prim_aoinds)
    D_AO = np.ascontiguousarray(D_AO, dtype=np.float64)
    naos = D_AO.shape[0]
    arrs = [_u(pair_i), _u(pair_k), _f(D_AO), _f(Q_ab), _f(Q_cd), _u(Dinds_ab), _u(Dinds_cd),
            _u(displs_ab), _u(displs_cd), _u(counts_ab), _u(counts_cd), _f(pdata_ab), _f(pdata_cd)]
    if rows is None:
        r, rp, nr = None, None, 0
    else:
        r, rp = _u(rows)
        nr = len(r)
    lib().oracle_exchange_fock(
        la, lb, lc, ld, mat_K.ctypes.data_as(_f64p), arrs[0][1], arrs[1][1], n_ik,
        infos, aoinds, counts.ctypes.data_as(_u32p), float(bd_max_D), arrs[2][1], naos,
        arrs[3][1], arrs[4][1], arrs[5][1], arrs[6][1], arrs[7][1], arrs[8][1],
        arrs[9][1], arrs[10][1], arrs[11][1], arrs[12][1], float(omega), float(thr), rp, nr)
    del keep, arrs, r
    return mat_K


def exchange_grad(la, lb, lc, ld, pair_i, pair_k, prim_info, prim_aoinds, prim_count,
                  bd_max_D, D_AO, Q_ab, Q_cd, Dinds_ab, Dinds_cd, displs_ab, displs_cd,
                  counts_ab, counts_cd, pdata_ab, pdata_cd, omega, thr, rows=None, grad=None):
    """Oracle energy-weighted centre derivatives of K for one class, per (i, k)
    entry: array (6, n_ik), rows 0..2 for i's centre, 3..5 for k's (+= onto grad)."""
    n_ik = len(pair_i)
    if grad is None:
        grad = np.zeros((6, n_ik))
    grad = np.ascontiguousarray(grad, dtype=np.float64)
    assert grad.shape == (6, n_ik)
    infos, aoinds, counts, keep = _prim_tables(prim_info, prim_count, prim_aoinds)
    D_AO = np.ascontiguousarray(D_AO, dtype=np.float64)
    naos = D_AO.shape[0]
    arrs = [_u(pair_i), _u(pair_k), _f(D_AO), _f(Q_ab), _f(Q_cd), _u(Dinds_ab), _u(Dinds_cd),
            _u(displs_ab), _u(displs_cd), _u(counts_ab), _u(counts_cd), _f(pdata_ab), _f(pdata_cd)]
    if rows is None:
        r, rp, nr = None, None, 0
    else:
        r, rp = _u(rows)
        nr = len(r)
    lib().oracle_exchange_grad(
        la, lb, lc, ld, grad.ctypes.data_as(_f64p), n_ik, arrs[0][1], arrs[1][1], n_ik,
        infos, aoinds, counts.ctypes.data_as(_u32p), float(bd_max_D), arrs[2][1], naos,
        arrs[3][1], arrs[4][1], arrs[5][1], arrs[6][1], arrs[7][1], arrs[8][1],
        arrs[9][1], arrs[10][1], arrs[11][1], arrs[12][1], float(omega), float(thr), rp, nr)
    del keep, arrs, r
    return grad
