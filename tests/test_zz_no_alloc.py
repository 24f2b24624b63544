"""The allocation-free SSSS Coulomb entry point (vlxb_computeCoulombFockSSSS_noalloc).

It exists for callers that cannot allocate device memory (hosts whose device
memory belongs to their own allocator, plugins that may not allocate): it
keeps its scratch in a fixed 64 MiB device array of the library.  This file
is collected last on purpose.  It checks, through the C ABI, that two calls in
a row give the regular entry point's mat_J within the tolerance of the other
parity tests, that warm calls leave the device's free memory and the
stream-ordered pool's usage untouched (nothing is allocated), and that a call
needing more scratch than the array holds is refused before any work is
queued.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from vlxb import basis, fock, lists
from vlxb._lib import ABI, lib

pytestmark = pytest.mark.gpu
RTOL = 1e-10
ETOOBIG = 4


def _noalloc_fn(L):
    f = L.cdll.vlxb_computeCoulombFockSSSS_noalloc
    f.argtypes = [ctypes.c_void_p if "*" in p.rsplit(" ", 1)[0] else
                  (ctypes.c_uint32 if p.startswith("uint32_t") else ctypes.c_double)
                  for p in ABI.j_params("ssss")]
    f.restype = ctypes.c_int
    return f


def _pool_used_high_reset():
    """Resets the high watermark of the device's stream-ordered pool (the pool
    the regular entry points allocate their scratch from) and returns a reader
    of (used now, high since the reset); None without cuda-python."""
    try:
        from cuda.bindings import driver as dr
        from cuda.bindings import runtime as rt
    except ImportError:
        return None
    err, pool = rt.cudaDeviceGetMemPool(torch.cuda.current_device())
    if err != rt.cudaError_t.cudaSuccess:
        return None
    A = rt.cudaMemPoolAttr
    rt.cudaMemPoolSetAttribute(pool, A.cudaMemPoolAttrUsedMemHigh, dr.cuuint64_t(0))

    def read():
        _, used = rt.cudaMemPoolGetAttribute(pool, A.cudaMemPoolAttrUsedMemCurrent)
        _, high = rt.cudaMemPoolGetAttribute(pool, A.cudaMemPoolAttrUsedMemHigh)
        return int(used), int(high)

    return read


def test_noalloc_matches_regular_entry_point_twice():
    L = lib()
    torch.cuda.set_device(0)
    wl = basis.config_custom(4, 5.0, {0: 2, 1: 1}, 3, 0.2, 2.8, 4, 1e-12, 31)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    dl = fock.to_device(rl)
    s = torch.cuda.current_stream().cuda_stream
    n = dl.j["ss"]["first"].numel()

    ref = torch.zeros(n, dtype=torch.float64, device="cuda")
    L.coulomb("ssss", fock.coulomb_args(dl, "ssss", ref, s))
    f = _noalloc_fn(L)
    outs = []
    for _ in range(2):
        out = torch.zeros(n, dtype=torch.float64, device="cuda")
        A = fock.coulomb_args(dl, "ssss", out, s)
        rc = f(*[A[p] for p in L.j_params["ssss"]])
        assert rc == 0, L.cdll.vlxb_status_string(rc)
        outs.append(out)
    torch.cuda.synchronize()
    exp = ref.cpu().numpy()
    scale = float(np.abs(exp).max())
    assert scale > 0.0
    for out in outs:
        got = out.cpu().numpy()
        assert float(np.abs(got - exp).max()) <= RTOL * scale + 1e-14

    # warm calls allocate nothing: the device's free memory and the pool's
    # usage (high watermark included) stay where they were
    warm = torch.zeros(n, dtype=torch.float64, device="cuda")
    A = fock.coulomb_args(dl, "ssss", warm, s)
    args = [A[p] for p in L.j_params["ssss"]]
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    pool = _pool_used_high_reset()
    used0 = pool()[0] if pool else None
    for _ in range(2):
        assert f(*args) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    if pool:
        used1, high1 = pool()
        assert used1 == used0 and high1 <= used0, (used0, used1, high1)


def test_noalloc_rejects_oversized_call():
    """Counts that need more than the 64 MiB array are refused (VLXB_ETOOBIG)
    by the host-side sizing pass, before anything is launched."""
    L = lib()
    torch.cuda.set_device(0)
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    ibuf = torch.zeros(16, dtype=torch.int32, device="cuda")
    A = {p: None for p in L.j_params["ssss"]}
    for p in A:
        if p.endswith("count") or p.endswith("count_local"):
            A[p] = 0
    A.update({"mat_J": buf.data_ptr(), "s_prim_info": buf.data_ptr(), "s_prim_count": 20000,
              "ss_mat_D": buf.data_ptr(), "ss_mat_Q_local": buf.data_ptr(), "ss_mat_Q": buf.data_ptr(),
              "ss_first_inds_local": ibuf.data_ptr(), "ss_second_inds_local": ibuf.data_ptr(),
              "ss_pair_data_local": buf.data_ptr(), "ss_prim_pair_count_local": 10_000_000,
              "ss_first_inds": ibuf.data_ptr(), "ss_second_inds": ibuf.data_ptr(),
              "ss_pair_data": buf.data_ptr(), "ss_prim_pair_count": 10_000_000,
              "boys_func_table": None, "boys_func_ft": None, "eri_threshold": 1e-12,
              "stream": torch.cuda.current_stream().cuda_stream})
    rc = _noalloc_fn(L)(*[A[p] for p in L.j_params["ssss"]])
    assert rc == ETOOBIG
    torch.cuda.synchronize()
    assert float(buf.abs().max()) == 0.0
