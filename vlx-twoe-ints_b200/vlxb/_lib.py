"""ctypes binding of libvlxb.so (the C ABI declared in include/vlxb.h).

The argument lists are taken from csrc/gen_abi.py, the same generator that
writes include/vlxb.h and the extern "C" definitions, so the three cannot
drift apart.  There is no fallback: if the library is missing the import of
this module's `lib()` raises.
"""
from __future__ import annotations

import ctypes
import importlib.util
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(_HERE)
LIB_PATH = os.path.join(_HERE, "libvlxb.so")


class VlxbError(RuntimeError):
    pass


def _load_spec():
    spec = importlib.util.spec_from_file_location("vlxb_gen_abi", os.path.join(PKG_ROOT, "csrc", "gen_abi.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


ABI = _load_spec()


def _ctype(decl: str):
    t = decl.rsplit(" ", 1)[0]
    if "*" in t:
        return ctypes.c_void_p
    if t.endswith("uint32_t"):
        return ctypes.c_uint32
    if t.endswith("uint64_t"):
        return ctypes.c_uint64
    if t.endswith("double"):
        return ctypes.c_double
    if t.endswith("int"):
        return ctypes.c_int
    raise ValueError(decl)


class Lib:
    def __init__(self, path: str = LIB_PATH):
        if not os.path.exists(path):
            raise VlxbError(f"{path} is missing: build it with `python -m vlxb.build` (nvcc, sm_100a)")
        self.path = path
        self.cdll = ctypes.CDLL(path)
        self.j_params = {}
        self.k_params = {}
        for cls in ABI.j_classes() + ABI.jf_classes():
            ps = ABI.j_params(cls)
            if "f" in cls and not hasattr(self.cdll, f"vlxb_computeCoulombFock{cls.upper()}"):
                continue  # a library built without the f classes: calling one raises KeyError
            f = getattr(self.cdll, f"vlxb_computeCoulombFock{cls.upper()}")
            f.argtypes = [_ctype(p) for p in ps]
            f.restype = ctypes.c_int
            self.j_params[cls] = [ABI.pname(p) for p in ps]
        self.g_params = {}
        for cls in ABI.j_classes():
            ps = ABI.g_params(cls)
            f = getattr(self.cdll, f"vlxb_computeCoulombGradient{cls.upper()}")
            f.argtypes = [_ctype(p) for p in ps]
            f.restype = ctypes.c_int
            self.g_params[cls] = [ABI.pname(p) for p in ps]
        self.kg_params = {}
        for cls in ABI.k_classes():
            ps = ABI.kg_params(cls)
            f = getattr(self.cdll, f"vlxb_computeExchangeGradient{cls.upper()}")
            f.argtypes = [_ctype(p) for p in ps]
            f.restype = ctypes.c_int
            self.kg_params[cls] = [ABI.pname(p) for p in ps]
        for cls in ABI.k_classes() + ABI.kf_classes():
            ps = ABI.k_params(cls)
            if "f" in cls and not hasattr(self.cdll, f"vlxb_computeExchangeFock{cls.upper()}"):
                continue
            f = getattr(self.cdll, f"vlxb_computeExchangeFock{cls.upper()}")
            f.argtypes = [_ctype(p) for p in ps]
            f.restype = ctypes.c_int
            self.k_params[cls] = [ABI.pname(p) for p in ps]
        c = self.cdll
        c.vlxb_init.argtypes = [ctypes.c_int]
        c.vlxb_status_string.restype = ctypes.c_char_p
        c.vlxb_status_string.argtypes = [ctypes.c_int]
        c.vlxb_schwarzBareMax.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32,
                                          ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
        c.vlxb_quartetCounters.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        c.vlxb_kernelErrors.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        c.vlxb_setSchedule.argtypes = [ctypes.c_int] * 6
        c.vlxb_getSchedule.argtypes = [ctypes.c_int] * 5
        c.vlxb_launchCount.argtypes = [ctypes.c_void_p, ctypes.c_int]
        c.vlxb_fp64Probe.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        c.vlxb_setFp32Cutoff.argtypes = [ctypes.c_double]
        c.vlxb_getFp32Cutoff.restype = ctypes.c_double
        c.vlxb_setFp32Budget.argtypes = [ctypes.c_double]
        c.vlxb_getFp32Budget.restype = ctypes.c_double
        c.vlxb_pairsToAO.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_int64, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]
        c.vlxb_fockEnergy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                      ctypes.c_void_p, ctypes.c_void_p]
        c.vlxb_shellPairData.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32,
                                         ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        c.vlxb_gatherPairDensity.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p,
                                             ctypes.c_int, ctypes.c_uint32, ctypes.c_int64, ctypes.c_void_p,
                                             ctypes.c_void_p]
        c.vlxb_blockMaxAbs.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_int64,
                                       ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
        c.vlxb_pairGradientToAtoms.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]
        for fn in (c.vlxb_coulombBatch, c.vlxb_exchangeBatch):
            fn.argtypes = [ctypes.c_int] * 4 + [ctypes.c_void_p, ctypes.c_void_p]
            fn.restype = ctypes.c_int

    def check(self, rc: int, what: str):
        if rc != 0:
            raise VlxbError(f"{what}: {self.cdll.vlxb_status_string(rc).decode()} (status {rc})")

    def init(self, device: int):
        self.check(self.cdll.vlxb_init(int(device)), "vlxb_init")

    def coulomb(self, cls: str, args: dict) -> None:
        vals = [args[n] for n in self.j_params[cls]]
        rc = getattr(self.cdll, f"vlxb_computeCoulombFock{cls.upper()}")(*vals)
        self.check(rc, f"vlxb_computeCoulombFock{cls.upper()}")

    def coulomb_grad(self, cls: str, args: dict) -> None:
        vals = [args[n] for n in self.g_params[cls]]
        rc = getattr(self.cdll, f"vlxb_computeCoulombGradient{cls.upper()}")(*vals)
        self.check(rc, f"vlxb_computeCoulombGradient{cls.upper()}")

    def exchange_grad(self, cls: str, args: dict) -> None:
        vals = [args[n] for n in self.kg_params[cls]]
        rc = getattr(self.cdll, f"vlxb_computeExchangeGradient{cls.upper()}")(*vals)
        self.check(rc, f"vlxb_computeExchangeGradient{cls.upper()}")

    def exchange(self, cls: str, args: dict) -> None:
        vals = [args[n] for n in self.k_params[cls]]
        rc = getattr(self.cdll, f"vlxb_computeExchangeFock{cls.upper()}")(*vals)
        self.check(rc, f"vlxb_computeExchangeFock{cls.upper()}")

    def quartet_counters(self, reset: bool = True, stream: int = 0):
        out = (ctypes.c_ulonglong * 2)()
        self.check(self.cdll.vlxb_quartetCounters(ctypes.cast(out, ctypes.c_void_p), int(reset), stream),
                   "vlxb_quartetCounters")
        return int(out[0]), int(out[1])

    def set_schedule(self, kind: str, cls: str, variant: int):
        """kind "J" or "K"; cls like "pdpd"; see include/vlxb.h for variants."""
        l = [{"s": 0, "p": 1, "d": 2}[x] for x in cls]
        self.check(self.cdll.vlxb_setSchedule(0 if kind == "J" else 1, *l, int(variant)), "vlxb_setSchedule")

    def get_schedule(self, kind: str, cls: str) -> int:
        l = [{"s": 0, "p": 1, "d": 2}[x] for x in cls]
        return int(self.cdll.vlxb_getSchedule(0 if kind == "J" else 1, *l))

    def set_fp32_cut(self, cutoff: float):
        """Quartets with screening bound below `cutoff` run in FP32 (0 = FP64)."""
        self.check(self.cdll.vlxb_setFp32Cutoff(float(cutoff)), "vlxb_setFp32Cutoff")

    def get_fp32_cut(self) -> float:
        return float(self.cdll.vlxb_getFp32Cutoff())

    def set_fp32_budget(self, budget: float):
        """FP32 error budget (0 = none: the cutoff alone decides)."""
        self.check(self.cdll.vlxb_setFp32Budget(float(budget)), "vlxb_setFp32Budget")

    def get_fp32_budget(self) -> float:
        return float(self.cdll.vlxb_getFp32Budget())

    def launch_count(self, reset: bool = False) -> int:
        out = ctypes.c_ulonglong(0)
        self.check(self.cdll.vlxb_launchCount(ctypes.byref(out), int(reset)), "vlxb_launchCount")
        return int(out.value)

    def pairs_to_ao(self, values: int, rowptr: int, row_ao: int, src: int, n_rows: int, out: int, naos: int,
                    stream: int = 0):
        """vlxb_pairsToAO on raw device pointers (see include/vlxb.h)."""
        self.check(self.cdll.vlxb_pairsToAO(values, rowptr, row_ao, src, int(n_rows), out, int(naos), stream),
                   "vlxb_pairsToAO")

    def fock_energy(self, D: int, J: int, K: int, naos: int, out3: int, stream: int = 0):
        """vlxb_fockEnergy on raw device pointers (J or K may be 0 = NULL)."""
        self.check(self.cdll.vlxb_fockEnergy(D, J or None, K or None, int(naos), out3, stream), "vlxb_fockEnergy")

    def shell_pair_data(self, la, lb, info_a, cnt_a, info_b, cnt_b, P, Q, n, S_out, q_out, stream: int = 0):
        self.check(self.cdll.vlxb_shellPairData(int(la), int(lb), info_a, int(cnt_a), info_b, int(cnt_b), P, Q,
                                                int(n), S_out, q_out, stream), "vlxb_shellPairData")

    def gather_pair_density(self, D, naos, first, second, ao_a, nca, cnt_a, ao_b, ncb, cnt_b, n, out,
                            stream: int = 0):
        self.check(self.cdll.vlxb_gatherPairDensity(D, int(naos), first, second, ao_a, int(nca), int(cnt_a), ao_b,
                                                    int(ncb), int(cnt_b), int(n), out, stream),
                   "vlxb_gatherPairDensity")

    def block_max_abs(self, D, naos, rows, nrows, cols, ncols, out, stream: int = 0):
        self.check(self.cdll.vlxb_blockMaxAbs(D, int(naos), rows, int(nrows), cols, int(ncols), out, stream),
                   "vlxb_blockMaxAbs")

    def kernel_errors(self, reset: bool = False, stream: int = 0) -> int:
        """Device error word of the kernels (0 = no bounded wait ran out)."""
        out = ctypes.c_ulonglong(0)
        self.check(self.cdll.vlxb_kernelErrors(ctypes.byref(out), int(reset), stream), "vlxb_kernelErrors")
        return int(out.value)

    def reset_counters(self, stream: int = 0):
        self.check(self.cdll.vlxb_quartetCounters(None, 1, stream), "vlxb_quartetCounters")


_LIB = None


def lib() -> Lib:
    global _LIB
    if _LIB is None:
        _LIB = Lib()
    return _LIB
