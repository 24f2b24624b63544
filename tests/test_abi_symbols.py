"""The C-ABI library loads and exports every function include/vlxb.h declares
(no compute calls: these run without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "vlxb.h")
LIBP = os.path.join(ROOT, "vlx-twoe-ints_b200", "vlxb", "libvlxb.so")


def declared():
    txt = open(HDR).read()
    return re.findall(r"^(?:int|const char\*)\s+(vlxb_\w+)\(", txt, flags=re.M)


def test_header_lists_all_reference_classes():
    names = declared()
    j = [n for n in names if n.startswith("vlxb_computeCoulombFock") and not n.endswith("_noalloc")]
    k = [n for n in names if n.startswith("vlxb_computeExchangeFock")]
    # the reference's 36 + 54 s/p/d classes, plus 64 + 106 with f shells
    assert len([n for n in j if "F" not in n[len("vlxb_computeCoulombFock"):]]) == 36
    assert len([n for n in k if "F" not in n[len("vlxb_computeExchangeFock"):]]) == 54
    assert len(j) == 36 + 64 and len(k) == 54 + 106
    assert [n for n in names if n.endswith("_noalloc")] == ["vlxb_computeCoulombFockSSSS_noalloc"]
    assert "vlxb_computeCoulombFockDDDD" in j and "vlxb_computeExchangeFockSDPD" in k and "vlxb_computeExchangeFockPDSD" not in k


def test_library_exports_every_declared_symbol():
    if not os.path.exists(LIBP):
        pytest.fail("libvlxb.so is not built (python -m vlxb.build)")
    lib = ctypes.CDLL(LIBP)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_version():
    lib = ctypes.CDLL(LIBP)
    lib.vlxb_status_string.restype = ctypes.c_char_p
    assert lib.vlxb_status_string(0) == b"ok"
    assert lib.vlxb_status_string(1) == b"invalid argument"
    assert lib.vlxb_version() >= 100


def test_python_binding_matches_header():
    from vlxb._lib import ABI

    hdr = open(HDR).read()
    for cls in ABI.j_classes():
        sig = f"int vlxb_computeCoulombFock{cls.upper()}(" + ", ".join(ABI.j_params(cls)) + ");"
        assert sig in hdr
    for cls in ABI.k_classes():
        sig = f"int vlxb_computeExchangeFock{cls.upper()}(" + ", ".join(ABI.k_params(cls)) + ");"
        assert sig in hdr


def test_f_shell_entry_points_declared_and_bound():
    """The 64 Coulomb and 106 exchange classes with f shells (this library's
    own: the reference emits s/p/d only) are declared with the generated
    entry points' conventions and bound by the Python layer."""
    from vlxb._lib import ABI, lib

    hdr = open(HDR).read()
    jf, kf = ABI.jf_classes(), ABI.kf_classes()
    assert len(jf) == 64 and len(kf) == 106
    assert all("f" in c for c in jf + kf)
    for cls in jf:
        assert f"int vlxb_computeCoulombFock{cls.upper()}(" + ", ".join(ABI.j_params(cls)) + ");" in hdr
    for cls in kf:
        assert f"int vlxb_computeExchangeFock{cls.upper()}(" + ", ".join(ABI.k_params(cls)) + ");" in hdr
    assert ABI.j_params("sfsf")[1:5] == ["const double* s_prim_info", "uint32_t s_prim_count",
                                         "const double* f_prim_info", "uint32_t f_prim_count"]
    L = lib()
    assert set(jf) <= set(L.j_params) and set(kf) <= set(L.k_params)


def test_gradient_entry_points_declared_and_bound():
    """One Coulomb-gradient entry point per J class and one exchange-gradient
    entry point per K class, with the argument lists the Python binding uses,
    plus the per-atom fold."""
    from vlxb._lib import ABI

    names = declared()
    jg = [n for n in names if n.startswith("vlxb_computeCoulombGradient")]
    kg = [n for n in names if n.startswith("vlxb_computeExchangeGradient")]
    assert len(jg) == 36 and len(kg) == 54
    assert "vlxb_pairGradientToAtoms" in names
    hdr = open(HDR).read()
    for cls in ABI.j_classes():
        ps = ABI.g_params(cls)
        assert ps[:2] == ["double* grad_J", "uint64_t grad_stride"] and ps[2:] == ABI.j_params(cls)[1:]
        assert f"int vlxb_computeCoulombGradient{cls.upper()}(" + ", ".join(ps) + ");" in hdr
    for cls in ABI.k_classes():
        ps = ABI.kg_params(cls)
        assert ps[:2] == ["double* grad_K", "uint64_t grad_stride"] and ps[2:] == ABI.k_params(cls)[1:]
        assert f"int vlxb_computeExchangeGradient{cls.upper()}(" + ", ".join(ps) + ");" in hdr


def test_gradient_argument_checks_without_gpu():
    """Checks the gradient entry points and the fold make before any device
    call: a component stride beyond int64, no atoms, and empty lists."""
    from vlxb._lib import Lib

    L = Lib()
    c = L.cdll
    dummy = ctypes.c_double(0.0)
    p = ctypes.addressof(dummy)  # never dereferenced: every call below returns before touching memory
    huge = (1 << 63) + 5
    # the fold: no atoms, stride past the int64 range
    assert c.vlxb_pairGradientToAtoms(p, 0, None, p, p, 0, p, None) == 1
    assert c.vlxb_pairGradientToAtoms(p, 1 << 62, None, p, p, 2, p, None) == 1
    # stride beyond int64: rejected before any list is read
    for cls, names, fn in (("ssss", L.g_params["ssss"], c.vlxb_computeCoulombGradientSSSS),
                           ("ssss", L.kg_params["ssss"], c.vlxb_computeExchangeGradientSSSS)):
        args = []
        for n in names:
            if n == "grad_stride":
                args.append(huge)
            elif n in ("eri_threshold", "omega") or n.endswith("_max_D"):
                args.append(0.0)
            elif n.endswith("_count") or n.endswith("_count_local") or n.startswith("pair_inds_count") or n == "naos":
                args.append(1)
            else:
                args.append(p)
        assert fn(*args) == 1, cls
    # empty bra list: success, nothing to do
    args = [p if n not in ("grad_stride", "eri_threshold") and "count" not in n else 0 for n in L.g_params["ssss"]]
    args[L.g_params["ssss"].index("grad_stride")] = 1
    assert c.vlxb_computeCoulombGradientSSSS(*args) == 0
