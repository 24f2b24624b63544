"""Access to tests/golden/jk_tiny.npz (written by tests/golden/make_golden.py).

The fixture holds the reference-format ABI arrays of a two-atom s/p/d system
and mat_J / mat_K computed from the reference generator's own emitted
expressions with the emitted kernels' loop semantics.
"""
from __future__ import annotations

import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LV = {"s": 0, "p": 1, "d": 2}
ANG = "spd"
THRESHOLDS = {"t12": 1e-12, "t3": 2e-3}


def load():
    return dict(np.load(os.path.join(HERE, "golden", "jk_tiny.npz")))


def j_classes():
    pairs = [a + b for i, a in enumerate(ANG) for b in ANG[i:]]
    return [ab + cd for ab in pairs for cd in pairs]


def k_classes():
    return [a + b + c + d for i, a in enumerate(ANG) for c in ANG[i:] for b in ANG for d in ANG]


def prim_tables(z):
    info = {l: z[f"prim_info_{l}"] for l in range(3)}
    aoinds = {l: z[f"prim_aoinds_{l}"] for l in range(3)}
    count = {l: info[l].shape[1] for l in range(3)}
    return info, aoinds, count


def j_args(z, cls):
    ab, cd = cls[:2], cls[2:]
    return dict(
        ab_first=z[f"J_{ab}_first"], ab_second=z[f"J_{ab}_second"], ab_pdata=z[f"J_{ab}_pdata"],
        ab_Q=z[f"J_{ab}_Q"],
        cd_first=z[f"J_{cd}_first"], cd_second=z[f"J_{cd}_second"], cd_pdata=z[f"J_{cd}_pdata"],
        cd_Q=z[f"J_{cd}_Q"], cd_D=z[f"J_{cd}_D"],
    )


def k_args(z, cls):
    a, b, c, d = cls
    return dict(
        pair_i=z[f"K_{a}{c}_pair_i"], pair_k=z[f"K_{a}{c}_pair_k"], maxD=float(z[f"K_{cls}_maxD"][0]),
        D_AO=z["D_AO"],
        Q_ab=z[f"K_{a}{b}_Q"], Q_cd=z[f"K_{c}{d}_Q"], Dinds_ab=z[f"K_{a}{b}_Dinds"], Dinds_cd=z[f"K_{c}{d}_Dinds"],
        displs_ab=z[f"K_{a}{b}_displs"], displs_cd=z[f"K_{c}{d}_displs"],
        counts_ab=z[f"K_{a}{b}_counts"], counts_cd=z[f"K_{c}{d}_counts"],
        pdata_ab=z[f"K_{a}{b}_pdata"], pdata_cd=z[f"K_{c}{d}_pdata"],
    )


# variants of the K fixture: (tag, threshold, omega, number of leading rows or None)
K_VARIANTS = (("t12", 1e-12, 0.0, None), ("t3", 2e-3, 0.0, None), ("w3", 1e-12, 0.3, 6))
