"""The ctypes mirror of VlxbBatchCall (vlxb.batchfuse) against include/vlxb.h."""
import ctypes
import re

from vlxb.batchfuse import VlxbBatchCall


def test_batch_struct_matches_header():
    """The ctypes mirror has the header's fields in the header's order."""
    import os
    hdr = open(os.path.join(os.path.dirname(__file__), "..", "include", "vlxb.h")).read()
    body = hdr[hdr.index("typedef struct {"):hdr.index("} VlxbBatchCall;")]
    names = []
    for line in body.splitlines()[1:]:
        line = line.split("/*")[0].strip()
        if not line:
            continue
        decl = line.rstrip(";").split(None, 1)[1] if not line.startswith("const") else line.rstrip(";")
        for part in decl.split(","):
            nm = re.sub(r"\[.*\]", "", part.replace("const", "").replace("*", " ")).split()[-1]
            names.append(nm)
    assert names == [f[0] for f in VlxbBatchCall._fields_]
    assert ctypes.sizeof(VlxbBatchCall) > 0


def test_union_lists_slices_are_the_molecules_lists():
    """Each molecule's slice of the union lists, with its primitive offsets
    removed, is its own reference-format lists; the density stack holds every
    molecule's block."""
    import numpy as np

    import helpers
    from test_lists_host import tiny_molecule
    from vlxb import lists
    from vlxb.batchfuse import union_lists
    from vlxb.lists import LV, NCART

    rls = []
    for seed in (1, 2, 3):
        mol, D = tiny_molecule(seed=seed)
        rls.append(lists.build_lists(mol, D, 1e-12, helpers.oracle_schwarz_fn))
    u = union_lists(rls)
    h, poff = u["arrays"], u["poff"]
    for key in u["jkeys"]:
        la, lb = LV[key[0]], LV[key[1]]
        for m, rl in enumerate(rls):
            s0, s1 = u["jslices"][key][m]
            jl = rl.jlists[key]
            first = h[f"j_{key}_first"][s0:s1].astype(np.int64) - poff[la][m] * NCART[la]
            second = h[f"j_{key}_second"][s0:s1].astype(np.int64) - poff[lb][m] * NCART[lb]
            assert np.array_equal(first, jl.first) and np.array_equal(second, jl.second)
            assert np.array_equal(h[f"j_{key}_D"][s0:s1], jl.D)
    for key in u["kpkeys"]:
        la, lb = LV[key[0]], LV[key[1]]
        c = h[f"kp_{key}_counts"].astype(np.int64)
        dsp = h[f"kp_{key}_displs"].astype(np.int64)
        for m, rl in enumerate(rls):
            kp = rl.kpartners[key]
            f0 = poff[la][m] * NCART[la]
            n = len(kp.counts)
            assert np.array_equal(c[f0:f0 + n], kp.counts)
            for i in range(n):
                a = dsp[f0 + i]
                got = h[f"kp_{key}_Dinds"][a:a + c[f0 + i]].astype(np.int64) - poff[lb][m] * NCART[lb]
                assert np.array_equal(got, kp.Dinds[kp.displs[i]:kp.displs[i] + kp.counts[i]])
    for m, rl in enumerate(rls):
        a0 = u["ao0"][m]
        assert np.array_equal(h["Dstack"][a0:a0 + rl.naos, :rl.naos], rl.D_AO)
        assert np.all(h["mol0"][poff[0][m]:poff[0][m + 1]] == m)


def test_fused_groups_split_and_map_molecules(monkeypatch):
    """FusedBatchGroups splits a batch into unions of at most `group`
    molecules in order and maps every molecule to its union and its index
    there (the unions themselves replaced by a recording stand-in)."""
    import pytest

    from vlxb import batchfuse

    made = []

    class Stub:
        def __init__(self, mols, dens, thr, device="cuda", **kw):
            self.nmol = len(mols)
            self.mols = list(mols)
            made.append(self)

        def results(self, m):
            return self.mols[m]

        def nbytes(self):
            return 10 * self.nmol

    monkeypatch.setattr(batchfuse, "FusedBatch", Stub)
    mols = [f"m{t}" for t in range(7)]
    fg = batchfuse.FusedBatchGroups(mols, [None] * 7, 1e-12, device="cpu", group=3)
    assert [p.nmol for p in made] == [3, 3, 1] and fg.nmol == 7
    assert [fg.results(t) for t in range(7)] == mols
    assert fg.where[4] == (1, 1) and fg.nbytes() == 70
    with pytest.raises(ValueError):
        batchfuse.FusedBatchGroups(mols, [None] * 7, 1e-12, device="cpu", group=0)
