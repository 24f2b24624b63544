"""On-device prim-pair -> AO contraction (vlxb_pairsToAO) and energy
(vlxb_fockEnergy) against the host contraction of the same GPU build, and the
end-to-end AO J/K against the FP64 oracle."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import helpers
from vlxb import aomap, basis, fock, lists
from vlxb._lib import lib

pytestmark = pytest.mark.gpu


def _system(seed=2, atoms=4):
    wl = basis.config_custom(atoms, 4.5, {0: 2, 1: 1, 2: 1}, 2, 0.3, 2.5, 4, 1e-12, seed)
    rl = lists.build_lists(wl.mol, wl.D, wl.threshold, fock.gpu_schwarz_fn())
    return wl, rl


def test_device_ao_contraction_and_energy():
    lib().init(0)
    wl, rl = _system()
    dl = fock.to_device(rl)
    am = aomap.AOMap(rl)
    fj, mJ, fk, mK = am.alloc_outputs()
    fock.build_jk(dl, matJ=mJ, matK=mK)
    Jd = am.to_ao("J", fj)
    Kd = am.to_ao("K", fk)
    e = aomap.energy(dl.D_AO, Jd, Kd)
    torch.cuda.synchronize()
    Jh = lists.contract_J(rl, {k: v.cpu().numpy() for k, v in mJ.items()})
    Kh = lists.contract_K(rl, {k: v.cpu().numpy() for k, v in mK.items()})
    Jg, Kg = Jd.cpu().numpy(), Kd.cpu().numpy()
    assert np.array_equal(Jg, Jg.T) and np.array_equal(Kg, Kg.T)
    assert np.abs(Jg - Jh).max() <= 1e-13 * np.abs(Jh).max()
    assert np.abs(Kg - Kh).max() <= 1e-13 * np.abs(Kh).max()
    E = e.cpu().numpy()
    Eh = lists.energy(wl.D, Jh, Kh)
    assert abs(E[0] - Eh) <= 1e-12 * max(1.0, abs(Eh))
    assert abs(E[1] - float(np.sum(wl.D * Jh))) <= 1e-12 * max(1.0, abs(E[1]))
    assert abs(E[2] - float(np.sum(wl.D * Kh))) <= 1e-12 * max(1.0, abs(E[2]))
    # J-only energy term with K = NULL
    e2 = aomap.energy(dl.D_AO, Jd, None)
    assert abs(float(e2[0].item()) - E[1]) <= 1e-13 * max(1.0, abs(E[1]))
    # bit-reproducible run to run
    Jd2 = am.to_ao("J", fj)
    assert torch.equal(Jd, Jd2)
    # against the oracle's AO J and K
    oJ, oK = helpers.oracle_jk_all(rl)
    Jo, Ko = lists.contract_J(rl, oJ), lists.contract_K(rl, oK)
    assert np.abs(Jg - Jo).max() <= 1e-10 * max(1.0, np.abs(Jo).max())
    assert np.abs(Kg - Ko).max() <= 1e-10 * max(1.0, np.abs(Ko).max())


def test_invalid_arguments():
    L = lib()
    L.init(0)
    out = torch.zeros((3, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(Exception):
        L.pairs_to_ao(0, 0, 0, 0, 5, out.data_ptr(), 3, 0)  # rows without arrays
    with pytest.raises(Exception):
        L.fock_energy(0, 0, 0, 3, out.data_ptr(), 0)  # no density
