"""The oracle's spin-unrestricted HF (numpy restatement over the pinned Fock builders): in the
closed-shell limit it gives the reference's own RHF energy of the water fixture; for the OH radical
its analytic gradient (one-electron terms with W = sum_s P_s F_s P_s, Coulomb from the total
density, exchange per spin) matches central finite differences of its energies."""
import numpy as np

import oracle
from conftest import ANGSTROM_TO_BOHR, HARTREE_TO_KJMOL, load_golden
from pdynamo3_b200.basis import ShellTable


def _jk(o):
    def jk(P):
        return o.fock(P, 0.0, True)[0], -o.fock(P, 2.0, False)[0]
    return jk


def uhf_gradient(o, Pa, Pb, W):
    g = np.zeros(3 * o.natom)
    L = oracle.lib()
    Pt = np.ascontiguousarray(Pa + Pb)
    L.orc_one_electron_gradient(Pt, np.ascontiguousarray(W), g)
    L.orc_eri_gradient(Pt, 0.0, 1, g)
    L.orc_eri_gradient(np.ascontiguousarray(Pa), 2.0, 0, g)
    L.orc_eri_gradient(np.ascontiguousarray(Pb), 2.0, 0, g)
    return g.reshape(-1, 3)


def test_closed_shell_limit_gives_the_reference_energy():
    g = load_golden("hf_water1_cart")
    o = oracle.Oracle(ShellTable("6-31g_st_cart", g["Z"]), g["xyz"] * ANGSTROM_TO_BOHR)
    S, H, enuc = o.one_electron()
    E, Pa, Pb, W, s2 = oracle.uscf(S, H, enuc, _jk(o), 5, 5)
    assert abs(E - float(g["energy_kjmol"]) / HARTREE_TO_KJMOL) < 1e-8
    assert abs(s2) < 1e-8


def test_radical_gradient_matches_finite_differences():
    Z = np.array([8, 1])
    x0 = np.array([[0.0, 0.0, 0.0], [0.1, 0.0, 0.97]]) * ANGSTROM_TO_BOHR
    sh = ShellTable("sto-3g", Z)  # small basis: five oracle SCFs

    def energy(x):
        o = oracle.Oracle(sh, x)
        S, H, enuc = o.one_electron()
        return o, oracle.uscf(S, H, enuc, _jk(o), 5, 4)
    o, (E, Pa, Pb, W, s2) = energy(x0)
    assert 0.75 < s2 < 0.77
    grad = uhf_gradient(o, Pa, Pb, W)
    h = 1e-4
    for (a, k) in [(1, 2), (1, 0)]:
        xp, xm = x0.copy(), x0.copy()
        xp[a, k] += h
        xm[a, k] -= h
        fd = (energy(xp)[1][0] - energy(xm)[1][0]) / (2 * h)
        assert abs(fd - grad[a, k]) < 1e-6, (a, k, fd, grad[a, k])
    assert np.abs(grad.sum(axis=0)).max() < 1e-8
