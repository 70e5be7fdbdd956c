"""QC/MM electrostatics in the oracle (CPU): with the MM charges put on the nuclei the electron-charge
potentials equal the electron-nuclear attraction that the reference fixtures pin; the analytic
gradients of tr(P V_mm) (atoms and charges) and of the nucleus-charge energy match central finite
differences."""
import numpy as np
import pytest

import oracle
from conftest import ANGSTROM_TO_BOHR, load_golden
from pdynamo3_b200.basis import ShellTable


def _oracle(g, ghost=False):
    sh = ShellTable("6-31g_st_cart", g["Z"])
    if ghost:  # the same shells on atoms without nuclear charge: H = T
        sh.nuclear_charges = np.zeros_like(np.asarray(sh.nuclear_charges, dtype=np.float64))
    return oracle.Oracle(sh, g["xyz"] * ANGSTROM_TO_BOHR)


def _charges(seed=3, n=5):
    rng = np.random.default_rng(seed)
    q = rng.uniform(-0.9, 0.9, n)
    x = rng.uniform(-6.0, 6.0, (n, 3))
    x[np.linalg.norm(x, axis=1) < 3.5] *= 2.0  # keep them off the molecule
    return q, x


def _trace(P, V, n):
    w = np.full(len(P), 2.0)
    w[np.cumsum(np.arange(1, n + 1)) - 1] = 1.0
    return float(np.sum(w * P * V))


def test_potentials_on_nuclei_equal_nuclear_attraction():
    g = load_golden("hf_water1_cart")
    x = g["xyz"] * ANGSTROM_TO_BOHR
    o = _oracle(g, ghost=True)
    _, T, _ = o.one_electron()
    o.set_point_charges(np.asarray(g["Z"], dtype=np.float64), x)
    Vmm = o.qcmm_potentials()
    o = _oracle(g)
    _, H, _ = o.one_electron()
    assert np.abs(H - g["H"]).max() < 1e-10          # the pinned core Hamiltonian
    assert np.abs((T + Vmm) - H).max() < 1e-11


def test_potential_gradients_match_finite_differences():
    g = load_golden("hf_water1_cart")
    x = g["xyz"] * ANGSTROM_TO_BOHR
    P = g["P"]
    q, cx = _charges()
    o = _oracle(g)
    n = o.n
    o.set_point_charges(q, cx)
    gq, gm = o.qcmm_gradients(P)
    h = 1e-4
    for (kind, i, k) in [("mm", 0, 0), ("mm", 3, 2), ("qc", 0, 1), ("qc", 2, 0)]:
        e = []
        for s in (+1, -1):
            xs, cs = x.copy(), cx.copy()
            if kind == "mm":
                cs[i, k] += s * h
            else:
                xs[i, k] += s * h
            oracle.lib().orc_geometry(np.ascontiguousarray(xs.reshape(-1)))
            o.set_point_charges(q, cs)
            e.append(_trace(P, o.qcmm_potentials(), n))
        fd = (e[0] - e[1]) / (2 * h)
        an = gm[i, k] if kind == "mm" else gq[i, k]
        assert abs(fd - an) < 1e-7 * max(1.0, abs(an)), (kind, i, k, fd, an)
    oracle.lib().orc_geometry(np.ascontiguousarray(x.reshape(-1)))


def test_core_energy_and_gradients():
    g = load_golden("hf_water1_cart")
    x = g["xyz"] * ANGSTROM_TO_BOHR
    q, cx = _charges(seed=5, n=4)
    o = _oracle(g)
    o.set_point_charges(q, cx)
    e, gq, gm = o.qcmm_core()
    Z = np.asarray(g["Z"], dtype=np.float64)
    d = x[:, None, :] - cx[None, :, :]
    r = np.linalg.norm(d, axis=2)
    assert abs(e - np.sum(Z[:, None] * q[None, :] / r)) < 1e-12
    ref_gq = -np.sum((Z[:, None] * q[None, :] / r ** 3)[:, :, None] * d, axis=1)
    ref_gm = np.sum((Z[:, None] * q[None, :] / r ** 3)[:, :, None] * d, axis=0)
    assert np.abs(gq - ref_gq).max() < 1e-12
    assert np.abs(gm - ref_gm).max() < 1e-12
