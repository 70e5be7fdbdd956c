"""QC/MM electrostatics with MM point charges on the GPU against the oracle (whose electron-charge
integrals are the pinned electron-nuclear ones with the charges moved, tests/test_qcmm_oracle.py):
potentials to 1e-11, their gradients (QC atoms and charges) to 1e-10 hartree/bohr, the
nucleus-charge term to 1e-11; an HF SCF in the field of the charges gives the oracle's SCF energy in
the same field to 1e-8 hartree, and the total energy's derivative with respect to a charge position
matches a central finite difference of SCF energies to 1e-6 hartree/bohr."""
import numpy as np
import pytest

import oracle
from conftest import ANGSTROM_TO_BOHR, load_golden
from pdynamo3_b200.basis import ShellTable

pytestmark = pytest.mark.gpu


def _charges(n, seed, box=9.0, keep_out=3.5):
    rng = np.random.default_rng(seed)
    q = rng.uniform(-0.9, 0.9, n)
    x = rng.uniform(-box, box, (n, 3))
    r = np.linalg.norm(x, axis=1)
    x[r < keep_out] *= (keep_out + 1.0) / np.maximum(r[r < keep_out], 0.5)[:, None]
    return q, x


def _pair(g, q, x, functional=None):
    from pdynamo3_b200.lib import Context
    xyz = g["xyz"] * ANGSTROM_TO_BOHR
    sh = ShellTable("6-31g_st_cart", g["Z"])
    ctx = Context(0)
    ctx.set_basis(sh)
    ctx.set_geometry(xyz)
    ctx.set_point_charges(q, x)
    o = oracle.Oracle(sh, xyz)
    o.set_point_charges(q, x)
    return ctx, o


@pytest.mark.parametrize("n,seed", [(5, 3), (300, 11)])
def test_potentials_gradients_and_core_match_oracle(cuda_device, n, seed):
    g = load_golden("hf_water1_cart")
    q, x = _charges(n, seed)
    ctx, o = _pair(g, q, x)
    try:
        V = ctx.qcmm_potentials()
        assert np.abs(V - o.qcmm_potentials()).max() < 1e-11
        gq, gm = ctx.qcmm_gradients(g["P"])
        oq, om = o.qcmm_gradients(g["P"])
        assert np.abs(gq - oq).max() < 1e-10
        assert np.abs(gm - om).max() < 1e-10
        e, cq, cm = ctx.qcmm_core()
        oe, oq2, om2 = o.qcmm_core()
        assert abs(e - oe) < 1e-11 * max(1.0, abs(oe))
        assert np.abs(cq - oq2).max() < 1e-10 and np.abs(cm - om2).max() < 1e-10
        # the core Hamiltonian carries the potentials while the charges are set
        S, H, _ = ctx.one_electron()
        S0, H0, _ = o.one_electron()
        assert np.abs(H - (H0 + o.qcmm_potentials())).max() < 1e-10
    finally:
        ctx.close()


def test_scf_in_the_field_matches_oracle_and_finite_differences(cuda_device):
    g = load_golden("hf_water1_cart")
    q, x = _charges(6, 5)
    ctx, o = _pair(g, q, x)
    try:
        P, r = ctx.scf(density_tolerance=1e-10, energy_tolerance=1e-10, maximum_iterations=100)
        assert r.converged
        S, H, enuc = o.one_electron()
        E, Po, W, it = oracle.scf(S, H + o.qcmm_potentials(), enuc, lambda p: o.fock(p, 1.0)[:2], nocc=5)
        assert abs(r.energy_total - E) < 1e-8
        # d(E_scf + E_core)/dx_c: electronic part from the converged density, core part analytic
        gq, gm = ctx.qcmm_gradients()
        _, cq, cm = ctx.qcmm_core()
        c, k, h = 2, 1, 1e-4
        es = []
        for s in (+1, -1):
            xs = x.copy()
            xs[c, k] += s * h
            ctx.set_point_charges(q, xs)
            _, rs = ctx.scf(density_tolerance=1e-10, energy_tolerance=1e-10, maximum_iterations=100)
            assert rs.converged
            es.append(rs.energy_total + ctx.qcmm_core(gradients=False))
        fd = (es[0] - es[1]) / (2 * h)
        assert abs(fd - (gm[c, k] + cm[c, k])) < 1e-6
    finally:
        ctx.close()
