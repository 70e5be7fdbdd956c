"""Spin-unrestricted Hartree-Fock on the device against the oracle's unrestricted restatement
(tests/test_uhf_oracle.py pins it): the NH2 radical (HF/6-31G*) energy to 1e-8 hartree, <S^2> to
1e-6, the spin densities to 1e-6 and the analytic gradient to 1e-6 hartree/bohr; the closed-shell
limit gives the restricted energy; a density functional is refused."""
import numpy as np
import pytest

import oracle
from conftest import ANGSTROM_TO_BOHR, load_golden
from pdynamo3_b200.basis import ShellTable
from test_uhf_oracle import _jk, uhf_gradient

pytestmark = pytest.mark.gpu


def _ctx(Z, x, functional=None):
    from pdynamo3_b200.lib import Context
    ctx = Context(0)
    ctx.set_basis(ShellTable("6-31g_st_cart", Z))
    ctx.set_geometry(x)
    if functional:
        ctx.set_functional(functional)
    return ctx


def test_radical_energy_spin_and_gradient_match_oracle(cuda_device):
    # NH2 (2B1, bent: a non-degenerate ground state, so the spin densities are unique)
    a = np.deg2rad(103.0) / 2
    Z = np.array([7, 1, 1])
    x = np.array([[0.0, 0.0, 0.0], [1.024 * np.sin(a), 0.0, 1.024 * np.cos(a)],
                  [-1.024 * np.sin(a), 0.0, 1.024 * np.cos(a)]]) * ANGSTROM_TO_BOHR
    ctx = _ctx(Z, x)
    try:
        Pa, Pb, r = ctx.uscf(5, 4, density_tolerance=1e-10, energy_tolerance=1e-10, maximum_iterations=200)
        assert r.converged
        g = ctx.scf_gradients()
    finally:
        ctx.close()
    o = oracle.Oracle(ShellTable("6-31g_st_cart", Z), x)
    S, H, enuc = o.one_electron()
    E, oPa, oPb, W, s2 = oracle.uscf(S, H, enuc, _jk(o), 5, 4)
    assert abs(r.energy_total - E) < 1e-8
    assert abs(r.s2 - s2) < 1e-6
    assert np.abs(Pa - oPa).max() < 1e-6 and np.abs(Pb - oPb).max() < 1e-6
    assert np.abs(g - uhf_gradient(o, oPa, oPb, W)).max() < 1e-6


def test_closed_shell_limit_equals_restricted(cuda_device):
    gd = load_golden("hf_water1_cart")
    x = gd["xyz"] * ANGSTROM_TO_BOHR
    ctx = _ctx(gd["Z"], x)
    try:
        _, r = ctx.scf(density_tolerance=1e-10, energy_tolerance=1e-10)
        g_r = ctx.scf_gradients()
        _, _, u = ctx.uscf(5, 5, density_tolerance=1e-10, energy_tolerance=1e-10)
        g_u = ctx.scf_gradients()
    finally:
        ctx.close()
    assert abs(u.energy_total - r.energy_total) < 1e-8
    assert abs(u.s2) < 1e-8
    assert np.abs(g_u - g_r).max() < 1e-7


def test_unrestricted_kohn_sham_is_refused(cuda_device):
    from pdynamo3_b200.lib import PDGError
    ctx = _ctx(np.array([8, 1]), np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.83]]), functional="pbe")
    try:
        with pytest.raises(PDGError):
            ctx.uscf(5, 4)
    finally:
        ctx.close()


def test_engine_with_multiplicity_runs_unrestricted_and_warm_starts(cuda_device):
    from pdynamo3_b200.qcmodel import GPUQCEngine
    a = np.deg2rad(103.0) / 2
    Z = np.array([7, 1, 1])
    x = np.array([[0.0, 0.0, 0.0], [1.024 * np.sin(a), 0.0, 1.024 * np.cos(a)],
                  [-1.024 * np.sin(a), 0.0, 1.024 * np.cos(a)]]) * ANGSTROM_TO_BOHR
    ctx = _ctx(Z, x)
    try:
        _, _, ref = ctx.uscf(5, 4, density_tolerance=1e-10, energy_tolerance=1e-10, maximum_iterations=200)
        g_ref = ctx.scf_gradients()
    finally:
        ctx.close()
    eng = GPUQCEngine(Z, orbital_basis="6-31g_st_cart", functional="hf", multiplicity=2,
                      density_tolerance=1e-10, energy_tolerance=1e-10, maximum_iterations=200)
    try:
        r = eng.energy(x)
        assert r.converged and abs(r.energy - ref.energy_total) < 1e-8
        assert np.abs(r.gradients - g_ref).max() < 1e-7
        assert abs(r.report["<S^2>"] - ref.s2) < 1e-8
        r2 = eng.energy(x)   # warm start from its own spin densities
        assert r2.converged and r2.iterations <= 3 and abs(r2.energy - r.energy) < 1e-9
    finally:
        eng.close()
    with pytest.raises(NotImplementedError):
        GPUQCEngine(Z, orbital_basis="6-31g_st_cart", functional="pbe", multiplicity=2)
