"""GPU parity at the benchmarked configurations, against fixtures the reference itself produced
(tests/golden/make_golden.py over the reference built by tests/golden/build_reference.sh).

* The default benchmark's first geometry: PBE/6-31G* (Cartesian) on 16 waters, on the reference's
  Medium grid and on the 75 radial x 302 Lebedev override, run through the drop-in engine with the
  benchmark's own settings (difference Fock builds with the 1e-13 density screen, the Schwarz x
  |Gamma| gradient screen, SCF to 1e-8 in the density).
* The reference's shipped, spherical 6-31G*: HF on 4 waters (one-electron matrices, two-electron
  Fock matrices of the converged and a random density for c_x = 1, 0.2, 0, energy, gradient) and
  B3LYP on 2 waters (quadrature Fock, energy, gradient).
* Two molecules of the organic batch (B3LYP/6-31G*, Medium grid) with the batch's settings, in
  FP64 and in the mixed-precision mode.

Tolerances (stated per result): FP64 energies 1e-8 hartree, gradients 1e-6 hartree/A; matrices
1e-10 (Fock) and 1e-9 (quadrature Fock); mixed precision 1e-5 hartree and 1e-4 hartree/A.
"""
import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR, HARTREE_TO_KJMOL, load_golden
from pdynamo3_b200.basis import ShellTable

pytestmark = pytest.mark.gpu

E_TOL, G_TOL = 1e-8, 1e-6            # hartree, hartree/A (plain FP64)
E_TOL_MIXED, G_TOL_MIXED = 1e-5, 1e-4  # hartree, hartree/A (mixed precision)


def ref_energy(g):
    return float(g["energy_kjmol"]) / HARTREE_TO_KJMOL


def ref_gradient_per_angstrom(g):
    return g["gradients_kjmol_A"] / HARTREE_TO_KJMOL


def engine(g, functional, basis="6-31g_st_cart", grid=None, precision_mode=0):
    from pdynamo3_b200.qcmodel import GPUQCEngine
    e = GPUQCEngine(g["Z"], orbital_basis=basis, functional=functional, grid_accuracy="medium", grid=grid,
                    density_tolerance=1e-8)
    if precision_mode:
        e.ctx.set_eri_options(precision_mode=precision_mode, mixed_cut=1e-6)
    return e


def check(result, g, e_tol, g_tol):
    assert result.converged
    de = abs(result.energy - ref_energy(g))
    dg = np.abs(result.gradients * ANGSTROM_TO_BOHR - ref_gradient_per_angstrom(g)).max()
    assert de < e_tol, de
    assert dg < g_tol, dg
    return de, dg


@pytest.mark.parametrize("name,grid", [("pbe_water16_s1000_cart_75x302", (75, 29)),
                                       ("pbe_water16_s1000_cart_medium", None)])
def test_water16_pbe_with_benchmark_settings(cuda_device, name, grid):
    g = load_golden(name)
    e = engine(g, "pbe", grid=grid)
    try:
        r = e.energy(g["xyz"] * ANGSTROM_TO_BOHR)
        check(r, g, E_TOL, G_TOL)
        # points within rounding of the reference's 1e-30 weight drop may fall either way
        assert abs(r.report["Quadrature Points"] - int(g["grid_points"])) <= max(2, int(2e-4 * int(g["grid_points"])))
    finally:
        e.close()


@pytest.fixture(scope="module")
def water4_spherical(cuda_device):
    from pdynamo3_b200.lib import Context
    g = load_golden("hf_water4_s0_sph")
    ctx = Context(0)
    sh = ShellTable("6-31g_st", g["Z"])
    assert sh.spherical and sh.n_functions() == int(g["n_functions"]) == 72
    ctx.set_basis(sh)
    ctx.set_geometry(g["xyz"] * ANGSTROM_TO_BOHR)
    yield g, ctx
    ctx.close()


def test_spherical_one_electron(water4_spherical):
    g, ctx = water4_spherical
    S, H, enuc = ctx.one_electron()
    assert np.abs(S - g["S"]).max() < 1e-10
    assert np.abs(H - g["H"]).max() < 1e-9
    assert abs(enuc - g["report_QC_Core_Core"]) < 1e-10


@pytest.mark.parametrize("tag,cx", [("cx1", 1.0), ("cx0.2", 0.2), ("cx0", 0.0), ("rand_cx1", 1.0), ("rand_cx0.2", 0.2),
                                    ("rand_cx0", 0.0)])
def test_spherical_fock_two_electron(water4_spherical, tag, cx):
    g, ctx = water4_spherical
    P = g["Prand"] if tag.startswith("rand") else g["P"]
    F, e2 = ctx.fock_two_electron(P, cx, True)
    assert np.abs(F - g["F2_" + tag]).max() < 1e-10
    assert abs(e2 - g["E2_" + tag]) < 1e-9


def test_spherical_hf_energy_and_gradient(cuda_device):
    g = load_golden("hf_water4_s0_sph")
    e = engine(g, "hf", basis="6-31g_st")
    try:
        r = e.energy(g["xyz"] * ANGSTROM_TO_BOHR)
        check(r, g, E_TOL, G_TOL)
        assert np.abs(r.density - g["P"]).max() < 1e-6
    finally:
        e.close()


def test_spherical_b3lyp_quadrature_energy_and_gradient(cuda_device):
    g = load_golden("b3lyp_water2_sph_medium")
    e = engine(g, "b3lyp", basis="6-31g_st")
    try:
        e.ctx.set_geometry(g["xyz"] * ANGSTROM_TO_BOHR)
        e.ctx.grid_build(3)
        F, exc, rho = e.ctx.fock_quadrature(g["P"])
        assert abs(exc - float(g["Exc"])) < 1e-9 and abs(rho - float(g["RhoQuad"])) < 1e-9
        assert np.abs(F - g["Vxc"]).max() < 1e-9
        r = e.energy(g["xyz"] * ANGSTROM_TO_BOHR)
        check(r, g, E_TOL, G_TOL)
    finally:
        e.close()


@pytest.mark.parametrize("name", ["b3lyp_batch4_cart_medium", "b3lyp_batch19_cart_medium"])
def test_organic_batch_molecules_fp64_and_mixed(cuda_device, name):
    g = load_golden(name)
    for mode, (et, gt) in ((0, (E_TOL, G_TOL)), (1, (E_TOL_MIXED, G_TOL_MIXED))):
        e = engine(g, "b3lyp", precision_mode=mode)
        try:
            r = e.energy(g["xyz"] * ANGSTROM_TO_BOHR)
            check(r, g, et, gt)
            assert r.report["Quadrature Points"] > 0
        finally:
            e.close()
