"""The drop-in engine (pdynamo3_b200.qcmodel.GPUQCEngine) against the reference's own results.

System.Energy(doGradients=True) of the reference (tests/golden, made by make_golden.py) gives the
total energy (kJ/mol), the gradients (kJ/mol/A) and the qcEnergyReport terms.  The engine runs the
same molecule end to end on the GPU (SCF to 1e-10 like the fixtures) and must give the energy to
1e-8 hartree, the gradients to 1e-6 hartree/bohr and the report terms to 1e-7 hartree.
"""
import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR, HARTREE_TO_KJMOL, load_golden

pytestmark = pytest.mark.gpu

CASES = [("hf_water1_cart", "hf", None), ("pbe_water1_cart_low", "pbe", "low"),
         ("blyp_water1_cart_medium", "blyp", "medium"), ("b3lyp_water2_cart_medium", "b3lyp", "medium")]
TERMS = ["QC Core-Core", "One-Electron Energy", "Two-Electron Energy", "Two-Electron Coulomb Energy", "Quadrature Energy"]


def _engine(functional, accuracy, z, **kw):
    from pdynamo3_b200.qcmodel import GPUQCEngine
    return GPUQCEngine(z, orbital_basis="6-31g_st_cart", functional=functional, grid_accuracy=accuracy or "medium",
                       density_tolerance=1e-10, energy_tolerance=1e-9, **kw)


@pytest.mark.parametrize("name,functional,accuracy", CASES, ids=[c[0] for c in CASES])
def test_engine_matches_reference_energy_gradients_and_report(cuda_device, name, functional, accuracy):
    g = load_golden(name)
    eng = _engine(functional, accuracy, g["Z"])
    try:
        r = eng.energy(g["xyz"] * ANGSTROM_TO_BOHR, do_gradients=True)
    finally:
        eng.close()
    assert r.converged
    assert abs(r.energy_kjmol - float(g["energy_kjmol"])) / HARTREE_TO_KJMOL < 1e-8
    dg = r.gradients_kjmol_per_angstrom() - g["gradients_kjmol_A"]
    assert np.abs(dg).max() / (HARTREE_TO_KJMOL * ANGSTROM_TO_BOHR) < 1e-6
    for key in TERMS:
        gk = "report_" + key.replace(" ", "_").replace("-", "_")
        assert (key in r.report) == (gk in g), key
        if gk in g:
            assert abs(r.report[key] - float(g[gk])) < 1e-7, key
    if "report_Quadrature_Points" in g:
        n_ref = int(g["report_Quadrature_Points"])
        assert abs(r.report["Quadrature Points"] - n_ref) <= max(2, int(2e-4 * n_ref))
        assert abs(r.report["Quadrature Electron Count"] - float(g["report_Quadrature_Electron_Count"])) < 1e-6


def test_warm_start_gives_the_cold_result_in_fewer_cycles(cuda_device):
    # an MD-like follow-up: the second geometry starts from the first one's density
    g = load_golden("b3lyp_water2_cart_medium")
    x0 = g["xyz"] * ANGSTROM_TO_BOHR
    x1 = x0 + np.random.default_rng(3).normal(scale=0.01 * ANGSTROM_TO_BOHR, size=x0.shape)
    warm = _engine("b3lyp", "medium", g["Z"])
    cold = _engine("b3lyp", "medium", g["Z"], warm_start=False)
    try:
        warm.energy(x0, do_gradients=False)
        rw = warm.energy(x1)
        rc = cold.energy(x1)
    finally:
        warm.close()
        cold.close()
    assert rw.converged and rc.converged
    assert rw.iterations < rc.iterations
    assert abs(rw.energy - rc.energy) < 1e-8
    assert np.abs(rw.gradients - rc.gradients).max() < 1e-6


def test_engine_rejects_wrong_atom_count(cuda_device):
    g = load_golden("hf_water1_cart")
    eng = _engine("hf", None, g["Z"])
    try:
        with pytest.raises(ValueError):
            eng.energy(np.zeros((2, 3)))
    finally:
        eng.close()


def test_unconverged_cold_scf_is_retried_once_and_reported(cuda_device):
    """An SCF that reaches its iteration limit from a cold start is run once more with complete
    Fock builds and a 16-deep DIIS; if that also stops at the limit the result says so (no gradient)
    and the engine's next energy, with a sane limit, converges as usual."""
    from conftest import ANGSTROM_TO_BOHR, HARTREE_TO_KJMOL, load_golden
    from pdynamo3_b200.qcmodel import GPUQCEngine
    g = load_golden("hf_water4_s0_cart")
    e = GPUQCEngine(g["Z"], orbital_basis="6-31g_st_cart", functional="hf", density_tolerance=1e-10,
                    energy_tolerance=1e-9, maximum_iterations=3, warm_start=False)
    try:
        r = e.energy(g["xyz"] * ANGSTROM_TO_BOHR)
        assert not r.converged and r.gradients is None and r.iterations > 3   # two attempts
        e.options["maximum_iterations"] = 100
        r = e.energy(g["xyz"] * ANGSTROM_TO_BOHR)
        assert r.converged and abs(r.energy - float(g["energy_kjmol"]) / HARTREE_TO_KJMOL) < 1e-8
    finally:
        e.close()


def test_mixed_mode_retry_returns_to_the_mixed_mode(cuda_device):
    """In the mixed mode the last retry runs in FP64; afterwards the context is in the mixed mode
    again: the next energy evaluates FP32 quartets and matches the reference to the mixed mode's
    1e-5 hartree."""
    from conftest import ANGSTROM_TO_BOHR, HARTREE_TO_KJMOL, load_golden
    from pdynamo3_b200.qcmodel import GPUQCEngine
    g = load_golden("hf_water4_s0_cart")
    e = GPUQCEngine(g["Z"], orbital_basis="6-31g_st_cart", functional="hf", density_tolerance=1e-10,
                    energy_tolerance=1e-9, maximum_iterations=3, warm_start=False)
    try:
        e.ctx.set_eri_options(precision_mode=1, mixed_cut=1e-6)
        r = e.energy(g["xyz"] * ANGSTROM_TO_BOHR)
        assert not r.converged and r.iterations > 3
        assert e.ctx.eri_options["precision_mode"] == 1
        n32 = e.ctx.fp32_quartets()
        e.options["maximum_iterations"] = 100
        r = e.energy(g["xyz"] * ANGSTROM_TO_BOHR)
        assert r.converged and abs(r.energy - float(g["energy_kjmol"]) / HARTREE_TO_KJMOL) < 1e-5
        assert e.ctx.fp32_quartets() > n32
    finally:
        e.close()
