"""GPU parity for the HF path through the C-ABI: one-electron, two-electron Fock, gradients, SCF.

Tolerances: integrals and Fock matrices to 1e-10 (absolute, hartree); gradients to 1e-8 hartree/bohr;
converged energies to 1e-8 hartree (the plain FP64 target) against fixtures made by the reference.
"""
import numpy as np
import pytest

import oracle
from conftest import ANGSTROM_TO_BOHR, HARTREE_TO_KJMOL, load_golden
from pdynamo3_b200 import geometry
from pdynamo3_b200.basis import ShellTable

pytestmark = pytest.mark.gpu


def make_ctx(g):
    from pdynamo3_b200.lib import Context
    ctx = Context(0)
    ctx.set_basis(ShellTable("6-31g_st_cart", g["Z"]))
    ctx.set_geometry(g["xyz"] * ANGSTROM_TO_BOHR)
    return ctx


@pytest.fixture(scope="module", params=["hf_water1_cart", "hf_water4_s0_cart"])
def case(request, cuda_device):
    g = load_golden(request.param)
    return g, make_ctx(g)


def test_one_electron(case):
    g, ctx = case
    S, H, enuc = ctx.one_electron()
    assert np.abs(S - g["S"]).max() < 1e-10
    assert np.abs(H - g["H"]).max() < 1e-9
    assert abs(enuc - g["report_QC_Core_Core"]) < 1e-10


@pytest.mark.parametrize("tag,cx,doj", [("cx1", 1.0, 1), ("cx0.2", 0.2, 1), ("cx0", 0.0, 1), ("rand_cx1", 1.0, 1),
                                        ("rand_cx0.2", 0.2, 1), ("rand_cx0", 0.0, 1)])
def test_fock_two_electron(case, tag, cx, doj):
    g, ctx = case
    P = g["Prand"] if tag.startswith("rand") else g["P"]
    F, e2 = ctx.fock_two_electron(P, cx, doj)
    assert np.abs(F - g["F2_" + tag]).max() < 1e-10
    assert abs(e2 - g["E2_" + tag]) < 1e-9


def test_gradients(case):
    g, ctx = case
    grad = ctx.gradients(g["P"], g["W"], 1.0, True)
    ref = g["gradients_kjmol_A"] / (HARTREE_TO_KJMOL * ANGSTROM_TO_BOHR)
    assert np.abs(grad - ref).max() < 1e-8


def test_scf_energy_and_gradient(case):
    g, ctx = case
    P, res = ctx.scf(density_tolerance=1e-10, energy_tolerance=1e-9, maximum_iterations=100)
    assert res.converged
    E_ref = float(g["energy_kjmol"]) / HARTREE_TO_KJMOL
    assert abs(res.energy_total - E_ref) < 1e-8
    grad = ctx.scf_gradients()
    ref = g["gradients_kjmol_A"] / (HARTREE_TO_KJMOL * ANGSTROM_TO_BOHR)
    assert np.abs(grad - ref).max() < 1e-7
    W = ctx.scf_weighted_density()
    assert np.abs(W - g["W"]).max() < 1e-6


def test_random_geometry_against_oracle(cuda_device):
    z, xyz = geometry.water_cluster(2, 4.0, 123)
    sh = ShellTable("6-31g_st_cart", z)
    from pdynamo3_b200.lib import Context
    ctx = Context(0)
    ctx.set_basis(sh)
    ctx.set_geometry(xyz * ANGSTROM_TO_BOHR)
    o = oracle.Oracle(sh, xyz * ANGSTROM_TO_BOHR)
    S, H, enuc = o.one_electron()
    Sg, Hg, eg = ctx.one_electron()
    assert np.abs(S - Sg).max() < 1e-12 and np.abs(H - Hg).max() < 1e-11
    rng = np.random.default_rng(3)
    a = rng.normal(size=(o.n, o.n))
    P = (a + a.T)[np.tril_indices(o.n)] * 0.05
    F, e2, _ = o.fock(P, 0.6)
    Fg, e2g = ctx.fock_two_electron(P, 0.6, True)
    assert np.abs(F - Fg).max() < 1e-11
    W = (a @ a.T)[np.tril_indices(o.n)] * 0.01
    go = o.gradients(P, W, 0.6)
    gg = ctx.gradients(P, W, 0.6, True)
    assert np.abs(go - gg).max() < 1e-10


def test_diis_history_bounds(cuda_device):
    """The DIIS history is batched into one reduction of at most 16 products: 16 runs, a longer
    history is refused with PDG_ERR_ARG before any device work."""
    from pdynamo3_b200.lib import PDGError
    g = load_golden("hf_water1_cart")
    ctx = make_ctx(g)
    P, res = ctx.scf(density_tolerance=1e-10, energy_tolerance=1e-9, maximum_history=16)
    assert res.converged and abs(res.energy_total - float(g["energy_kjmol"]) / HARTREE_TO_KJMOL) < 1e-8
    with pytest.raises(PDGError, match="maximum_history"):
        ctx.scf(maximum_history=20)
    ctx.close()


def test_non_finite_inputs_fail_with_pdg_err_nan_and_the_context_stays_usable(cuda_device):
    """A non-finite coordinate is refused at the boundary and a non-finite guess density ends the SCF
    with PDG_ERR_NAN (the 'injected NaN density' failure case); the same context then runs a normal
    SCF to the reference energy."""
    from pdynamo3_b200.lib import PDG_ERR_NAN, PDGError
    g = load_golden("hf_water1_cart")
    ctx = make_ctx(g)
    bad = g["xyz"] * ANGSTROM_TO_BOHR
    bad = bad.copy()
    bad[0, 0] = np.nan
    with pytest.raises(PDGError) as err:
        ctx.set_geometry(bad)
    assert err.value.status == PDG_ERR_NAN
    ctx.set_geometry(g["xyz"] * ANGSTROM_TO_BOHR)
    P = np.array(g["P"], dtype=np.float64)
    P[3] = np.nan
    with pytest.raises(PDGError) as err:
        ctx.scf(guess=P, density_tolerance=1e-10)
    assert err.value.status == PDG_ERR_NAN
    P2, res = ctx.scf(density_tolerance=1e-10, energy_tolerance=1e-9)
    assert res.converged and abs(res.energy_total - float(g["energy_kjmol"]) / HARTREE_TO_KJMOL) < 1e-8
    ctx.close()


def test_eri_autotuner_keeps_results(cuda_device):
    """The tile autotuner picks one of its lanes tables per class pair and the Fock matrices built
    afterwards still match the reference's to 1e-10."""
    g = load_golden("hf_water4_s0_cart")
    ctx = make_ctx(g)
    ctx.fock_two_electron(g["P"], 1.0, True)
    chosen = ctx.autotune_eri()
    assert chosen and set(chosen.values()) <= {0, 1, 2, 3, 4}
    F, e2 = ctx.fock_two_electron(g["P"], 1.0, True)
    assert np.abs(F - g["F2_cx1"]).max() < 1e-10 and abs(e2 - g["E2_cx1"]) < 1e-9
    ctx.close()


def test_gradient_work_estimate_counts_evaluated_quartets(cuda_device):
    """Before any gradient the gradient's work estimate covers every Schwarz-screened quartet; after
    one it covers only those the gradient kernels evaluated (one-centre quartets and those below
    the Schwarz x |Gamma| cut excluded), so it shrinks but stays positive."""
    g = load_golden("hf_water4_s0_cart")
    ctx = make_ctx(g)
    try:
        _, _, q_jk = ctx.work_estimate("eri_jk")
        f_all, _, q_all = ctx.work_estimate("eri_grad")
        assert q_all == q_jk > 0 and f_all > 0
        ctx.gradients(g["P"], g["W"], 1.0, True)
        f_eval, _, q_eval = ctx.work_estimate("eri_grad")
        assert 0 < q_eval < q_all and 0 < f_eval < f_all
    finally:
        ctx.close()
