"""The oracle (CPU restatement) against fixtures produced by the pDynamo3 reference itself."""
import numpy as np
import pytest

import oracle
from conftest import ANGSTROM_TO_BOHR, HARTREE_TO_KJMOL, load_golden
from pdynamo3_b200.basis import ShellTable


@pytest.fixture(scope="module")
def water1():
    g = load_golden("hf_water1_cart")
    o = oracle.Oracle(ShellTable("6-31g_st_cart", g["Z"]), g["xyz"] * ANGSTROM_TO_BOHR)
    return g, o


def test_one_electron_matches_reference(water1):
    g, o = water1
    S, H, enuc = o.one_electron()
    assert np.abs(S - g["S"]).max() < 1e-11
    assert np.abs(H - g["H"]).max() < 1e-10
    assert abs(enuc - g["report_QC_Core_Core"]) < 1e-11


@pytest.mark.parametrize("tag,cx", [("cx1", 1.0), ("cx0.2", 0.2), ("cx0", 0.0), ("rand_cx1", 1.0), ("rand_cx0.2", 0.2),
                                    ("rand_cx0", 0.0)])
def test_fock_matches_reference(water1, tag, cx):
    g, o = water1
    P = g["Prand"] if tag.startswith("rand") else g["P"]
    F, e2, count = o.fock(P, cx)
    assert np.abs(F - g["F2_" + tag]).max() < 1e-11
    assert abs(e2 - g["E2_" + tag]) < 1e-10
    assert count == int(g["report_TEI_Number"])


def test_gradients_match_reference(water1):
    g, o = water1
    grad = o.gradients(g["P"], g["W"])
    ref = g["gradients_kjmol_A"] / (HARTREE_TO_KJMOL * ANGSTROM_TO_BOHR)
    assert np.abs(grad - ref).max() < 1e-10


def test_scf_energy_matches_reference(water1):
    g, o = water1
    S, H, enuc = o.one_electron()
    E, P, W, it = oracle.scf(S, H, enuc, lambda p: o.fock(p, 1.0)[:2], nocc=5)
    assert abs(E - float(g["energy_kjmol"]) / HARTREE_TO_KJMOL) < 1e-8


def test_rys_rule_exact_on_moments():
    # The n-point rule integrates u^k exp(-x u) (du / 2 sqrt(u)) exactly for k <= 2n-1 (Boys moments).
    from math import erf, exp, pi, sqrt
    for n in range(1, 8):
        for x in (0.0, 0.3, 2.7, 11.0, 37.5, 150.0):
            u, w = oracle.rys_roots(n, x)
            # F_0(x) and upward recursion F_{k+1} = ((2k+1) F_k - exp(-x)) / (2x) (stable for x >= 10)
            if x == 0.0:
                F = [1.0 / (2 * k + 1) for k in range(2 * n)]
            elif x >= 10.0:
                F = [0.5 * sqrt(pi / x) * erf(sqrt(x))]
                for k in range(2 * n - 1):
                    F.append(((2 * k + 1) * F[-1] - exp(-x)) / (2 * x))
            else:
                continue
            for k in range(2 * n):
                approx = float(np.sum(w * u ** k))
                assert abs(approx - F[k]) <= 1e-13 * max(1.0, abs(F[k])) + 1e-300


@pytest.mark.skipif(not oracle.reference_roots_available(), reason="reference libcint build (oracle/_ref) absent")
def test_rys_rule_matches_reference_libcint():
    # The reference's own Rys routine (RysQuadrature.c:33-36 -> libcint CINTrys_roots), compiled from
    # its sources by oracle/build_ref.sh, against the restated rule over the root counts the energy
    # (<= 5) and gradient (<= 6) passes use and arguments spanning every branch of the fitted formulas.
    for n in range(1, 8):
        for x in (0.0, 1e-9, 1e-3, 0.3, 1.0, 2.9, 3.1, 5.5, 9.9, 10.1, 15.0, 23.0, 33.0, 36.0, 45.0, 49.9, 80.0, 250.0):
            u, w = oracle.rys_roots(n, x)
            ur, wr = oracle.reference_rys_roots(n, x)
            o = np.argsort(ur)
            assert np.abs(ur[o] - u).max() <= 1e-11 * max(1.0, np.abs(u).max())
            assert np.abs(wr[o] - w).max() <= 1e-11 * np.abs(w).max()


@pytest.mark.skipif(not oracle.reference_roots_available(), reason="reference libcint build (oracle/_ref) absent")
def test_fock_with_reference_roots_matches_reference(water1):
    g, o = water1
    try:
        assert oracle.use_reference_roots(True)
        F, E2 = o.fock(g["P"], 1.0)[:2]
    finally:
        oracle.use_reference_roots(False)
    assert np.abs(F - g["F2_cx1"]).max() < 1e-10
    assert abs(E2 - float(g["E2_cx1"])) < 1e-10


def test_stored_integral_digest_matches_the_direct_digest_and_the_reference():
    """The stored-integral mode (integrals once, one digest per SCF cycle, as the reference's
    conventional SCF) gives the same Fock matrices as the direct digest and the reference's, and
    stores the reference's number of integrals."""
    g = load_golden("hf_water4_s0_cart")
    sh = ShellTable("6-31g_st_cart", g["Z"])
    o = oracle.Oracle(sh, g["xyz"] * ANGSTROM_TO_BOHR)
    n = o.store_integrals()
    assert n == int(g["report_TEI_Number"])
    try:
        for tag, cx in (("cx1", 1.0), ("rand_cx0.2", 0.2)):
            P = g["Prand"] if tag.startswith("rand") else g["P"]
            F, e2 = o.fock_stored(P, cx)
            Fd, e2d, _ = o.fock(P, cx)
            assert np.abs(F - Fd).max() < 1e-12 and abs(e2 - e2d) < 1e-10
            assert np.abs(F - g["F2_" + tag]).max() < 1e-11
    finally:
        o.free_stored()
