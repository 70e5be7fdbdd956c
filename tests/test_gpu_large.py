"""Size-independent checks at the benchmark size (PBE/6-31G*, 16 waters, 75x302 grid, 304
functions), where the oracle is too slow to run: the SCF converges; the total gradient sums to zero
(translational invariance of every term, including the grid-weight derivatives); restarting the
SCF from its own converged density reproduces the energy in one or two cycles; the two-electron
energy returned equals 1/2 tr(P F2) of the returned Fock matrix."""
import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR
from pdynamo3_b200 import geometry

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def water16(cuda_device):
    from pdynamo3_b200.qcmodel import GPUQCEngine
    z, x = geometry.water_cluster(16, 8.0, 1000)
    eng = GPUQCEngine(z, orbital_basis="6-31g_st_cart", functional="pbe", grid_accuracy=3, grid=(75, 29),
                      density_tolerance=1e-8)
    r = eng.energy(x * ANGSTROM_TO_BOHR)
    yield eng, x * ANGSTROM_TO_BOHR, r
    eng.close()


def test_scf_converges_and_gradient_is_translation_invariant(water16):
    eng, x, r = water16
    assert r.converged and r.iterations < 40
    assert np.abs(r.gradients.sum(axis=0)).max() < 1e-7
    assert abs(r.report["Quadrature Electron Count"] - 160.0) < 1e-3


def test_restart_from_converged_density_is_idempotent(water16):
    eng, x, r = water16
    r2 = eng.energy(x)   # warm start from r's density
    assert r2.converged and r2.iterations <= 3
    assert abs(r2.energy - r.energy) < 1e-8
    assert np.abs(r2.gradients - r.gradients).max() < 1e-6


def test_two_electron_energy_is_half_trace_of_p_f2(water16):
    eng, x, r = water16
    F2, E2 = eng.ctx.fock_two_electron(r.density, 0.0)
    n = int((np.sqrt(8 * len(F2) + 1) - 1) / 2)
    w = np.full(len(F2), 2.0)
    w[np.cumsum(np.arange(1, n + 1)) - 1] = 1.0     # diagonal entries of the packed triangle
    assert abs(0.5 * np.sum(w * r.density * F2) - E2) < 1e-9 * max(1.0, abs(E2))
