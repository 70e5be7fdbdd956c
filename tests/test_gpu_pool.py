"""The GPU process-pool backend on the device: a 4-image chain of a water dimer (HF/6-31G*, two
server slots) gives each image's energy and gradients of a lone engine's cold SCF to 1e-6 kJ/mol and
1e-5 kJ/mol/A, and the next call (moved images) starts every image from its own last density."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

OPTS = dict(orbital_basis="6-31g_st_cart", functional="hf", density_tolerance=1e-10, energy_tolerance=1e-10)


def test_chain_of_images_matches_lone_engines_and_warm_starts(cuda_device):
    from pdynamo3_b200.pool import ArrayObjective, SGOFProcessPoolGPU
    from pdynamo3_b200.qcmodel import GPUQCEngine
    g0 = load_golden("b3lyp_water2_cart_medium")
    xyz = np.asarray(g0["xyz"], dtype=np.float64)
    obj = ArrayObjective(g0["Z"], xyz, **OPTS)
    rng = np.random.default_rng(2)
    images = [(xyz + rng.normal(scale=0.03, size=xyz.shape)).reshape(-1) for _ in range(4)]
    pool = SGOFProcessPoolGPU.FromObjectiveFunction(obj, maximumProcesses=2)
    try:
        g = [np.zeros(obj.numberOfVariables) for _ in images]
        f = pool.FunctionGradients(images, g)
        for x, fi, gi in zip(images, f, g):
            e = GPUQCEngine(g0["Z"], warm_start=False, **OPTS)
            try:
                r = e.energy(obj.coordinates_bohr(x))
            finally:
                e.close()
            assert abs(fi - r.energy_kjmol) < 1e-6
            assert np.abs(gi.reshape(-1, 3) - r.gradients_kjmol_per_angstrom()).max() < 1e-5
        cold = [r.result.iterations for r in pool.last_requests]
        moved = [x + rng.normal(scale=0.005, size=x.shape) for x in images]
        pool.FunctionGradients(moved, [np.zeros(obj.numberOfVariables) for _ in moved])
        assert all(r.warm for r in pool.last_requests)
        assert sum(r.result.iterations for r in pool.last_requests) < sum(cold)
    finally:
        pool.Finalize()
