"""Mixed precision: shell quartets whose Schwarz x density bound is below mixed_cut (1e-6) are
evaluated in FP32, the rest in FP64.  Against the FP64 path on the same inputs the mixed form must
stay within 1e-5 hartree in energy and 1e-4 hartree/angstrom in gradient, and the FP32 kernels must
really have run (the library's count of FP32 quartets is positive in mixed mode, zero in FP64).
The two-electron Fock matrix of a fixed density is held to 1e-6.
"""
import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR, load_golden
from pdynamo3_b200.basis import ShellTable

pytestmark = pytest.mark.gpu

E_TOL = 1e-5                       # hartree
G_TOL = 1e-4 / ANGSTROM_TO_BOHR    # 1e-4 hartree/angstrom in hartree/bohr


def _ctx(g, functional=None, accuracy=3, mode=0):
    from pdynamo3_b200.lib import Context
    ctx = Context(0)
    ctx.set_basis(ShellTable("6-31g_st_cart", g["Z"]))
    ctx.set_geometry(g["xyz"] * ANGSTROM_TO_BOHR)
    ctx.set_eri_options(precision_mode=mode, mixed_cut=1e-6)
    if functional:
        ctx.set_functional(functional)
        ctx.grid_build(accuracy)
    return ctx


def test_mixed_fock_build_close_to_fp64(cuda_device):
    g = load_golden("hf_water4_s0_cart")
    out, n32 = [], []
    for mode in (0, 1):
        ctx = _ctx(g, mode=mode)
        out.append(ctx.fock_two_electron(g["P"], 1.0))
        n32.append(ctx.fp32_quartets())
        ctx.close()
    (F64, E64), (F32, E32) = out
    assert n32[0] == 0 and n32[1] > 0
    assert np.abs(F32 - F64).max() < 1e-6
    assert abs(E32 - E64) < 1e-6


@pytest.mark.parametrize("name,functional", [("hf_water4_s0_cart", None), ("b3lyp_water2_cart_medium", "b3lyp")])
def test_mixed_scf_energy_and_gradient_within_tolerance(cuda_device, name, functional):
    g = load_golden(name)
    res, n32 = [], []
    for mode in (0, 1):
        ctx = _ctx(g, functional, mode=mode)
        P, r = ctx.scf(density_tolerance=1e-8, energy_tolerance=1e-8, maximum_iterations=100)
        assert r.converged
        res.append((r.energy_total, ctx.scf_gradients()))
        n32.append(ctx.fp32_quartets())
        ctx.close()
    (e64, g64), (e32, g32) = res
    assert n32[0] == 0 and n32[1] > 0
    assert abs(e32 - e64) < E_TOL
    assert np.abs(g32 - g64).max() < G_TOL
