"""GPU parity for the DFT path through the C-ABI against fixtures made by the reference.

Functionals: relative 1e-11 against the reference's own libxc build (oracle/_ref).  Grid: the
same number of points.  Quadrature Fock and energy of the reference's converged density: 1e-9.
SCF energies: 1e-8 hartree; gradients: 1e-6 hartree/bohr.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR, HARTREE_TO_KJMOL, ROOT, load_golden
from pdynamo3_b200.basis import ShellTable

pytestmark = pytest.mark.gpu

CASES = [("pbe_water1_cart_low", "pbe", 2), ("blyp_water1_cart_medium", "blyp", 3), ("b3lyp_water2_cart_medium", "b3lyp", 3)]
LIBXC_REF = os.path.join(ROOT, "oracle", "_ref", "libxc_ref.so")


def make_ctx(g, functional, accuracy):
    from pdynamo3_b200.lib import Context
    ctx = Context(0)
    ctx.set_basis(ShellTable("6-31g_st_cart", g["Z"]))
    ctx.set_geometry(g["xyz"] * ANGSTROM_TO_BOHR)
    cx = ctx.set_functional(functional)
    npts = ctx.grid_build(accuracy)
    return ctx, cx, npts


@pytest.fixture(scope="module", params=CASES, ids=[c[0] for c in CASES])
def case(request, cuda_device):
    name, functional, acc = request.param
    g = load_golden(name)
    ctx, cx, npts = make_ctx(g, functional, acc)
    return g, ctx, cx, npts


def test_grid_point_count(case):
    # Points whose partition weight lands within rounding of the reference's 1e-30 drop threshold
    # (DFTGrid.c:103,194) may be kept on one side and dropped on the other; they carry no weight.
    g, ctx, cx, npts = case
    assert abs(npts - int(g["grid_points"])) <= max(2, int(2e-4 * int(g["grid_points"])))


def test_quadrature_fock(case):
    g, ctx, cx, npts = case
    F, exc, rho = ctx.fock_quadrature(g["P"])
    assert abs(exc - float(g["Exc"])) < 1e-9
    assert abs(rho - float(g["RhoQuad"])) < 1e-9
    assert np.abs(F - g["Vxc"]).max() < 1e-9


def test_scf_energy_and_gradients(case):
    g, ctx, cx, npts = case
    P, res = ctx.scf(density_tolerance=1e-10, energy_tolerance=1e-9, maximum_iterations=100)
    assert res.converged
    assert abs(res.energy_total - float(g["energy_kjmol"]) / HARTREE_TO_KJMOL) < 1e-8
    grad = ctx.scf_gradients()
    ref = g["gradients_kjmol_A"] / (HARTREE_TO_KJMOL * ANGSTROM_TO_BOHR)
    assert np.abs(grad - ref).max() < 1e-6


@pytest.mark.skipif(not os.path.exists(LIBXC_REF), reason="reference libxc build (oracle/_ref) absent")
@pytest.mark.parametrize("name,fid,gga", [("lda_x", 1, False), ("vwn_rpa", 8, False), ("lyp", 131, True),
                                          ("b88", 106, True), ("pbe_x", 101, True), ("pbe_c", 130, True),
                                          ("b3lyp", 402, True), ("pbe", None, True), ("blyp", None, True)])
def test_functionals_against_reference_libxc(cuda_device, name, fid, gga):
    from pdynamo3_b200.lib import xc_evaluate
    ref = ctypes.CDLL(LIBXC_REF)
    dp = ctypes.POINTER(ctypes.c_double)
    rng = np.random.default_rng(11)
    rho = np.exp(rng.uniform(np.log(1e-6), np.log(1e3), 3000))
    sigma = rho ** (8.0 / 3.0) * np.exp(rng.uniform(np.log(1e-6), np.log(1e3), 3000))

    scale = [np.zeros_like(rho), np.zeros_like(rho), np.zeros_like(rho)]  # sum of component magnitudes

    def libxc(fids):
        F = np.zeros_like(rho); VR = np.zeros_like(rho); VS = np.zeros_like(rho)
        for f in fids:
            buf = ctypes.create_string_buffer(16384)
            assert ref.xc_func_init(buf, f, 1) == 0
            zk, vr, vs = np.zeros_like(rho), np.zeros_like(rho), np.zeros_like(rho)
            if gga:
                ref.xc_gga_exc_vxc(buf, len(rho), rho.ctypes.data_as(dp), sigma.ctypes.data_as(dp), zk.ctypes.data_as(dp),
                                   vr.ctypes.data_as(dp), vs.ctypes.data_as(dp))
            else:
                ref.xc_lda_exc_vxc(buf, len(rho), rho.ctypes.data_as(dp), zk.ctypes.data_as(dp), vr.ctypes.data_as(dp))
            ref.xc_func_end(buf)
            F += zk * rho; VR += vr; VS += vs
            scale[0] += np.abs(zk * rho); scale[1] += np.abs(vr); scale[2] += np.abs(vs)
        return F, VR, VS
    fids = {"pbe": [101, 130], "blyp": [106, 131]}.get(name, [fid])
    a = libxc(fids)
    b = xc_evaluate(name, rho, sigma)
    for x, y, s in zip(a, b, scale):
        if np.any(x):
            assert np.max(np.abs(x - y) / np.maximum(s, 1e-300)) < 1e-11
