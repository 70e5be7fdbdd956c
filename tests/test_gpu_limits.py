"""Boundary behaviour of the C-ABI on the GPU: inputs outside the implemented set are refused with
the documented status before any device work, and the context stays usable.

* a shell above d (f functions): PDG_ERR_UNSUPPORTED from pdg_basis_upload;
* a DFT grid for more than 256 atoms: PDG_ERR_UNSUPPORTED from pdg_grid_build;
* out-of-order calls (a Fock build without a geometry): PDG_ERR_STATE;
* empty point sets for the functional entry points: no work, empty results;
* an unknown functional name: PDG_ERR_UNSUPPORTED.
"""
import numpy as np
import pytest

from conftest import ANGSTROM_TO_BOHR, HARTREE_TO_KJMOL, load_golden
from pdynamo3_b200.basis import ShellTable

pytestmark = pytest.mark.gpu


class RawShells:
    """A hand-made shell table in the upload layout of basis.ShellTable."""

    def __init__(self, z, shells, spherical=False):
        self.atomic_numbers = np.asarray(z, dtype=np.int32)
        atom, lo, hi, npr, ex, co = [], [], [], [], [], []
        for a, l_low, l_high, exps, coefs in shells:
            atom.append(a); lo.append(l_low); hi.append(l_high); npr.append(len(exps))
            ex.extend(exps)
            for _ in range(l_low, l_high + 1):
                co.extend(coefs)
        self.args = (len(z), np.asarray(z, dtype=np.float64), len(atom), np.asarray(atom, dtype=np.int32),
                     np.asarray(lo, dtype=np.int32), np.asarray(hi, dtype=np.int32), np.asarray(npr, dtype=np.int32),
                     np.asarray(ex), np.asarray(co), 1)
        self.spherical = spherical

    def upload_args(self):
        return self.args


def test_f_shells_are_refused_and_the_context_stays_usable(cuda_device):
    from pdynamo3_b200.lib import PDG_ERR_UNSUPPORTED, Context, PDGError
    ctx = Context(0)
    with pytest.raises(PDGError) as err:
        ctx.set_basis(RawShells([8], [(0, 0, 0, [1.0], [1.0]), (0, 3, 3, [0.8], [1.0])]))
    assert err.value.status == PDG_ERR_UNSUPPORTED
    g = load_golden("hf_water1_cart")
    ctx.set_basis(ShellTable("6-31g_st_cart", g["Z"]))
    ctx.set_geometry(g["xyz"] * ANGSTROM_TO_BOHR)
    P, res = ctx.scf(density_tolerance=1e-10, energy_tolerance=1e-9)
    assert res.converged and abs(res.energy_total - float(g["energy_kjmol"]) / HARTREE_TO_KJMOL) < 1e-8
    ctx.close()


def test_grid_for_more_than_256_atoms_is_refused(cuda_device):
    from pdynamo3_b200.lib import PDG_ERR_UNSUPPORTED, Context, PDGError
    n = 258
    z = np.ones(n, dtype=np.int32)
    rng = np.random.default_rng(2)
    xyz = rng.uniform(0.0, 40.0, size=(n, 3))
    ctx = Context(0)
    ctx.set_basis(RawShells(z, [(a, 0, 0, [1.0], [1.0]) for a in range(n)]))
    ctx.set_geometry(xyz)
    ctx.set_functional("pbe")
    with pytest.raises(PDGError) as err:
        ctx.grid_build(3)
    assert err.value.status == PDG_ERR_UNSUPPORTED
    ctx.close()


def test_out_of_order_calls_and_unknown_names_are_refused(cuda_device):
    from pdynamo3_b200.lib import PDG_ERR_STATE, PDG_ERR_UNSUPPORTED, Context, PDGError, xc_evaluate, xc_evaluate_static
    g = load_golden("hf_water1_cart")
    ctx = Context(0)
    ctx.set_basis(ShellTable("6-31g_st_cart", g["Z"]))
    with pytest.raises(PDGError) as err:
        ctx.fock_two_electron(np.zeros(ctx.npacked()), 1.0, True)
    assert err.value.status == PDG_ERR_STATE
    with pytest.raises(PDGError) as err:
        ctx.set_functional("m06")
    assert err.value.status == PDG_ERR_UNSUPPORTED
    ctx.close()
    for fn in (xc_evaluate, xc_evaluate_static):
        f, vr, vs = fn("pbe", np.zeros(0), np.zeros(0))
        assert f.size == vr.size == vs.size == 0
