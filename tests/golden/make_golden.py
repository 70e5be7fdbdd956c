"""Generate the golden fixtures in this directory by running the pDynamo3 reference.

This script needs a built pDynamo3 (the reference) importable from Python, with the usual
environment (PDYNAMO3_HOME, PDYNAMO3_PARAMETERS, PDYNAMO3_SCRATCH, PYTHONPATH).  The
Cartesian 6-31G* basis is a copy of ``parameters/gaussianBasisSets/6-31g_st`` named
``6-31g_st_cart`` with ``Is Spherical: false`` in every element file; PDYNAMO3_PARAMETERS must
point at a parameter directory that contains it.

For every case it records, through the reference's own public API (System.Energy and the
Fock-construction and integral functions it calls):
  Z, coordinates (A), overlap S and core Hamiltonian H (packed), converged density P and
  weighted density W (packed), the two-electron Fock matrix F2 = J - (c/2) K of P for
  c = 1, 0.2 and 0 with E2 = 1/2 tr(P F2), the same for a seeded random density, the energy
  terms (hartree), the total energy (kJ/mol) and the gradients (kJ/mol/A).

Usage:  python make_golden.py [case ...]
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from pdynamo3_b200 import geometry  # noqa: E402

HARTREE_TO_KJMOL = 2625.5


def packed(m):
    return np.array(list(m.iterator), dtype=np.float64)


def run_case(name, z, xyz, functional="hf", basis="6-31g_st_cart", grid=None, density_tol=1e-10, light=False,
             grid_override=None):
    """light: record only the energies, gradients, report terms and grid size (large systems).
    grid_override: (n_radial, l) for the patched reference (PDYNAMO3_GRID_OVERRIDE, see
    build_reference.sh); the library's pdg_grid_build(accuracy, n_radial, l) makes the same grid."""
    if grid_override is not None:
        os.environ["PDYNAMO3_GRID_OVERRIDE"] = "%d,%d" % tuple(grid_override)
    else:
        os.environ.pop("PDYNAMO3_GRID_OVERRIDE", None)
    from pBabel import ImportSystem
    from pMolecule.QCModel import DFTGridAccuracy, DFTGridIntegrator, DIISSCFConverger, QCModelDFT
    from pMolecule.QCModel.FockConstruction import (FockConstruction_MakeFromTEIs,
                                                     FockConstruction_MakeFromTEIsCoulomb)
    from pScientific.Arrays import Array, StorageType

    with tempfile.NamedTemporaryFile("w", suffix=".xyz", delete=False) as f:
        path = f.name
    geometry.write_xyz(path, z, xyz, name)
    system = ImportSystem(path)
    os.unlink(path)
    conv = DIISSCFConverger.WithOptions(densityTolerance=density_tol, maximumIterations=250)
    opts = dict(converger=conv, functional=functional, orbitalBasis=basis, maximumMemory=48.0)
    if grid is not None:
        opts["gridIntegrator"] = DFTGridIntegrator.WithOptions(accuracy=DFTGridAccuracy[grid], inCore=False)
    system.DefineQCModel(QCModelDFT.WithOptions(**opts))
    energy = system.Energy(doGradients=True, log=None)
    sc = system.scratch
    xyz_used = np.array(list(system.coordinates3.iterator), dtype=np.float64).reshape(-1, 3)
    out = {"Z": np.asarray(z, dtype=np.int32), "xyz": xyz_used,
           "energy_kjmol": np.float64(energy),
           "gradients_kjmol_A": np.array(list(sc.gradients3.iterator), dtype=np.float64).reshape(-1, 3)}
    if grid_override is not None:
        out["grid_override"] = np.asarray(grid_override, dtype=np.int32)
    if not light:
        out.update({"S": packed(sc.overlapMatrix), "H": packed(sc.oneElectronMatrix),
                    "P": packed(sc.onePDMP.density), "W": packed(sc.weightedDensity)})
    rep = sc.qcEnergyReport
    for key in ("QC Core-Core", "One-Electron Energy", "Two-Electron Energy", "Two-Electron Coulomb Energy",
                "Quadrature Energy", "SCF Iterations", "TEI Number", "Quadrature Points", "Quadrature Electron Count"):
        if key in rep:
            v = rep[key]
            out["report_" + key.replace(" ", "_").replace("-", "_")] = np.float64(v[0] if isinstance(v, tuple) else v)
    n = sc.overlapMatrix.rows
    out["n_functions"] = np.int64(n)
    tei = None if light else sc.twoElectronIntegrals
    if tei is not None:
        def fock(p_packed, cx):
            d = Array.WithExtent(n, storageType=StorageType.Symmetric)
            vals = iter(p_packed)
            for i in range(n):
                for j in range(i + 1):
                    d[i, j] = float(next(vals))
            fm = Array.WithExtent(n, storageType=StorageType.Symmetric)
            if cx == 0.0:
                e2 = FockConstruction_MakeFromTEIsCoulomb(d, tei, fm)
            else:
                e2 = FockConstruction_MakeFromTEIs(d, None, tei, cx, fm, None)
            return packed(fm), np.float64(e2)

        rng = np.random.default_rng(7)
        a = rng.normal(size=(n, n)) * 0.1
        prand = (a + a.T)[np.tril_indices(n)]
        # packed order i(i+1)/2 + j equals numpy tril_indices row-major order
        out["Prand"] = prand
        for tag, pk in (("", out["P"]), ("rand_", prand)):
            for cx in (1.0, 0.2, 0.0):
                f2, e2 = fock(pk, cx)
                key = "%scx%g" % (tag, cx)
                out["F2_" + key] = f2
                out["E2_" + key] = e2
    if grid is not None and light:
        out["grid_points"] = np.int64(sc.dftGrid.numberOfPoints)
    elif grid is not None:
        # Quadrature Fock contribution V_xc of the converged density (DFTGridIntegrator.Fock).
        from pMolecule.QCModel.DFTIntegrator import DFTIntegrator_Integrate
        fm = Array.WithExtent(n, storageType=StorageType.Symmetric)
        fm.Set(0.0)
        eq, rq = DFTIntegrator_Integrate(system.qcModel.functionalModel, sc.dftGrid, system.qcState.orbitalBases,
                                         sc.qcCoordinates3AU, sc.onePDMP.density, None, False, False, fm, None, None)
        out["Vxc"] = packed(fm)
        out["Exc"] = np.float64(eq)
        out["RhoQuad"] = np.float64(rq)
        out["grid_points"] = np.int64(sc.dftGrid.numberOfPoints)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name, "E(Eh) = %.10f" % (energy / HARTREE_TO_KJMOL), "n =", n, "iterations", rep.get("SCF Iterations"))


CASES = {
    "hf_water1_cart": lambda: run_case("hf_water1_cart", *geometry.water_cluster(1, 3.0, 11)),
    "hf_water4_s0_cart": lambda: run_case("hf_water4_s0_cart", *geometry.water_cluster(4, 5.0, 0)),
    "pbe_water1_cart_low": lambda: run_case("pbe_water1_cart_low", *geometry.water_cluster(1, 3.0, 11), functional="pbe",
                                            grid="Low"),
    "b3lyp_water2_cart_medium": lambda: run_case("b3lyp_water2_cart_medium", *geometry.water_cluster(2, 4.0, 5),
                                                 functional="b3lyp", grid="Medium"),
    "blyp_water1_cart_medium": lambda: run_case("blyp_water1_cart_medium", *geometry.water_cluster(1, 3.0, 3),
                                                functional="blyp", grid="Medium"),
}



def _batch_molecule(index):
    """Molecule `index` of the 256-molecule organic batch (seed 1), coordinates in angstrom."""
    from pdynamo3_b200 import workloads
    from pdynamo3_b200.qcmodel import ANGSTROM_TO_BOHR
    name, z, x = workloads.batch_molecules(index + 1, seed=1)[index]
    return z, x / ANGSTROM_TO_BOHR


CASES.update({
    # the reference's shipped (spherical, 5d) 6-31G*
    "hf_water4_s0_sph": lambda: run_case("hf_water4_s0_sph", *geometry.water_cluster(4, 5.0, 0), basis="6-31g_st"),
    "b3lyp_water2_sph_medium": lambda: run_case("b3lyp_water2_sph_medium", *geometry.water_cluster(2, 4.0, 5),
                                                functional="b3lyp", grid="Medium", basis="6-31g_st"),
    # the default benchmark's first timed geometry (16 waters, seed 1000), on the reference's Medium
    # grid and on the 75 radial x 302 Lebedev override
    "pbe_water16_s1000_cart_medium": lambda: run_case("pbe_water16_s1000_cart_medium",
                                                      *geometry.water_cluster(16, 8.0, 1000), functional="pbe",
                                                      grid="Medium", light=True),
    "pbe_water16_s1000_cart_75x302": lambda: run_case("pbe_water16_s1000_cart_75x302",
                                                      *geometry.water_cluster(16, 8.0, 1000), functional="pbe",
                                                      grid="Medium", light=True, grid_override=(75, 29)),
    # two molecules of the organic batch (B3LYP/6-31G*, Medium grid)
    "b3lyp_batch4_cart_medium": lambda: run_case("b3lyp_batch4_cart_medium", *_batch_molecule(4),
                                                 functional="b3lyp", grid="Medium", light=True),
    "b3lyp_batch19_cart_medium": lambda: run_case("b3lyp_batch19_cart_medium", *_batch_molecule(19),
                                                  functional="b3lyp", grid="Medium", light=True),
})

if __name__ == "__main__":
    for c in (sys.argv[1:] or list(CASES)):
        CASES[c]()
