"""QCModelDFTGPU inside pDynamo3's own System.Energy (runs where pDynamo3 is importable).

The engine is replaced by a stand-in that returns fixed values, so the test checks the wiring
only: the model is accepted by System.DefineQCModel, System.Energy(doGradients=True) returns the
engine's energy in kJ/mol, QCModel.EnergyFinalize scatters the engine's hartree/bohr gradients
into system.scratch.gradients3 in kJ/mol/A, the qcEnergyReport carries the engine's terms, the
engine sees the coordinates in bohr, and a non-converged SCF raises QCModelError with the
converger's message.  The GPU numbers themselves are covered by test_gpu_qcmodel.py.
"""
import os
import tempfile

import numpy as np
import pytest

pytest.importorskip("pMolecule")

from pdynamo3_b200 import geometry, qcmodel  # noqa: E402
from pdynamo3_b200.basis import ShellTable  # noqa: E402
from pdynamo3_b200.qcmodel import ANGSTROM_TO_BOHR, HARTREE_TO_KJMOL, EnergyResult  # noqa: E402


class FakeEngine:
    instances = []

    def __init__(self, atomic_numbers, converged=True, **options):
        self.atomic_numbers = np.asarray(atomic_numbers, dtype=np.int32)
        self.options = options
        self.converged = converged
        self.seen = []
        FakeEngine.instances.append(self)

    def energy(self, coordinates_bohr, do_gradients=True):
        self.seen.append(np.array(coordinates_bohr))
        n = len(self.atomic_numbers)
        g = np.arange(3 * n, dtype=np.float64).reshape(n, 3) * 1e-3 if do_gradients else None
        report = {"QC Core-Core": 9.0, "One-Electron Energy": -120.0, "Two-Electron Energy": 35.0,
                  "SCF Converged": self.converged, "SCF Iterations": 7}
        nb = ShellTable(self.options.get("orbital_basis", "6-31g_st"), self.atomic_numbers).n_functions()
        return EnergyResult(-76.0, report, g, np.zeros(nb * (nb + 1) // 2), self.converged, 7)

    def close(self):
        pass


def _system(model):
    from pBabel import ImportSystem
    z, xyz = geometry.water_cluster(1, 3.0, 11)
    with tempfile.NamedTemporaryFile("w", suffix=".xyz", delete=False) as f:
        path = f.name
    geometry.write_xyz(path, z, xyz, "water")
    system = ImportSystem(path)
    os.unlink(path)
    system.DefineQCModel(model)
    return system, xyz


def test_system_energy_through_the_gpu_model(monkeypatch):
    monkeypatch.setattr(qcmodel, "GPUQCEngine", FakeEngine)
    cls = qcmodel.qcmodel_class()
    system, xyz = _system(cls.WithOptions(functional="hf", orbitalBasis="6-31g_st"))
    e = system.Energy(doGradients=True, log=None)
    assert abs(e - (-76.0 * HARTREE_TO_KJMOL)) < 1e-9
    eng = FakeEngine.instances[-1]
    assert list(eng.atomic_numbers) == [8, 1, 1]
    assert np.abs(eng.seen[-1] - xyz * ANGSTROM_TO_BOHR).max() < 1e-9
    g3 = system.scratch.gradients3
    ref = np.arange(9, dtype=np.float64).reshape(3, 3) * 1e-3 * HARTREE_TO_KJMOL * ANGSTROM_TO_BOHR
    got = np.array([[g3[i, j] for j in range(3)] for i in range(3)])
    assert np.abs(got - ref).max() < 1e-9
    rep = system.scratch.qcEnergyReport
    assert rep["QC Core-Core"] == 9.0 and rep["Two-Electron Energy"] == 35.0 and rep["SCF Iterations"] == 7
    # a second energy reuses the engine (resident basis and warm-start density)
    system.Energy(doGradients=False, log=None)
    assert FakeEngine.instances[-1] is eng and len(eng.seen) == 2


def test_non_converged_scf_raises_the_converger_error(monkeypatch):
    from pMolecule.QCModel import QCModelError
    monkeypatch.setattr(qcmodel, "GPUQCEngine", lambda z, **kw: FakeEngine(z, converged=False, **kw))
    cls = qcmodel.qcmodel_class()
    system, _ = _system(cls.WithOptions(functional="hf", orbitalBasis="6-31g_st"))
    with pytest.raises(QCModelError) as err:
        system.Energy(doGradients=True, log=None)
    assert "Too many iterations" in str(err.value)


def test_bulk_copy_into_reference_arrays():
    """Densities and gradients reach pDynamo3's own arrays by one bulk copy through their storage
    block, in the reference's orders (packed lower triangle, row-major N x 3)."""
    from pScientific.Arrays import Array, StorageType
    from pScientific.Geometry3 import Coordinates3
    n = 7
    d = Array.WithExtent(n, storageType=StorageType.Symmetric)
    vals = np.linspace(-1.0, 2.0, n * (n + 1) // 2)
    assert qcmodel.copy_into_array(d, vals)
    k = 0
    for i in range(n):
        for j in range(i + 1):
            assert d[i, j] == vals[k] and d[j, i] == vals[k]
            k += 1
    g3 = Coordinates3.WithExtent(5)
    g = np.arange(15.0).reshape(5, 3) * 0.5
    assert qcmodel.copy_into_array(g3, g)
    assert all(g3[i, j] == g[i, j] for i in range(5) for j in range(3))
