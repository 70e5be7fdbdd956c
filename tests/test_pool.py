"""Host logic of the GPU process-pool backend (pdynamo3_b200.pool) with stand-in engines: the
SGOFProcessPool interface (FromObjectiveFunction, FunctionGradients filling g in place and returning
the function values in task order, Finalize), units and free-atom mapping of the array objective,
task i staying on one slot across calls (warm), errors and unconverged SCFs raised, and the
factory registration."""
import threading
import time

import numpy as np
import pytest

from pdynamo3_b200.pool import ArrayObjective, SGOFProcessPoolGPU, register
from pdynamo3_b200.qcmodel import ANGSTROM_TO_BOHR, HARTREE_TO_KJMOL


class Result:
    def __init__(self, x, converged=True):
        self.energy = float(np.sum(x ** 2))           # hartree
        self.gradients = 2.0 * x                       # hartree/bohr
        self.converged = converged


class Engine:
    lock = threading.Lock()
    calls = []

    def __init__(self, request, converged=True, fail_on=None):
        self.atomic_numbers = request.atomic_numbers
        self.key = request.system
        self.converged = converged
        self.fail_on = fail_on

    def energy(self, coordinates_bohr, do_gradients=True):
        time.sleep(0.002)
        with Engine.lock:
            Engine.calls.append(self.key)
        if self.fail_on == self.key:
            raise RuntimeError("boom")
        return Result(np.asarray(coordinates_bohr, dtype=np.float64).reshape(-1, 3), self.converged)

    def close(self):
        pass


def _objective(free=None):
    z = [8, 1, 1, 8, 1, 1]
    xyz = np.arange(18, dtype=np.float64).reshape(6, 3) * 0.1
    return ArrayObjective(z, xyz, free=free)


def _pool(objective, n=3, **kw):
    return SGOFProcessPoolGPU.FromObjectiveFunction(objective, maximumProcesses=n,
                                                    engine_factory=lambda r: Engine(r, **kw), free_memory=lambda: None)


def test_function_gradients_order_units_and_free_atoms():
    Engine.calls = []
    obj = _objective(free=[0, 2, 4])
    pool = _pool(obj)
    try:
        rng = np.random.default_rng(0)
        x = [rng.normal(size=obj.numberOfVariables) for _ in range(7)]
        g = [np.zeros(obj.numberOfVariables) for _ in range(7)]
        f = pool.FunctionGradients(x, g)
        for xi, gi, fi in zip(x, g, f):
            full = obj.coordinates_bohr(xi)
            assert np.allclose(full[[1, 3, 5]], obj.reference_xyz[[1, 3, 5]] * ANGSTROM_TO_BOHR)   # fixed atoms
            assert abs(fi - np.sum(full ** 2) * HARTREE_TO_KJMOL) < 1e-9 * abs(fi)
            ref = 2.0 * full[[0, 2, 4]] * HARTREE_TO_KJMOL * ANGSTROM_TO_BOHR
            assert np.allclose(gi.reshape(-1, 3), ref)
        assert pool.FunctionGradients(x[:2], None) == pytest.approx(f[:2])
    finally:
        pool.Finalize()


def test_each_task_stays_resident_on_one_slot():
    obj = _objective()
    pool = _pool(obj, n=3)
    try:
        x = [np.full(18, 0.1 * (i + 1)) for i in range(6)]
        pool.FunctionGradients(x, [np.zeros(18) for _ in x])
        first = {r.id: r.slot for r in pool.last_requests}
        pool.FunctionGradients(x, [np.zeros(18) for _ in x])
        second = pool.last_requests
        assert all(r.warm for r in second)
        assert {r.id: r.slot for r in second} == first
    finally:
        pool.Finalize()


def test_errors_and_unconverged_tasks_raise():
    obj = _objective()
    pool = _pool(obj, n=2, fail_on="task-1")
    try:
        with pytest.raises(ValueError, match="task 1 failed"):
            pool.FunctionGradients([np.zeros(18), np.ones(18)], [np.zeros(18), np.zeros(18)])
    finally:
        pool.Finalize()
    pool = _pool(obj, n=2, converged=False)
    try:
        with pytest.raises(ValueError, match="not converged"):
            pool.FunctionGradients([np.zeros(18)], [np.zeros(18)])
    finally:
        pool.Finalize()


def test_registration_in_a_pool_type_table():
    table = {"Serial": object}
    register(table)
    assert table["GPU"] is SGOFProcessPoolGPU


class StubCoordinates3:
    """The parts of pScientific's Coordinates3 the pool touches: rows, (i, j) item access, the
    flat iterator, RowIterator(selection) and the WithExtent constructor."""

    def __init__(self, n):
        self.rows = n
        self.a = np.zeros((n, 3))

    @classmethod
    def WithExtent(cls, n):
        return cls(n)

    def __getitem__(self, ij):
        return float(self.a[ij])

    def __setitem__(self, ij, value):
        self.a[ij] = float(value)

    @property
    def iterator(self):
        return _StubIterator(self.a.reshape(-1))

    def RowIterator(self, selection=None):
        return _StubIterator(self.a[np.asarray(selection)].reshape(-1))


class _StubIterator:
    def __init__(self, values):
        self.values = values

    def __iter__(self):
        return iter(float(v) for v in self.values)

    def CopyTo(self, other):
        other.values[:] = self.values


class _StubVector:
    def __init__(self, g):
        self.g = g

    @property
    def iterator(self):
        return _StubIterator(self.g)


class StubScratch:
    def __init__(self):
        self._d = {}

    def Get(self, key, default=None):
        return self._d.get(key, default)

    def __getattr__(self, key):
        try:
            return self.__dict__["_d"][key]
        except KeyError:
            raise AttributeError(key)

    def __setattr__(self, key, value):
        if key == "_d":
            object.__setattr__(self, key, value)
        else:
            self._d[key] = value


class StubSystem:
    def __init__(self, z, xyz, qc):
        self.atoms = type("Atoms", (), {"atomicNumbers": list(z)})()
        self.qcModel = qc
        self.coordinates3 = StubCoordinates3(len(z))
        self.coordinates3.a[:] = xyz
        self.scratch = StubScratch()


class StubObjectiveFunction:
    """SystemGeometryObjectiveFunction's variable and gradient plumbing
    (pMolecule/SystemGeometryObjectiveFunction.py:181-197): free atoms selected by RowIterator,
    gradients divided by the variable weights."""

    def __init__(self, system, free, weights):
        self.system = system
        self.freeAtoms = free
        self.variableWeights = weights
        self.numberOfVariables = 3 * len(free)

    def VariablesPut(self, x):
        x = np.asarray(x, dtype=np.float64) * self.variableWeights
        self.system.coordinates3.a[self.freeAtoms] = x.reshape(-1, 3)

    def GradientsGet(self, g):
        self.system.scratch.gradients3.RowIterator(selection=self.freeAtoms).CopyTo(_StubVector(g).iterator)
        g /= self.variableWeights


def test_system_objective_goes_through_coordinates3_and_gradients_get():
    """A pDynamo3-style objective: the gradients reach the caller through the system's own
    gradients3 (a Coordinates3, created on first use) and the objective's GradientsGet, so free-atom
    selection and variable weights apply as in the reference."""
    from pdynamo3_b200.pool import SystemObjective
    z = [8, 1, 1, 8, 1, 1]
    xyz = np.arange(18, dtype=np.float64).reshape(6, 3) * 0.1
    qc = type("QC", (), {"orbitalBasis": "6-31g_st", "functional": "hf", "gridIntegrator": None})()
    free = np.array([0, 2, 4])
    weights = np.linspace(1.0, 2.0, 9)
    of = StubObjectiveFunction(StubSystem(z, xyz, qc), free, weights)
    so = SystemObjective(of)
    assert so.engine_options["functional"] == "hf" and list(so.atomic_numbers) == z
    pool = SGOFProcessPoolGPU.FromObjectiveFunction(of, maximumProcesses=2, engine_factory=lambda r: Engine(r),
                                                    free_memory=lambda: None)
    try:
        assert isinstance(pool.objective, SystemObjective)
        rng = np.random.default_rng(1)
        x = [rng.normal(size=9) for _ in range(3)]
        g = [np.zeros(9) for _ in range(3)]
        f = pool.FunctionGradients(x, g)
        for xi, gi, fi in zip(x, g, f):
            full = xyz.copy()
            full[free] = (xi * weights).reshape(-1, 3)
            full *= ANGSTROM_TO_BOHR
            assert abs(fi - np.sum(full ** 2) * HARTREE_TO_KJMOL) < 1e-9 * abs(fi)
            ref = (2.0 * full[free] * HARTREE_TO_KJMOL * ANGSTROM_TO_BOHR).reshape(-1) / weights
            assert np.allclose(gi, ref)
        assert isinstance(of.system.scratch.gradients3, StubCoordinates3)
    finally:
        pool.Finalize()
