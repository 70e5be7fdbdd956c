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
