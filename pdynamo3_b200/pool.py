"""GPU backend for the reference's process pool of objective-function evaluations.

pSimulation/SGOFProcessPool.py:20-230 defines the pool pDynamo3's chain-of-states optimiser
(ChainOfStatesOptimizer.py:40,202) and other multi-geometry drivers use: ``FromObjectiveFunction``
(objective function, maximumProcesses), ``FunctionGradients(x, g)`` returning the function values of
all tasks and filling their gradients in place, ``Initialize`` and ``Finalize``; a factory picks the
pool class by name.  ``SGOFProcessPoolGPU`` keeps that interface and evaluates the tasks on one GPU
through the continuous-batching server (``serving.GPUServer``): ``maximumProcesses`` is the number of
server slots (concurrent SCFs on their own streams), and task i of every call is the same system
key, so chain-of-states image i stays resident on one slot and its SCF starts from its previous
density.  Results do not depend on the slot count (each SCF's arithmetic is the same alone and in
the mix).

Objective functions: a pDynamo3 ``SystemGeometryObjectiveFunction`` whose system carries a
closed-shell DFT/HF QC model (``SystemObjective`` reads its atoms, QC options, ``VariablesPut`` and
``GradientsGet``), or any object with the small ``objective`` protocol below (used by the tests and
the benchmark, which cannot import pDynamo3 on the GPU host).
"""
import numpy as np

from .qcmodel import ANGSTROM_TO_BOHR, HARTREE_TO_KJMOL, copy_into_array
from .serving import GPUServer, Request


class ArrayObjective:
    """The objective protocol on plain arrays: variables are the Cartesian coordinates (angstrom)
    of the free atoms, the function is the energy in kJ/mol, the gradients are in kJ/mol/angstrom
    (pDynamo3's units).

    atomic_numbers   all atoms
    reference_xyz    coordinates (angstrom) of all atoms; fixed atoms keep theirs
    free             indices of the atoms the variables move (default all)
    engine_options   GPUQCEngine options (orbital_basis, functional, grid_accuracy, tolerances)
    """

    def __init__(self, atomic_numbers, reference_xyz, free=None, **engine_options):
        self.atomic_numbers = np.asarray(atomic_numbers, dtype=np.int32)
        self.reference_xyz = np.array(reference_xyz, dtype=np.float64).reshape(-1, 3)
        self.free = np.arange(len(self.atomic_numbers)) if free is None else np.asarray(free, dtype=np.int64)
        self.engine_options = engine_options

    @property
    def numberOfVariables(self):
        return 3 * len(self.free)

    def coordinates_bohr(self, x):
        xyz = self.reference_xyz.copy()
        xyz[self.free] = np.asarray(x, dtype=np.float64).reshape(-1, 3)
        return xyz * ANGSTROM_TO_BOHR

    def function_gradients(self, result, g):
        """kJ/mol and, into g, kJ/mol/angstrom of the free atoms."""
        if g is not None:
            grad = result.gradients * (HARTREE_TO_KJMOL * ANGSTROM_TO_BOHR)
            np.copyto(np.asarray(g).reshape(-1, 3), grad[self.free])
        return result.energy * HARTREE_TO_KJMOL


class SystemObjective:
    """The protocol over a pDynamo3 SystemGeometryObjectiveFunction (pMolecule/
    SystemGeometryObjectiveFunction.py): VariablesPut(x) places the variables in the system's
    coordinates3 (angstrom), GradientsGet(g) reads scratch.gradients3 back into the variables."""

    def __init__(self, objective_function):
        self.of = objective_function
        system = objective_function.system
        qc = system.qcModel
        self.atomic_numbers = np.asarray(system.atoms.atomicNumbers, dtype=np.int32)
        orbital = getattr(qc, "orbitalBasis", "6-31g_st")
        accuracy = getattr(qc, "gridIntegrator", None)
        accuracy = getattr(accuracy, "accuracy", "medium") if accuracy is not None else "medium"
        self.engine_options = dict(orbital_basis=orbital, functional=getattr(qc, "functional", "hf"),
                                   grid_accuracy=accuracy)

    @property
    def numberOfVariables(self):
        return self.of.numberOfVariables

    def coordinates_bohr(self, x):
        self.of.VariablesPut(x)
        crd = self.of.system.coordinates3
        xyz = np.array(list(crd.iterator), dtype=np.float64).reshape(-1, 3)
        return xyz * ANGSTROM_TO_BOHR

    def function_gradients(self, result, g):
        """Energy in kJ/mol; the gradients go through the system's own gradients3 array (a
        Coordinates3, kJ/mol/A) and the objective's GradientsGet, which selects the free atoms and
        applies variable weights and linear constraints (SystemGeometryObjectiveFunction.py:181-197)."""
        if g is not None:
            scratch = self.of.system.scratch
            grad = result.gradients * (HARTREE_TO_KJMOL * ANGSTROM_TO_BOHR)
            g3 = scratch.Get("gradients3", None) if hasattr(scratch, "Get") else getattr(scratch, "gradients3", None)
            if g3 is None or getattr(g3, "rows", None) != grad.shape[0]:
                g3 = self._new_coordinates3(grad.shape[0])
                scratch.gradients3 = g3
            copy_into_array(g3, grad)
            self.of.GradientsGet(g)
        return result.energy * HARTREE_TO_KJMOL

    def _new_coordinates3(self, n):
        factory = getattr(self.of.system.coordinates3, "WithExtent", None)
        if factory is None:
            from pScientific.Geometry3 import Coordinates3
            factory = Coordinates3.WithExtent
        return factory(n)


class SGOFProcessPoolGPU:
    """SGOFProcessPool on one GPU (see the module docstring).  server_options go to GPUServer
    (device, precision_mode, resident_per_slot, memory_reserve)."""

    def __init__(self):
        self.maximumProcesses = 1
        self.objectiveFunction = None
        self.objective = None
        self.server = None
        self.server_options = {}
        self.last_requests = []

    @classmethod
    def FromObjectiveFunction(cls, objectiveFunction, maximumProcesses=1, **server_options):
        self = cls()
        self.maximumProcesses = max(1, int(maximumProcesses))
        self.objectiveFunction = objectiveFunction
        self.server_options = server_options
        self.Initialize()
        return self

    def Initialize(self):
        of = self.objectiveFunction
        self.objective = of if hasattr(of, "function_gradients") else SystemObjective(of)
        opts = dict(self.objective.engine_options)
        opts.update(self.server_options)
        self.server = GPUServer(n_slots=self.maximumProcesses, **opts)

    def FunctionGradients(self, x, g):
        """Function values of the tasks x[i]; their gradients into g[i] (g may be None)."""
        obj = self.objective
        reqs = [self.server.submit(Request(i, "task-%d" % i, obj.atomic_numbers, obj.coordinates_bohr(xi),
                                           do_gradients=g is not None)) for i, xi in enumerate(x)]
        for r in reqs:
            r.done.wait()
        self.last_requests = reqs
        f = []
        for i, r in enumerate(reqs):
            if r.error is not None:
                raise ValueError("GPU pool task %d failed: %s" % (i, r.error))
            if not r.result.converged:
                raise ValueError("GPU pool task %d: SCF not converged" % i)
            f.append(obj.function_gradients(r.result, None if g is None else g[i]))
        return f

    def Finalize(self):
        if self.server is not None:
            self.server.close()
            self.server = None


def register(pool_types):
    """Add the GPU pool to a pool-type table (the reference's SGOFProcessPool._PoolTypes) under
    "GPU", so SGOFProcessPoolFactory(poolType="GPU", maximumProcesses=n) creates it."""
    pool_types["GPU"] = SGOFProcessPoolGPU
    return pool_types
