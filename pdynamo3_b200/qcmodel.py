"""Drop-in B200 QC model for pDynamo3's Gaussian-basis HF/DFT path.

Two layers:

* ``GPUQCEngine`` needs nothing from pDynamo3: atomic numbers, a basis name and a functional in,
  energy terms (hartree), gradients (hartree/bohr) and the converged density out, with the SCF,
  integrals, grid and gradients all in libpdgpu on one GPU.  It keeps the basis, the grid buffers
  and the last converged density resident, so consecutive geometries of one molecule (MD steps,
  optimisation steps, chain-of-states images) start from the previous density.
* ``QCModelDFTGPU`` (built by ``qcmodel_class()`` when pDynamo3 is importable) subclasses the
  reference's ``QCModelDFT`` (pMolecule/QCModel/QCModelDFT.py:36) with the same ``WithOptions``
  keys.  Like the reference's own external-program models (addOns/pySCF/QCModelPySCF.py:109-138)
  it replaces the whole energy closure: ``Energy(target)`` runs the engine, writes
  ``scratch.energyTerms`` ("QC Core-Core", "QC Electronic", kJ/mol), ``scratch.qcEnergyReport``
  (the keys of QCModelBase.py:175-271 and GaussianBasisIntegralEvaluator.pyx:589, hartree), the
  density into ``scratch.onePDMP`` when it exists, and ``scratch.qcGradients3AU`` (hartree/bohr);
  ``QCModel.EnergyFinalize`` (QCModel.py:152-159) converts and scatters the gradients as usual.
  Users keep calling ``system.Energy(doGradients=True)``.

Errors follow the reference: an SCF that does not converge raises ``QCModelError`` with the
converger's message ("SCF Converger error: Too many iterations.", QCModelBase.py:184 and
DIISSCFConverger.py:214); library failures raise ``PDGError`` with the library's message.
"""
import numpy as np

from .basis import ShellTable
from .lib import Context

HARTREE_TO_KJMOL = 2625.5                     # pScientific Units.Energy_Hartrees_To_Kilojoules_Per_Mole
ANGSTROM_TO_BOHR = 1.0e-10 / 5.291772083e-11  # pScientific Units.Length_Angstroms_To_Bohrs

# DFTGridAccuracy (pMolecule/QCModel/DFTGridIntegrator.py) -> pdg_grid_build accuracy code
GRID_ACCURACY = {"verylow": 1, "low": 2, "medium": 3, "high": 4, "veryhigh": 5}


def grid_accuracy_code(accuracy):
    """1..5 from an int, a DFTGridAccuracy member or its name."""
    if isinstance(accuracy, (int, np.integer)):
        return int(accuracy)
    name = getattr(accuracy, "name", accuracy)
    return GRID_ACCURACY[str(name).replace(" ", "").replace("_", "").lower()]


class EnergyResult:
    """One energy (and gradient) evaluation.

    energy          total energy (hartree)
    report          the reference's qcEnergyReport entries for this model (hartree, counts)
    gradients       (n_atoms, 3) hartree/bohr, or None
    density         converged density, packed lower triangle (output basis)
    converged, iterations
    """

    def __init__(self, energy, report, gradients, density, converged, iterations):
        self.energy = energy
        self.report = report
        self.gradients = gradients
        self.density = density
        self.converged = converged
        self.iterations = iterations

    @property
    def energy_kjmol(self):
        return self.energy * HARTREE_TO_KJMOL

    def gradients_kjmol_per_angstrom(self):
        return None if self.gradients is None else self.gradients * (HARTREE_TO_KJMOL * ANGSTROM_TO_BOHR)


class GPUQCEngine:
    """Closed-shell HF/DFT energies and gradients of one molecule through libpdgpu.

    atomic_numbers     per atom
    orbital_basis      basis name (the reference's parameter names: "6-31g_st", "sto-3g"; a
                       "_cart" suffix selects Cartesian d functions)
    functional         "hf", "pbe", "blyp", "b3lyp", "lda" ... (DFTFunctionalModel names)
    grid_accuracy      DFTGridAccuracy member, name or 1..5 (VeryLow..VeryHigh)
    grid               optional (n_radial, angular_l) override of the per-atom grid
    density_tolerance, energy_tolerance, maximum_iterations, maximum_history
                       the DIISSCFConverger options (DIISSCFConverger.py:175-189)
    total_charge       molecular charge
    multiplicity       spin multiplicity 2S+1; above 1 (or unrestricted=True) the SCF is
                       spin-unrestricted (Hartree-Fock only), with S_z = S
    warm_start         start each SCF from the previous converged density of this molecule
    context            an existing lib.Context to work in (its basis, options and buffers are
                       replaced; the caller keeps ownership and close() leaves it open), so a server
                       slot reuses one context, its device buffers and cached atomic guesses, for
                       one molecule after another
    """

    def __init__(self, atomic_numbers, orbital_basis="6-31g_st", functional="hf", grid_accuracy="medium", grid=None,
                 density_tolerance=1.0e-8, energy_tolerance=2.0e-4, maximum_iterations=100, maximum_history=10,
                 total_charge=0.0, warm_start=True, device=0, multiplicity=1, unrestricted=None, context=None):
        self.atomic_numbers = np.asarray(atomic_numbers, dtype=np.int32)
        self.shells = ShellTable(orbital_basis, self.atomic_numbers)
        self.functional = functional
        self.grid_accuracy = grid_accuracy_code(grid_accuracy)
        self.grid = tuple(grid) if grid is not None else (0, 0)
        self.options = dict(density_tolerance=density_tolerance, energy_tolerance=energy_tolerance,
                            maximum_iterations=maximum_iterations, maximum_history=maximum_history)
        self.total_charge = float(total_charge)
        self.warm_start = warm_start
        self._owns_ctx = context is None
        self.ctx = Context(device) if context is None else context
        if context is not None:
            # a reused context starts from the library defaults
            self.ctx.set_eri_options()
            self.ctx.set_incremental()
            if getattr(self.ctx, "nmm", 0):
                self.ctx.set_point_charges(np.zeros(0), np.zeros((0, 3)))
        self.ctx.set_basis(self.shells)
        self.exchange_scaling = self.ctx.set_functional(functional)
        self.is_dft = functional.lower() != "hf"
        self.multiplicity = int(multiplicity)
        self.unrestricted = (self.multiplicity > 1) if unrestricted is None else bool(unrestricted)
        n_el = int(round(float(np.sum(self.shells.nuclear_charges)) - self.total_charge))
        self.n_alpha = (n_el + self.multiplicity - 1) // 2
        self.n_beta = n_el - self.n_alpha
        if self.n_alpha - self.n_beta != self.multiplicity - 1 or self.n_beta < 0:
            self.close()
            raise ValueError("%d electrons cannot have multiplicity %d" % (n_el, self.multiplicity))
        if self.unrestricted and self.is_dft:
            self.close()
            raise NotImplementedError("spin-unrestricted Kohn-Sham is not supported (Hartree-Fock only)")
        self._density = None

    def close(self):
        if self.ctx is not None:
            if self._owns_ctx:
                self.ctx.close()
            self.ctx = None

    def forget_density(self):
        """Start the next SCF from the library's atomic-density guess."""
        self._density = None

    def energy(self, coordinates_bohr, do_gradients=True):
        coordinates_bohr = np.ascontiguousarray(coordinates_bohr, dtype=np.float64).reshape(-1, 3)
        if coordinates_bohr.shape[0] != len(self.atomic_numbers):
            raise ValueError("coordinates for %d atoms, molecule has %d" % (coordinates_bohr.shape[0],
                                                                            len(self.atomic_numbers)))
        ctx = self.ctx
        ctx.set_geometry(coordinates_bohr)
        if self.unrestricted:
            return self._energy_unrestricted(do_gradients)
        npts = ctx.grid_build(self.grid_accuracy, *self.grid) if self.is_dft else None
        guess = self._density if self.warm_start else None
        opts = dict(self.options)
        if guess is not None:
            opts["maximum_iterations"] = min(opts["maximum_iterations"], 40)
        P, res = ctx.scf(guess=guess, total_charge=self.total_charge, raise_on_noconv=False, **opts)
        if guess is not None and not res.converged:
            # a density from a neighbouring geometry can lead DIIS into a stagnating excited
            # solution; start again from the atomic-density guess, as a cold request would
            cycles = int(res.iterations)
            P, res = ctx.scf(guess=None, total_charge=self.total_charge, raise_on_noconv=False, **self.options)
            res.iterations += cycles
        if not res.converged:
            # a cold SCF that reached its limit (DIIS stagnating on a small-gap molecule): once more
            # with every Fock build complete (no difference builds) and the longest DIIS history, and
            # in the mixed mode in FP64, whose Fock builds screen at the FP64 path's tighter bound
            cycles = int(res.iterations)
            retry = dict(self.options, maximum_history=16)
            eri = dict(getattr(ctx, "eri_options", None) or {})
            fp64_retry = eri.get("precision_mode", 0) == 1
            ctx.set_incremental(False)
            if fp64_retry:
                ctx.set_eri_options(**dict(eri, precision_mode=0))
            try:
                P, res = ctx.scf(guess=None, total_charge=self.total_charge, raise_on_noconv=False, **retry)
            finally:
                ctx.set_incremental(True)
                if fp64_retry:
                    ctx.set_eri_options(**eri)
            res.iterations += cycles
        report = {"QC Core-Core": res.energy_nuclear, "One-Electron Energy": res.energy_one}
        if not self.is_dft or self.exchange_scaling != 0.0:
            report["Two-Electron Energy"] = res.energy_two
        else:
            report["Two-Electron Coulomb Energy"] = res.energy_two
        if self.is_dft:
            report["Quadrature Energy"] = res.energy_xc
            report["Quadrature Points"] = int(npts)
            report["Quadrature Electron Count"] = res.rho_integral
        report["SCF Converged"] = bool(res.converged)
        report["SCF Iterations"] = int(res.iterations)
        g = ctx.scf_gradients() if (do_gradients and res.converged) else None
        if res.converged:
            self._density = P
        return EnergyResult(res.energy_total, report, g, P, bool(res.converged), int(res.iterations))

    def _energy_unrestricted(self, do_gradients):
        """Spin-unrestricted HF at the geometry already set; density = P_alpha + P_beta, and the
        spin densities in result.spin_densities."""
        ctx = self.ctx
        guess = self._density if self.warm_start else None
        opts = dict(self.options)
        if guess is not None:
            opts["maximum_iterations"] = min(opts["maximum_iterations"], 40)
        Pa, Pb, res = ctx.uscf(self.n_alpha, self.n_beta, guess=guess, total_charge=self.total_charge,
                               raise_on_noconv=False, **opts)
        if guess is not None and not res.converged:
            cycles = int(res.iterations)
            Pa, Pb, res = ctx.uscf(self.n_alpha, self.n_beta, guess=None, total_charge=self.total_charge,
                                   raise_on_noconv=False, **self.options)
            res.iterations += cycles
        report = {"QC Core-Core": res.energy_nuclear, "One-Electron Energy": res.energy_one,
                  "Two-Electron Energy": res.energy_two, "SCF Converged": bool(res.converged),
                  "SCF Iterations": int(res.iterations), "<S^2>": float(res.s2)}
        g = ctx.scf_gradients() if (do_gradients and res.converged) else None
        if res.converged:
            self._density = (Pa, Pb)
        r = EnergyResult(res.energy_total, report, g, Pa + Pb, bool(res.converged), int(res.iterations))
        r.spin_densities = (Pa, Pb)
        return r


_QCMODEL_CLASS = None


def copy_into_array(array, values):
    """Copy a flat float64 sequence into a pDynamo3 array in its storage order (packed lower
    triangle for a SymmetricMatrix, row-major for a Coordinates3): one bulk copy through the
    array's RealBlock (built from the values in one C loop, then RealBlock.CopyTo), checked on a few
    elements; an element loop where the array exposes no block of matching size.  Returns True for
    the bulk path."""
    values = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
    block = getattr(array, "block", None)
    if block is not None and hasattr(block, "CopyTo") and hasattr(block.__class__, "Raw") and len(block) == values.size:
        src = block.__class__.Raw()
        src.__setstate__({"items": values.tolist()})
        src.CopyTo(block)
        # the array must read back what was written (a view with an offset into a larger block
        # would not): spot checks at both ends
        if _reads_back(array, values):
            return True
    _element_copy(array, values)
    return False


def _is_packed(array, n):
    rows = getattr(array, "rows", 0)
    return rows * (rows + 1) // 2 == n and getattr(array, "columns", rows) == rows


def _reads_back(array, values):
    n = values.size
    for k in (0, n // 2, n - 1):
        i, j = (_index_of_packed(k) if _is_packed(array, n) else divmod(k, 3))
        if array[i, j] != values[k]:
            return False
    return True


def _index_of_packed(k):
    i = int((np.sqrt(8 * k + 1) - 1) // 2)
    while i * (i + 1) // 2 > k:
        i -= 1
    while (i + 1) * (i + 2) // 2 <= k:
        i += 1
    return i, k - i * (i + 1) // 2


def _element_copy(array, values):
    n = values.size
    if _is_packed(array, n):
        k = 0
        for i in range(array.rows):
            for j in range(i + 1):
                array[i, j] = float(values[k])
                k += 1
    else:
        for k in range(n):
            i, j = divmod(k, 3)
            array[i, j] = float(values[k])


def qcmodel_class():
    """The ``QCModelDFTGPU`` class (needs pDynamo3's pMolecule and pScientific importable)."""
    global _QCMODEL_CLASS
    if _QCMODEL_CLASS is not None:
        return _QCMODEL_CLASS
    from pMolecule.QCModel import QCModelDFT, QCModelError
    from pMolecule.QCModel.QCModel import QCModel

    class QCModelDFTGPU(QCModelDFT):
        """QCModelDFT with the Fock build, quadrature, SCF and gradients on one B200."""

        _attributable = dict(QCModelDFT._attributable)
        _classLabel = "DFT QC Model (B200)"
        _summarizable = dict(QCModelDFT._summarizable)
        _attributable.update({"device": 0, "gridOverride": None, "engine": None, "warmStart": True})
        _summarizable.update({"device": "CUDA Device"})

        def EnergyClosures(self, target):
            # initialization, energy, finalization only: integrals, grid, orthogonaliser and
            # gradient closures of the reference all run inside the engine
            return QCModel.EnergyClosures(self, target)

        def _Engine(self, target, state):
            z = np.asarray(list(state.atomicNumbers), dtype=np.int32)
            e = self.engine
            if e is None or not np.array_equal(e.atomic_numbers, z):
                if e is not None:
                    e.close()
                conv = self.converger
                accuracy = getattr(self.gridIntegrator, "accuracy", "medium") if self.gridIntegrator is not None \
                    else "medium"
                charge = float(sum(state.nuclearCharges)) - float(state.alphaCharge + state.betaCharge)
                es = getattr(target, "electronicState", None)
                multiplicity = int(getattr(es, "multiplicity", 1)) if es is not None else 1
                restricted = bool(getattr(es, "isSpinRestricted", True)) if es is not None else True
                e = GPUQCEngine(z, orbital_basis=self.orbitalBasis, functional=self.functional,
                                multiplicity=multiplicity, unrestricted=not restricted,
                                grid_accuracy=accuracy, grid=self.gridOverride,
                                density_tolerance=getattr(conv, "densityTolerance", 1.0e-8),
                                energy_tolerance=getattr(conv, "energyTolerance", 2.0e-4),
                                maximum_iterations=getattr(conv, "maximumIterations", 100),
                                maximum_history=getattr(conv, "maximumHistory", 10),
                                total_charge=charge, warm_start=self.warmStart, device=self.device)
                self.engine = e
            return e

        def Energy(self, target):
            state = getattr(target, self.__class__._stateName)
            scratch = target.scratch
            crd = scratch.qcCoordinates3AU
            xyz = np.array([[crd[i, 0], crd[i, 1], crd[i, 2]] for i in range(crd.rows)], dtype=np.float64)
            result = self._Engine(target, state).energy(xyz, do_gradients=scratch.doGradients)
            report = scratch.qcEnergyReport
            report.update(result.report)
            if not result.converged:
                raise QCModelError("SCF Converger error: Too many iterations.")
            ecc = result.report["QC Core-Core"]
            scratch.energyTerms["QC Core-Core"] = ecc * HARTREE_TO_KJMOL
            scratch.energyTerms["QC Electronic"] = (result.energy - ecc) * HARTREE_TO_KJMOL
            onepdm = scratch.Get("onePDMP", None)
            if onepdm is not None and getattr(onepdm, "density", None) is not None:
                d = onepdm.density
                if len(result.density) != d.rows * (d.rows + 1) // 2:
                    raise QCModelError("GPU density has %d packed elements, the model's basis needs %d."
                                       % (len(result.density), d.rows * (d.rows + 1) // 2))
                copy_into_array(d, result.density)
            if scratch.doGradients:
                copy_into_array(scratch.qcGradients3AU, result.gradients)

    _QCMODEL_CLASS = QCModelDFTGPU
    return QCModelDFTGPU
