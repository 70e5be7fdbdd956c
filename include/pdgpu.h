/*
 * pdgpu: B200 (sm_100a) Fock-build engine for pDynamo3's Gaussian-basis HF/DFT models.
 *
 * C ABI.  Every function returns a status code (PDG_OK = 0); pdg_last_error() gives the
 * message of the last failure on the calling thread.  All host arrays are FP64,
 * C-contiguous, owned by the caller and never freed by the library.  Symmetric matrices
 * use the reference's packed lower-triangle layout, element (i, j), i >= j, at
 * i(i+1)/2 + j (pScientific/Arrays/__extensions__/cinclude/SymmetricMatrix.h:43-46).
 * Lengths are in bohr, energies in hartree, gradients in hartree/bohr.
 *
 * Status codes mirror pCore's Status (pCore/__extensions__/cinclude/Status.h:24-39) plus the
 * GPU-specific ones.
 */
#ifndef PDGPU_H
#define PDGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define PDG_OK 0
#define PDG_ERR_ARG 1          /* invalid argument */
#define PDG_ERR_CUDA 2         /* CUDA runtime / library failure */
#define PDG_ERR_ALLOC 3        /* device memory allocation failed */
#define PDG_ERR_STATE 4        /* call out of order (no basis, no geometry, ...) */
#define PDG_ERR_NOCONV 5       /* SCF did not converge ("Too many iterations.") */
#define PDG_ERR_TIMEOUT 6      /* a bounded device wait ran out */
#define PDG_ERR_NAN 7          /* non-finite value detected */
#define PDG_ERR_UNSUPPORTED 8  /* feature outside the implemented set */

typedef struct pdg_context pdg_context;

/* Library version (major*10000 + minor*100 + patch) and the last error message. */
int pdg_version(void);
const char *pdg_last_error(void);

/* Context on one CUDA device.  Replaces the per-model C state the reference keeps in its
 * GaussianBasisContainer (pMolecule/QCModel/GaussianBases/__extensions__/pyrex/
 * pMolecule.QCModel.GaussianBases.GaussianBasisContainer.pyx:17-232). */
int pdg_context_create(int device, pdg_context **ctx);
int pdg_context_destroy(pdg_context *ctx);

/* Orbital basis, one entry per shell in atom order (the order of
 * GaussianBasisContainer.FromParameterDirectory).  Shell s has angular momenta
 * shell_l_low[s]..shell_l_high[s] (an SP shell is 0..1), shell_nprim[s] primitives whose
 * exponents follow in `exponents`, and for each l of the shell (low to high) shell_nprim[s]
 * contraction coefficients in `coefficients`.  If normalized_primitives is nonzero the
 * coefficients refer to normalised primitives and are unnormalised as in
 * GaussianBasis_UnnormalizePrimitives (GaussianBases/__extensions__/csource/GaussianBasis.c:727-751);
 * Cartesian components are normalised as in GaussianBasis_NormalizePrimitiveCCBF (:460-497).
 * spherical selects real solid harmonics (order m = 0, 1c, 1s, 2c, 2s) for l >= 1. */
int pdg_basis_upload(pdg_context *ctx, int n_atoms, const double *nuclear_charges, int n_shells,
                     const int *shell_atom, const int *shell_l_low, const int *shell_l_high, const int *shell_nprim,
                     const double *exponents, const double *coefficients, int normalized_primitives, int spherical);

/* Number of basis functions of the output basis (spherical or Cartesian) and of the
 * Cartesian work basis. */
int pdg_basis_size(const pdg_context *ctx, int *n_functions, int *n_cartesian);

/* Atom coordinates (n_atoms x 3, bohr).  Invalidates pair lists, grids and Schwarz bounds. */
int pdg_geometry_set(pdg_context *ctx, const double *coordinates3);

/* Two-electron options: quartets with Schwarz bound product below schwarz_cut are skipped;
 * contracted integrals with |value| <= tei_underflow are dropped as the reference's
 * BlockStorage does (GaussianBasisContainerIntegrals_f2Xf2.c:72-73, BlockStorage.c:160-181);
 * precision_mode 0 = FP64 throughout, 1 = mixed (quartets whose Schwarz x density bound is
 * below mixed_cut are evaluated in FP32; the SCF's Fock builds skip quartets whose bound is
 * below 1e-11 instead of the density cut of pdg_set_incremental when that is smaller, and the
 * two-electron gradient those whose Schwarz x |Gamma| bound is below 1e-10). */
int pdg_set_eri_options(pdg_context *ctx, double schwarz_cut, double tei_underflow, int precision_mode,
                        double mixed_cut);

/* SCF difference Fock builds: after a full two-electron build, cycle k builds only
 * G(D_k - D_{k-1}), skipping quartets whose Schwarz bound times the largest contracted density
 * difference is below density_cut, and adds it to the previous Fock matrix; a full build is made
 * again every rebuild_period cycles.  enable = 0 makes every cycle a full build.  Defaults: on,
 * 1e-13, 16.  (The reference stores all integrals and digests the full density every cycle,
 * FockConstruction.c:209-273; this replaces that loop.) */
int pdg_set_incremental(pdg_context *ctx, int enable, double density_cut, int rebuild_period);

/* Overlap S and core Hamiltonian H = T + V_ne (packed), and the nuclear repulsion energy.
 * Replaces f1KOf1i + f2Cm1V + m1Cm1ER1 (GaussianBasisIntegralEvaluator.pyx:97-114,488-509,565-590).
 * Any output pointer may be NULL. */
int pdg_one_electron(pdg_context *ctx, double *overlap, double *core_hamiltonian, double *e_nuclear);

/* Two-electron Fock matrix F2 = J(D) - (exchange_scaling/2) K(D) from the packed total
 * density (F2 zeroed first), and E2 = 1/2 tr(D F2).  do_coulomb = 0 gives the exchange part
 * only.  Replaces Fock_MakeFromTEIs / _Coulomb / _Exchange
 * (pMolecule/QCModel/__extensions__/csource/FockConstruction.c:209-377). */
int pdg_fock_two_electron(pdg_context *ctx, const double *density, double exchange_scaling, int do_coulomb,
                          double *fock, double *e2);

/* Gradient of the SCF energy terms that do not depend on a DFT grid: nuclear repulsion,
 * electron-nuclear, kinetic, overlap (weighted density in the reference's convention,
 * W = sum_i -2 e_i n_i C_i C_i^T, QCOrbitals.py:43-49) and two-electron
 * (GaussianBasisContainerIntegrals_f2Cf2R1, GaussianBasisContainerIntegrals_f2Xf2.c:146-209).
 * The result is ADDED to gradients3 (n_atoms x 3, hartree/bohr). */
int pdg_gradients(pdg_context *ctx, const double *density, const double *weighted_density, double exchange_scaling,
                  int do_coulomb, double *gradients3);

/* DFT functional (case-insensitive names of pMolecule/QCModel/DFTDefinitions.py: "hf",
 * "lda", "pbe", "blyp", "b3lyp").  Sets *exchange_scaling to the exact-exchange fraction. */
int pdg_set_functional(pdg_context *ctx, const char *name, double *exchange_scaling);

/* DFT grid for the current geometry.  accuracy: 1..5 = VeryLow..VeryHigh of the reference's
 * DFTGridAccuracy (pMolecule/QCModel/DFTDefinitions.py:11-17); n_radial > 0 and
 * angular_l > 0 override the per-atom radial count and Lebedev order.  Returns the number of
 * points.  Replaces DFTGrid_Construct (pMolecule/QCModel/__extensions__/csource/DFTGrid.c:105-263). */
int pdg_grid_build(pdg_context *ctx, int accuracy, int n_radial, int angular_l, long long *n_points);

/* Quadrature Fock contribution: adds V_xc to `fock` (packed) and returns E_xc and the
 * integrated density.  Replaces DFTIntegrator_Integrate (DFTIntegrator.c:159-509). */
int pdg_fock_quadrature(pdg_context *ctx, const double *density, double *fock, double *e_xc, double *rho_integral);

/* XC gradient including grid-weight derivatives, ADDED to gradients3.  Replaces the gradient
 * branch of DFTIntegrator_Integrate (DFTIntegrator.c:405-487) and DFTGridWeights_Derivatives
 * (DFTGridWeights.c:98-215). */
int pdg_gradients_quadrature(pdg_context *ctx, const double *density, double *gradients3);

/* Exchange-correlation energy per volume F = rho e(rho, sigma) and its derivatives at n points for a
 * functional combination ("pbe", "blyp", "b3lyp") or a single term ("lda_x", "pw92", "vwn_rpa",
 * "lyp", "b88", "pbe_x", "pbe_c"), spin-unpolarised, evaluated on the device.  Replaces the
 * functional evaluation of DFTFunctionalModel_Evaluate (pMolecule/QCModel/__extensions__/csource/
 * DFTFunctionalModel.c:108-154) over the vendored libxc; its energy density is rho * zk. */
int pdg_xc_evaluate(const char *functional, int n, const double *rho, const double *sigma, double *f, double *vrho,
                    double *vsigma);

/* The same evaluation as pdg_xc_evaluate without any device memory allocation, for callers that
 * must not allocate (a fixed device-memory budget, no cudaMalloc/cudaFree synchronisation while
 * other streams run).  No counterpart in the reference.  Inputs and outputs stay host arrays; the
 * device staging is a fixed array inside the library of at most 65536 points per call (larger n is
 * refused with PDG_ERR_ARG).  The first call on a device looks up that array's device address and
 * should come before any stream capture.  Calls share the array, so calls that overlap on the GPU
 * race; callers serialise them. */
int pdg_xc_evaluate_static(const char *functional, int n, const double *rho, const double *sigma, double *f,
                           double *vrho, double *vsigma);

/* SCF options and result, names after DIISSCFConverger (pMolecule/QCModel/DIISSCFConverger.py:175-189). */
typedef struct {
    double density_tolerance;  /* RMS density change */
    double energy_tolerance;   /* |dE| between cycles, hartree */
    int maximum_iterations;
    int maximum_history;       /* DIIS history, 0 (default 10) to 16; larger is refused with PDG_ERR_ARG */
    int use_guess;             /* 1: start from the density passed in; 0: core-Hamiltonian guess */
    double total_charge;       /* molecular charge (closed shell) */
} pdg_scf_options;

typedef struct {
    double energy_total;       /* E1 + E2 + E_xc + E_nuclear */
    double energy_one;         /* tr(D H) */
    double energy_two;         /* 1/2 tr(D F2) */
    double energy_xc;          /* quadrature energy */
    double energy_nuclear;     /* nuclear repulsion */
    double rho_integral;       /* integrated density (DFT) */
    double rms_density;        /* last RMS density change */
    int iterations;
    int converged;
    long long quartets;        /* screened shell quartets per Fock build */
    double s2;                 /* <S^2> (unrestricted runs; Sz(Sz+1) + n_beta - tr(Pa S Pb S)) */
} pdg_scf_result;

/* Closed-shell SCF on the device (S^-1/2, DIIS, FP64 diagonalisation, density).  density is
 * the guess on entry when use_guess is set and the converged density on exit (packed; may be
 * NULL if use_guess is 0).  The converged density and weighted density stay on the device
 * for pdg_scf_gradients.  Returns PDG_ERR_NOCONV when maximum_iterations is reached. */
int pdg_scf_run(pdg_context *ctx, const pdg_scf_options *options, double *density, pdg_scf_result *result);

/* Spin-unrestricted Hartree-Fock (the reference's unrestricted path: FockConstruction.c:258-264,
 * DIISSCFConverger.py:77-108): n_alpha + n_beta electrons; density_alpha / density_beta receive the
 * converged spin densities (packed, output basis; may be NULL unless options->use_guess, when they
 * are the start).  result->s2 is <S^2>.  Unrestricted Kohn-Sham is not supported
 * (PDG_ERR_UNSUPPORTED when a functional is set).  pdg_scf_gradients then gives its gradient. */
int pdg_uscf_run(pdg_context *ctx, const pdg_scf_options *options, int n_alpha, int n_beta, double *density_alpha,
                 double *density_beta, pdg_scf_result *result);

/* Full analytic gradient of the last converged pdg_scf_run (all terms, including the DFT
 * quadrature when a functional with a grid is set), ADDED to gradients3. */
int pdg_scf_gradients(pdg_context *ctx, double *gradients3);

/* Energy-weighted density of the last pdg_scf_run in the reference's convention (packed). */
int pdg_scf_weighted_density(pdg_context *ctx, double *weighted_density);

/* ---- QC/MM electrostatics with MM point charges ----
 * Replace the evaluator calls of NBModel/QCMMElectrostaticModelDensityFullGaussianBasis.py:131-185:
 * f2Cm1V (QCMMPotentials), f2Cm1R1 (QCMMGradients) and m1Cn1ER1 (QCMMCore), i.e.
 * GaussianBasisContainerIntegrals_f2Cp1.c:104,30 and GaussianBasisContainerIntegrals_p1Cq1.c:20 with
 * the MM charges; like the reference without widths, each charge is a normalised Gaussian of the
 * nuclear width.  Coordinates in bohr, charges in e, gradients in hartree/bohr. */

/* Set the MM charges the context's QC density feels (n = 0 clears them).  While set, the core
 * Hamiltonian of pdg_one_electron and pdg_scf_run includes their potentials, as the reference adds
 * its qcmmPotentials to the one-electron matrix; the nucleus-charge term is not included anywhere
 * else than pdg_qcmm_core. */
int pdg_set_point_charges(pdg_context *ctx, int n, const double *charges, const double *xyz);

/* Packed (output basis) electron-charge potentials V_ab = -sum_c q_c (ab|c). */
int pdg_qcmm_potentials(pdg_context *ctx, double *potentials);

/* Gradients of tr(P V) for the QC atoms and the charges, ADDED to gradients_qc (natom x 3) and
 * gradients_mm (n x 3).  density: packed output-basis P, or NULL for the last pdg_scf_run's. */
int pdg_qcmm_gradients(pdg_context *ctx, const double *density, double *gradients_qc, double *gradients_mm);

/* Nucleus-charge energy (hartree) and, when both arrays are given, its gradients ADDED to them. */
int pdg_qcmm_core(pdg_context *ctx, double *energy, double *gradients_qc, double *gradients_mm);

/* ---- instrumentation (no counterpart in the reference, which has no device code) ---- */

/* Number of kernel launches this library has issued in the process so far. */
int pdg_launch_count(long long *count);

/* The CUDA stream (cudaStream_t) on which the context issues all its work. */
int pdg_context_stream(pdg_context *ctx, void **stream);

/* Enable (1) or disable (0) per-region CUDA-event timing on the context stream; clears records.
 * Regions: "eri_jk", "eri_grad", "oneint", "oneint_grad", "xc_rho", "xc_vxc", "xc_grad",
 * "xc_weight_grad". */
int pdg_profile_enable(pdg_context *ctx, int enable);

/* Number of recorded calls of a region and their total device time in milliseconds. */
int pdg_profile_region(pdg_context *ctx, const char *region, int *count, double *total_ms);

/* Algorithmic FLOPs (and resident bytes read, for the XC kernels) of one call of a region
 * ("eri_jk", "eri_grad", "xc_rho", "xc_vxc") for the current geometry; quartets counts the
 * screened shell quartets of the ERI regions ("eri_grad": the quartets the last gradient
 * evaluated, by its Schwarz x |Gamma| screen; every Schwarz-screened one before any gradient). */
int pdg_work_estimate(pdg_context *ctx, const char *region, double *flops, double *bytes, long long *quartets);

/* Measured FP64 throughput of this device in TFLOP/s, the denominator of the FP64 kernels' roofline
 * fractions: kind 0 = the FP64 FMA pipe (DFMA on registers), 1 = the FP64 tensor path (DMMA,
 * mma.sync m8n8k4 f64).  Best of three event-timed launches of 4 CTAs per SM. */
int pdg_measure_fp64_peak(int device, int kind, double *tflops);

/* Tile autotuner of the two-electron kernels (no counterpart in the reference): for the current
 * geometry, times each candidate number of lanes per shell quartet (five tables by the ket pair's
 * primitive-count bucket) for every (bra class, ket class) of the J+K kernels that split quartets
 * over lanes, on a full J+K build of the density last loaded into the context, and keeps the
 * fastest for every later build in the process.  variants (36 ints, bra class x 6 + ket class, may
 * be NULL) receives the chosen table index per class pair (-1: not tuned). */
int pdg_autotune_eri(pdg_context *ctx, int *variants);

#ifdef __cplusplus
}
#endif
#endif
