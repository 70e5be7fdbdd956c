"""ctypes binding of the C-ABI library libpdgpu.so (declared in include/pdgpu.h).

The library is the product: there is no CPU fallback.  ``load()`` raises if the in-tree
library is missing (build it with ``python -m pdynamo3_b200.build``) and ``Context`` raises
``PDGError`` on any non-zero status, carrying the library's message.
"""
import ctypes
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libpdgpu.so")

PDG_OK = 0
PDG_ERR_ARG = 1
PDG_ERR_CUDA = 2
PDG_ERR_ALLOC = 3
PDG_ERR_STATE = 4
PDG_ERR_NOCONV = 5
PDG_ERR_TIMEOUT = 6
PDG_ERR_NAN = 7
PDG_ERR_UNSUPPORTED = 8

EXPORTS = [
    "pdg_version", "pdg_last_error", "pdg_context_create", "pdg_context_destroy", "pdg_basis_upload",
    "pdg_basis_size", "pdg_geometry_set", "pdg_set_eri_options", "pdg_one_electron", "pdg_fock_two_electron",
    "pdg_gradients", "pdg_set_functional", "pdg_grid_build", "pdg_fock_quadrature", "pdg_gradients_quadrature",
    "pdg_scf_run", "pdg_scf_gradients", "pdg_scf_weighted_density", "pdg_xc_evaluate",
    "pdg_launch_count", "pdg_context_stream", "pdg_profile_enable", "pdg_profile_region", "pdg_work_estimate",
    "pdg_xc_evaluate_static", "pdg_set_incremental", "pdg_set_point_charges", "pdg_qcmm_potentials",
    "pdg_qcmm_gradients", "pdg_qcmm_core", "pdg_uscf_run", "pdg_measure_fp64_peak", "pdg_autotune_eri",
]


class PDGError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("pdgpu error %d: %s" % (status, message))
        self.status = status


class ScfOptions(ctypes.Structure):
    _fields_ = [("density_tolerance", ctypes.c_double), ("energy_tolerance", ctypes.c_double),
                ("maximum_iterations", ctypes.c_int), ("maximum_history", ctypes.c_int),
                ("use_guess", ctypes.c_int), ("total_charge", ctypes.c_double)]


class ScfResult(ctypes.Structure):
    _fields_ = [("energy_total", ctypes.c_double), ("energy_one", ctypes.c_double), ("energy_two", ctypes.c_double),
                ("energy_xc", ctypes.c_double), ("energy_nuclear", ctypes.c_double), ("rho_integral", ctypes.c_double),
                ("rms_density", ctypes.c_double), ("iterations", ctypes.c_int), ("converged", ctypes.c_int),
                ("quartets", ctypes.c_longlong), ("s2", ctypes.c_double)]


_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_vp = ctypes.c_void_p


def load():
    """Load libpdgpu.so (no fallback: raises if it is missing or incomplete)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libpdgpu.so not built at %s (run python -m pdynamo3_b200.build)" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    for name in EXPORTS:
        getattr(L, name)  # raises AttributeError when a symbol is missing
    L.pdg_last_error.restype = ctypes.c_char_p
    L.pdg_context_create.argtypes = [ctypes.c_int, ctypes.POINTER(_vp)]
    L.pdg_context_destroy.argtypes = [_vp]
    L.pdg_basis_upload.argtypes = [_vp, ctypes.c_int, _dp, ctypes.c_int, _ip, _ip, _ip, _ip, _dp, _dp, ctypes.c_int,
                                   ctypes.c_int]
    L.pdg_basis_size.argtypes = [_vp, _ip, _ip]
    L.pdg_geometry_set.argtypes = [_vp, _dp]
    L.pdg_set_eri_options.argtypes = [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double]
    L.pdg_one_electron.argtypes = [_vp, _dp, _dp, _dp]
    L.pdg_fock_two_electron.argtypes = [_vp, _dp, ctypes.c_double, ctypes.c_int, _dp, _dp]
    L.pdg_gradients.argtypes = [_vp, _dp, _dp, ctypes.c_double, ctypes.c_int, _dp]
    L.pdg_set_functional.argtypes = [_vp, ctypes.c_char_p, _dp]
    L.pdg_grid_build.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_longlong)]
    L.pdg_fock_quadrature.argtypes = [_vp, _dp, _dp, _dp, _dp]
    L.pdg_gradients_quadrature.argtypes = [_vp, _dp, _dp]
    L.pdg_scf_run.argtypes = [_vp, ctypes.POINTER(ScfOptions), _dp, ctypes.POINTER(ScfResult)]
    L.pdg_scf_gradients.argtypes = [_vp, _dp]
    L.pdg_scf_weighted_density.argtypes = [_vp, _dp]
    L.pdg_xc_evaluate.argtypes = [ctypes.c_char_p, ctypes.c_int, _dp, _dp, _dp, _dp, _dp]
    L.pdg_launch_count.argtypes = [ctypes.POINTER(ctypes.c_longlong)]
    L.pdg_context_stream.argtypes = [_vp, ctypes.POINTER(_vp)]
    L.pdg_profile_enable.argtypes = [_vp, ctypes.c_int]
    L.pdg_profile_region.argtypes = [_vp, ctypes.c_char_p, _ip, _dp]
    L.pdg_work_estimate.argtypes = [_vp, ctypes.c_char_p, _dp, _dp, ctypes.POINTER(ctypes.c_longlong)]
    L.pdg_xc_evaluate_static.argtypes = [ctypes.c_char_p, ctypes.c_int, _dp, _dp, _dp, _dp, _dp]
    L.pdg_set_incremental.argtypes = [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_int]
    L.pdg_set_point_charges.argtypes = [_vp, ctypes.c_int, _dp, _dp]
    L.pdg_qcmm_potentials.argtypes = [_vp, _dp]
    L.pdg_qcmm_gradients.argtypes = [_vp, _dp, _dp, _dp]
    L.pdg_qcmm_core.argtypes = [_vp, _dp, _dp, _dp]
    L.pdg_uscf_run.argtypes = [_vp, ctypes.POINTER(ScfOptions), ctypes.c_int, ctypes.c_int, _dp, _dp,
                               ctypes.POINTER(ScfResult)]
    L.pdg_measure_fp64_peak.argtypes = [ctypes.c_int, ctypes.c_int, _dp]
    L.pdg_autotune_eri.argtypes = [_vp, _ip]
    _lib = L
    return L


def _d(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_ip)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def xc_evaluate(functional, rho, sigma):
    """Energy per volume and its derivatives of a functional at points (device evaluation)."""
    L = load()
    rho = _f64(rho)
    sigma = _f64(sigma)
    n = len(rho)
    f, vr, vs = np.zeros(n), np.zeros(n), np.zeros(n)
    st = L.pdg_xc_evaluate(functional.encode(), n, _d(rho), _d(sigma), _d(f), _d(vr), _d(vs))
    if st != PDG_OK:
        raise PDGError(st, L.pdg_last_error().decode(errors="replace"))
    return f, vr, vs


def xc_evaluate_static(functional, rho, sigma):
    """xc_evaluate through the library's fixed device staging area (no device allocation; at most
    65536 points per call; calls must not overlap)."""
    L = load()
    rho = _f64(rho)
    sigma = _f64(sigma)
    n = len(rho)
    f, vr, vs = np.zeros(n), np.zeros(n), np.zeros(n)
    st = L.pdg_xc_evaluate_static(functional.encode(), n, _d(rho), _d(sigma), _d(f), _d(vr), _d(vs))
    if st != PDG_OK:
        raise PDGError(st, L.pdg_last_error().decode(errors="replace"))
    return f, vr, vs


class Context:
    """One device context (basis, geometry, resident SCF state)."""

    def __init__(self, device=0):
        self.L = load()
        h = _vp()
        self._check(self.L.pdg_context_create(int(device), ctypes.byref(h)))
        self.h = h
        self.n = 0
        # the two-electron options last set (the library's defaults until set_eri_options)
        self.eri_options = dict(schwarz_cut=1e-13, tei_underflow=1e-12, precision_mode=0, mixed_cut=1e-6)
        self.natom = 0

    def _check(self, st):
        if st != PDG_OK:
            raise PDGError(st, self.L.pdg_last_error().decode(errors="replace"))

    def close(self):
        if getattr(self, "h", None):
            self.L.pdg_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_basis(self, shells):
        args = shells.upload_args()
        self._keep = [_f64(args[1]), np.ascontiguousarray(args[3], dtype=np.int32),
                      np.ascontiguousarray(args[4], dtype=np.int32), np.ascontiguousarray(args[5], dtype=np.int32),
                      np.ascontiguousarray(args[6], dtype=np.int32), _f64(args[7]), _f64(args[8])]
        z, sa, lo, hi, npr, ex, co = self._keep
        self._check(self.L.pdg_basis_upload(self.h, int(args[0]), _d(z), int(args[2]), _i(sa), _i(lo), _i(hi), _i(npr),
                                            _d(ex), _d(co), int(args[9]), int(shells.spherical)))
        n, nc = ctypes.c_int(0), ctypes.c_int(0)
        self._check(self.L.pdg_basis_size(self.h, ctypes.byref(n), ctypes.byref(nc)))
        self.n, self.ncart = n.value, nc.value
        self.natom = int(args[0])

    def set_geometry(self, coordinates_bohr):
        self._check(self.L.pdg_geometry_set(self.h, _d(_f64(coordinates_bohr).reshape(-1))))

    def set_eri_options(self, schwarz_cut=1e-13, tei_underflow=1e-12, precision_mode=0, mixed_cut=1e-6):
        self._check(self.L.pdg_set_eri_options(self.h, float(schwarz_cut), float(tei_underflow), int(precision_mode),
                                               float(mixed_cut)))
        self.eri_options = dict(schwarz_cut=float(schwarz_cut), tei_underflow=float(tei_underflow),
                                precision_mode=int(precision_mode), mixed_cut=float(mixed_cut))

    def set_incremental(self, enable=True, density_cut=1e-13, rebuild_period=16):
        self._check(self.L.pdg_set_incremental(self.h, int(enable), float(density_cut), int(rebuild_period)))

    def npacked(self):
        return self.n * (self.n + 1) // 2

    def one_electron(self):
        S = np.zeros(self.npacked())
        H = np.zeros(self.npacked())
        e = ctypes.c_double(0.0)
        self._check(self.L.pdg_one_electron(self.h, _d(S), _d(H), ctypes.byref(e)))
        return S, H, e.value

    def fock_two_electron(self, density, exchange_scaling=1.0, do_coulomb=True):
        P = _f64(density)
        F = np.zeros(self.npacked())
        e2 = ctypes.c_double(0.0)
        self._check(self.L.pdg_fock_two_electron(self.h, _d(P), float(exchange_scaling), int(do_coulomb), _d(F),
                                                 ctypes.byref(e2)))
        return F, e2.value

    def gradients(self, density, weighted_density, exchange_scaling=1.0, do_coulomb=True):
        g = np.zeros(3 * self.natom)
        self._check(self.L.pdg_gradients(self.h, _d(_f64(density)), _d(_f64(weighted_density)), float(exchange_scaling),
                                         int(do_coulomb), _d(g)))
        return g.reshape(-1, 3)

    def set_functional(self, name):
        cx = ctypes.c_double(1.0)
        self._check(self.L.pdg_set_functional(self.h, name.encode(), ctypes.byref(cx)))
        return cx.value

    def grid_build(self, accuracy=3, n_radial=0, angular_l=0):
        n = ctypes.c_longlong(0)
        self._check(self.L.pdg_grid_build(self.h, int(accuracy), int(n_radial), int(angular_l), ctypes.byref(n)))
        return n.value

    def fock_quadrature(self, density, fock=None):
        F = np.zeros(self.npacked()) if fock is None else _f64(fock).copy()
        exc, rho = ctypes.c_double(0.0), ctypes.c_double(0.0)
        self._check(self.L.pdg_fock_quadrature(self.h, _d(_f64(density)), _d(F), ctypes.byref(exc), ctypes.byref(rho)))
        return F, exc.value, rho.value

    def gradients_quadrature(self, density):
        g = np.zeros(3 * self.natom)
        self._check(self.L.pdg_gradients_quadrature(self.h, _d(_f64(density)), _d(g)))
        return g.reshape(-1, 3)

    def scf(self, density_tolerance=1e-8, energy_tolerance=2e-4, maximum_iterations=100, maximum_history=10,
            guess=None, total_charge=0.0, raise_on_noconv=True):
        opt = ScfOptions(float(density_tolerance), float(energy_tolerance), int(maximum_iterations), int(maximum_history),
                         1 if guess is not None else 0, float(total_charge))
        P = _f64(guess).copy() if guess is not None else np.zeros(self.npacked())
        res = ScfResult()
        st = self.L.pdg_scf_run(self.h, ctypes.byref(opt), _d(P), ctypes.byref(res))
        if st != PDG_OK and not (st == PDG_ERR_NOCONV and not raise_on_noconv):
            self._check(st)
        return P, res

    def uscf(self, n_alpha, n_beta, density_tolerance=1e-8, energy_tolerance=2e-4, maximum_iterations=100,
             maximum_history=10, guess=None, total_charge=0.0, raise_on_noconv=True):
        """Spin-unrestricted Hartree-Fock; returns (Pa, Pb, result), result.s2 = <S^2>."""
        opt = ScfOptions(float(density_tolerance), float(energy_tolerance), int(maximum_iterations), int(maximum_history),
                         1 if guess is not None else 0, float(total_charge))
        Pa = _f64(guess[0]).copy() if guess is not None else np.zeros(self.npacked())
        Pb = _f64(guess[1]).copy() if guess is not None else np.zeros(self.npacked())
        res = ScfResult()
        st = self.L.pdg_uscf_run(self.h, ctypes.byref(opt), int(n_alpha), int(n_beta), _d(Pa), _d(Pb), ctypes.byref(res))
        if st != PDG_OK and not (st == PDG_ERR_NOCONV and not raise_on_noconv):
            self._check(st)
        return Pa, Pb, res

    def scf_gradients(self):
        g = np.zeros(3 * self.natom)
        self._check(self.L.pdg_scf_gradients(self.h, _d(g)))
        return g.reshape(-1, 3)

    # ---- QC/MM electrostatics with MM point charges (bohr, e; hartree/bohr) ----
    def set_point_charges(self, charges, coordinates_bohr):
        q = _f64(charges).reshape(-1)
        x = _f64(coordinates_bohr).reshape(-1)
        if len(x) != 3 * len(q):
            raise ValueError("set_point_charges: %d charges but %d coordinates" % (len(q), len(x)))
        self.nmm = len(q)
        self._check(self.L.pdg_set_point_charges(self.h, len(q), _d(q) if len(q) else None, _d(x) if len(q) else None))

    def qcmm_potentials(self):
        V = np.zeros(self.npacked())
        self._check(self.L.pdg_qcmm_potentials(self.h, _d(V)))
        return V

    def qcmm_gradients(self, density=None):
        """Gradients of tr(P V_mm): (atoms x 3, charges x 3); density None = the last SCF's."""
        nm = getattr(self, "nmm", 0)
        gq = np.zeros(3 * self.natom)
        gm = np.zeros(3 * max(1, nm))
        P = None if density is None else _f64(density)
        self._check(self.L.pdg_qcmm_gradients(self.h, _d(P), _d(gq), _d(gm)))
        return gq.reshape(-1, 3), gm[:3 * nm].reshape(-1, 3)

    def qcmm_core(self, gradients=True):
        nm = getattr(self, "nmm", 0)
        e = np.zeros(1)
        gq = np.zeros(3 * self.natom)
        gm = np.zeros(3 * max(1, nm))
        self._check(self.L.pdg_qcmm_core(self.h, _d(e), _d(gq) if gradients else None, _d(gm) if gradients else None))
        return (float(e[0]), gq.reshape(-1, 3), gm[:3 * nm].reshape(-1, 3)) if gradients else float(e[0])

    def scf_weighted_density(self):
        W = np.zeros(self.npacked())
        self._check(self.L.pdg_scf_weighted_density(self.h, _d(W)))
        return W

    # ---- instrumentation ----
    def stream_handle(self):
        s = _vp()
        self._check(self.L.pdg_context_stream(self.h, ctypes.byref(s)))
        return s.value or 0

    def profile(self, enable=True):
        self._check(self.L.pdg_profile_enable(self.h, int(enable)))

    def profile_region(self, name):
        c, t = ctypes.c_int(0), ctypes.c_double(0.0)
        self._check(self.L.pdg_profile_region(self.h, name.encode(), ctypes.byref(c), ctypes.byref(t)))
        return c.value, t.value

    def autotune_eri(self):
        """Tune the J+K kernels' lanes per quartet on this context's geometry and last density
        (process-wide); returns {(bra class, ket class): table index}."""
        v = np.zeros(36, dtype=np.int32)
        self._check(self.L.pdg_autotune_eri(self.h, v.ctypes.data_as(_ip)))
        return {(k // 6, k % 6): int(v[k]) for k in range(36) if v[k] >= 0}

    def fp32_quartets(self):
        """Shell quartets evaluated in FP32 by this context's mixed-precision builds so far."""
        return self.work_estimate("eri_jk_fp32")[2]

    def work_estimate(self, region):
        f, b, q = ctypes.c_double(0.0), ctypes.c_double(0.0), ctypes.c_longlong(0)
        self._check(self.L.pdg_work_estimate(self.h, region.encode(), ctypes.byref(f), ctypes.byref(b), ctypes.byref(q)))
        return f.value, b.value, q.value


def measure_fp64_peak(device=0, kind=0):
    """Measured FP64 TFLOP/s of the device: kind 0 the FMA pipe (DFMA), 1 the DMMA tensor path."""
    t = np.zeros(1)
    st = load().pdg_measure_fp64_peak(int(device), int(kind), _d(t))
    if st != PDG_OK:
        raise PDGError(st, load().pdg_last_error().decode(errors="replace"))
    return float(t[0])


def launch_count():
    c = ctypes.c_longlong(0)
    load().pdg_launch_count(ctypes.byref(c))
    return c.value
