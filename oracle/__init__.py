"""ORACLE -- test infrastructure only (checker for tests/, smoke() and bench.py's CPU baseline).

ctypes binding of the C restatement in oracle.c (built into oracle/_build/liboracle.so by
oracle/build.py) plus numpy restatements of the SCF driver.  Parity with the pDynamo3 reference is
pinned by tests/test_oracle.py against fixtures the reference produced (tests/golden).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def lib():
    global _lib
    if _lib is None:
        from oracle.build import build
        build()   # rebuilds when oracle.c is newer than the library
        L = ctypes.CDLL(LIB_PATH)
        L.orc_rys_roots.argtypes = [ctypes.c_int, ctypes.c_double, _dp, _dp]
        L.orc_basis.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _ip, _ip, _ip, _ip, _dp, _dp, ctypes.c_int]
        L.orc_basis.restype = ctypes.c_int
        L.orc_nbf.restype = ctypes.c_int
        L.orc_geometry.argtypes = [_dp]
        L.orc_fock.argtypes = [_dp, ctypes.c_double, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_long)]
        L.orc_fock.restype = ctypes.c_double
        L.orc_eri_gradient.argtypes = [_dp, ctypes.c_double, ctypes.c_int, _dp]
        L.orc_one_electron.argtypes = [_dp, _dp]
        L.orc_one_electron.restype = ctypes.c_double
        L.orc_one_electron_gradient.argtypes = [_dp, _dp, _dp]
        L.orc_set_sample.argtypes = [ctypes.c_uint, ctypes.c_uint, ctypes.c_uint]
        L.orc_store_integrals.restype = ctypes.c_long
        L.orc_fock_stored.argtypes = [_dp, ctypes.c_double, ctypes.c_int, _dp]
        L.orc_fock_stored.restype = ctypes.c_double
        L.orc_set_root_provider.argtypes = [ctypes.c_void_p]
        L.orc_set_point_charges.argtypes = [ctypes.c_int, _dp, _dp]
        L.orc_qcmm_potentials.argtypes = [_dp]
        L.orc_qcmm_gradient.argtypes = [_dp, _dp, _dp]
        L.orc_qcmm_core.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_qcmm_core.restype = ctypes.c_double
        _lib = L
    return _lib


REF_ROOTS_PATH = os.path.join(HERE, "_ref", "librys_ref.so")
_ref_roots = None


def reference_roots_available():
    return os.path.exists(REF_ROOTS_PATH)


def use_reference_roots(enable=True):
    """Switch the oracle's Rys rule to the reference's libcint routine compiled from its own
    sources (oracle/_ref/librys_ref.so, built by oracle/build_ref.sh); False restores the
    restated rule.  Returns whether the reference routine is in use."""
    global _ref_roots
    L = lib()
    if not enable or not reference_roots_available():
        L.orc_set_root_provider(None)
        return False
    if _ref_roots is None:
        _ref_roots = ctypes.CDLL(REF_ROOTS_PATH)
    L.orc_set_root_provider(ctypes.cast(_ref_roots.CINTrys_roots, ctypes.c_void_p).value)
    return True


def reference_rys_roots(n, x):
    """Nodes u = t^2 and weights of the reference's libcint rule (needs oracle/_ref/librys_ref.so)."""
    global _ref_roots
    if _ref_roots is None:
        _ref_roots = ctypes.CDLL(REF_ROOTS_PATH)
    r = np.zeros(n)
    w = np.zeros(n)
    dp = ctypes.POINTER(ctypes.c_double)
    _ref_roots.CINTrys_roots(int(n), ctypes.c_double(x), r.ctypes.data_as(dp), w.ctypes.data_as(dp))
    return r / (1.0 + r), w


def rys_roots(n, x):
    u = np.zeros(n)
    w = np.zeros(n)
    lib().orc_rys_roots(n, float(x), u, w)
    return u, w


class Oracle:
    """CPU restatement of the reference's HF integral path for one molecule (Cartesian basis)."""

    def __init__(self, shells, coordinates_bohr):
        L = lib()
        st = L.orc_basis(*shells.upload_args())
        if st != 0:
            raise RuntimeError("oracle basis setup failed (%d)" % st)
        self.n = L.orc_nbf()
        self.natom = len(shells.atomic_numbers)
        L.orc_geometry(np.ascontiguousarray(coordinates_bohr, dtype=np.float64).reshape(-1))

    def one_electron(self):
        npk = self.n * (self.n + 1) // 2
        S = np.zeros(npk)
        H = np.zeros(npk)
        enuc = lib().orc_one_electron(S, H)
        return S, H, enuc

    def fock(self, P, cx=1.0, do_coulomb=True):
        F = np.zeros(self.n * (self.n + 1) // 2)
        cnt = ctypes.c_long(0)
        e2 = lib().orc_fock(np.ascontiguousarray(P, dtype=np.float64), float(cx), int(do_coulomb), F, ctypes.byref(cnt))
        return F, e2, cnt.value

    def store_integrals(self):
        """Compute and keep the unique integrals above the storage underflow (the reference's
        conventional path); returns their number."""
        return int(lib().orc_store_integrals())

    def fock_stored(self, P, cx=1.0, do_coulomb=True):
        """F2, E2 of P from the stored integrals (store_integrals first)."""
        F = np.zeros(self.n * (self.n + 1) // 2)
        e2 = lib().orc_fock_stored(np.ascontiguousarray(P, dtype=np.float64), float(cx), int(do_coulomb), F)
        return F, e2

    def free_stored(self):
        lib().orc_free_stored()

    def gradients(self, P, Wref, cx=1.0, do_coulomb=True):
        """Gradient (hartree/bohr) of nuclear + one-electron + two-electron terms; Wref in the
        reference's convention (-2 sum e n C C^T)."""
        g = np.zeros(3 * self.natom)
        P = np.ascontiguousarray(P, dtype=np.float64)
        lib().orc_one_electron_gradient(P, np.ascontiguousarray(-0.5 * np.asarray(Wref)), g)
        lib().orc_eri_gradient(P, float(cx), int(do_coulomb), g)
        return g.reshape(-1, 3)

    # QC/MM electrostatics with MM point charges (charges in e, coordinates in bohr)
    def set_point_charges(self, charges, coordinates_bohr):
        q = np.ascontiguousarray(charges, dtype=np.float64).reshape(-1)
        x = np.ascontiguousarray(coordinates_bohr, dtype=np.float64).reshape(-1)
        self.nmm = len(q)
        lib().orc_set_point_charges(len(q), q if len(q) else np.zeros(1), x if len(q) else np.zeros(3))

    def qcmm_potentials(self):
        """Packed normalised Cartesian V_mm = -sum_c q_c (ab|c) (added to the core Hamiltonian)."""
        V = np.zeros(self.n * (self.n + 1) // 2)
        lib().orc_qcmm_potentials(V)
        return V

    def qcmm_gradients(self, P):
        """Gradient of tr(P V_mm): (atoms x 3, charges x 3) in hartree/bohr."""
        gq = np.zeros(3 * self.natom)
        gm = np.zeros(3 * max(1, self.nmm))
        lib().orc_qcmm_gradient(np.ascontiguousarray(P, dtype=np.float64), gq, gm)
        return gq.reshape(-1, 3), gm[:3 * self.nmm].reshape(-1, 3)

    def qcmm_core(self):
        """Nucleus-charge energy and its gradients (atoms x 3, charges x 3)."""
        gq = np.zeros(3 * self.natom)
        gm = np.zeros(3 * max(1, self.nmm))
        e = lib().orc_qcmm_core(gq.ctypes.data, gm.ctypes.data)
        return e, gq.reshape(-1, 3), gm[:3 * self.nmm].reshape(-1, 3)


def unpack(p, n):
    m = np.zeros((n, n))
    i, j = np.tril_indices(n)
    m[i, j] = p
    m[j, i] = p
    return m


def pack(m):
    return m[np.tril_indices(m.shape[0])].copy()


def scf(S, H, enuc, fock, nocc, tol=1e-10, maxit=200, guess=None):
    """Closed-shell DIIS SCF in numpy (restates the converger's fixed point: F C = S C e with
    P = 2 C_occ C_occ^T).  fock(P_packed) -> (F2_packed, E2)."""
    n = int(round((np.sqrt(8 * len(S) + 1) - 1) / 2))
    Sm, Hm = unpack(S, n), unpack(H, n)
    s, U = np.linalg.eigh(Sm)
    X = U @ np.diag(s ** -0.5) @ U.T
    def diag(F):
        e, C = np.linalg.eigh(X.T @ F @ X)
        C = X @ C
        return e, C
    if guess is None:
        e, C = diag(Hm)
        P = 2 * C[:, :nocc] @ C[:, :nocc].T
    else:
        P = unpack(guess, n)
    fs, es = [], []
    E_old = 0.0
    for it in range(maxit):
        F2, e2 = fock(pack(P))
        F = Hm + unpack(F2, n)
        E = np.sum(P * Hm) + e2 + enuc
        err = X.T @ (F @ P @ Sm - Sm @ P @ F) @ X
        fs.append(F); es.append(err)
        fs, es = fs[-10:], es[-10:]
        k = len(fs)
        B = -np.ones((k + 1, k + 1)); B[k, k] = 0
        for a in range(k):
            for b in range(k):
                B[a, b] = np.sum(es[a] * es[b])
        rhs = np.zeros(k + 1); rhs[k] = -1
        try:
            c = np.linalg.solve(B, rhs)[:k]
            Fx = sum(ci * fi for ci, fi in zip(c, fs))
        except np.linalg.LinAlgError:
            Fx = F
        eps, C = diag(Fx)
        Pn = 2 * C[:, :nocc] @ C[:, :nocc].T
        rms = np.sqrt(np.mean((Pn - P) ** 2))
        P = Pn
        if rms < tol and abs(E - E_old) < 1e-10 and it > 0:
            F2, e2 = fock(pack(P))
            E = np.sum(P * Hm) + e2 + enuc
            W = -2.0 * (2 * (C[:, :nocc] * eps[:nocc]) @ C[:, :nocc].T)
            return E, pack(P), pack(W), it + 1
        E_old = E
    raise RuntimeError("oracle SCF did not converge")


def uscf(S, H, enuc, jk, na, nb, tol=1e-10, maxit=300):
    """Spin-unrestricted DIIS SCF in numpy (the fixed point F_s C_s = S C_s e_s, P_s = C_s,occ C_s,occ^T
    with F_s = H + J(P_a + P_b) - K(P_s)).  jk(P_packed) -> (J_packed, K_packed) with K = 2 x the
    exchange part of the restricted Fock builder's convention.  Returns (E, Pa, Pb, Wa + Wb, <S^2>),
    W standard convention (sum e C C^T), packed."""
    n = int(round((np.sqrt(8 * len(S) + 1) - 1) / 2))
    Sm, Hm = unpack(S, n), unpack(H, n)
    s, U = np.linalg.eigh(Sm)
    X = U @ np.diag(s ** -0.5) @ U.T

    def diag(F):
        e, C = np.linalg.eigh(X.T @ F @ X)
        return e, X @ C
    e, C = diag(Hm)
    Pa, Pb = C[:, :na] @ C[:, :na].T, C[:, :nb] @ C[:, :nb].T
    if na == nb:  # break the spin symmetry of a singlet start
        Pa = Pa + 0.05 * (C[:, [na]] @ C[:, [na]].T - C[:, [na - 1]] @ C[:, [na - 1]].T)
    hist, E_old = [], None
    for it in range(maxit):
        Ja, Ka = jk(pack(Pa))
        Jb, Kb = jk(pack(Pb))
        J = unpack(Ja, n) + unpack(Jb, n)
        Fa, Fb = Hm + J - unpack(Ka, n), Hm + J - unpack(Kb, n)
        E = 0.5 * (np.sum((Pa + Pb) * Hm) + np.sum(Pa * Fa) + np.sum(Pb * Fb)) + enuc
        ea = X.T @ (Fa @ Pa @ Sm - Sm @ Pa @ Fa) @ X
        eb = X.T @ (Fb @ Pb @ Sm - Sm @ Pb @ Fb) @ X
        hist.append((Fa, Fb, ea, eb))
        hist = hist[-10:]
        k = len(hist)
        B = -np.ones((k + 1, k + 1)); B[k, k] = 0
        for i in range(k):
            for j in range(k):
                B[i, j] = np.sum(hist[i][2] * hist[j][2]) + np.sum(hist[i][3] * hist[j][3])
        rhs = np.zeros(k + 1); rhs[k] = -1
        try:
            c = np.linalg.solve(B, rhs)[:k]
            Fxa = sum(ci * h[0] for ci, h in zip(c, hist))
            Fxb = sum(ci * h[1] for ci, h in zip(c, hist))
        except np.linalg.LinAlgError:
            Fxa, Fxb = Fa, Fb
        ea_, Ca = diag(Fxa)
        eb_, Cb = diag(Fxb)
        Pan, Pbn = Ca[:, :na] @ Ca[:, :na].T, Cb[:, :nb] @ Cb[:, :nb].T
        rms = max(np.sqrt(np.mean((Pan - Pa) ** 2)), np.sqrt(np.mean((Pbn - Pb) ** 2)))
        Pa, Pb = Pan, Pbn
        if rms < tol and E_old is not None and abs(E - E_old) < 1e-11:
            Ja, Ka = jk(pack(Pa))
            Jb, Kb = jk(pack(Pb))
            J = unpack(Ja, n) + unpack(Jb, n)
            Fa, Fb = Hm + J - unpack(Ka, n), Hm + J - unpack(Kb, n)
            E = 0.5 * (np.sum((Pa + Pb) * Hm) + np.sum(Pa * Fa) + np.sum(Pb * Fb)) + enuc
            W = Pa @ Fa @ Pa + Pb @ Fb @ Pb
            sz = 0.5 * (na - nb)
            s2 = sz * (sz + 1) + nb - np.trace(Pa @ Sm @ Pb @ Sm)
            return E, pack(Pa), pack(Pb), pack(W), s2
        E_old = E
    raise RuntimeError("oracle UHF did not converge")
