// Closed-shell SCF on the device in FP64: symmetric orthogonaliser, Pulay DIIS on the
// commutator error X^T (F P S - S P F) X, cuSOLVER diagonalisation, density and energy.
//
// Plays the role of DIISSCFConverger.Iterate (pMolecule/QCModel/DIISSCFConverger.py:365-385),
// QCOrbitals.MakeFromFock (QCOrbitals.py:130-144), GetOrthogonalizer (QCModelBase.py:313-342)
// and GetWeightedDensity (QCModelDFT.py:346-353) for spin-restricted closed shells.
// Convergence follows DIISSCFConverger.Continue (:206-216): RMS density change <= tolerance and
// signed energy change <= energy tolerance.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "context.h"

int pdg_compute_one_electron(pdg_context *ctx);
int pdg_cart_to_out(pdg_context *ctx, const double *Mc, double *Mo);
int pdg_out_to_cart(pdg_context *ctx, const double *Mo, double *Mc);
int pdg_fock2_scf(pdg_context *ctx, double cx, bool doJ, double *d_F2);
int pdg_store_packed(pdg_context *ctx, const double *d_full_out, double *packed_host);
int pdg_gradients_device(pdg_context *ctx, double cx, bool doJ, std::vector<double> &g);
int pdg_oneint_grad(pdg_context *ctx, const double *d_P, const double *d_W, double *d_grad);
int pdg_eri_grad(pdg_context *ctx, const double *d_D, double cx, bool doJ, double *d_grad);
int pdg_shell_pair_dmax(pdg_context *ctx, const double *d_D, double *d_dmax);
int pdg_eri_jk_screened(pdg_context *ctx, const double *d_D, double *d_J, double *d_K, bool doJ, bool doK,
                        const double *d_dmax, double dcut);
void pdg_launch_sym_combine2(pdg_context *ctx, int n, const double *J, const double *K, double cJ, double cK,
                             const double *norm, double *F);
double pdg_nuclear_energy(const pdg_context *ctx, std::vector<double> *grad);
void pdg_launch_unpack(pdg_context *ctx, int n, const double *packed_dev, const double *norm, double *full);
void pdg_launch_scale_full(pdg_context *ctx, int n, double *M, const double *norm);
// DFT hooks (dft.cu)
bool pdg_dft_active(const pdg_context *ctx);
double pdg_dft_exchange_scaling(const pdg_context *ctx);
int pdg_dft_fock_device(pdg_context *ctx, double *d_Fcart, double *exc, double *rho);
int pdg_dft_grad_device(pdg_context *ctx, double *d_grad);
double pdg_dft_last_vxc_trace(const pdg_context *ctx);  // tr(D' V_xc') of the last quadrature Fock

namespace {

struct ScfState {
    int m = 0;
    double *S = nullptr, *H = nullptr, *X = nullptr, *P = nullptr, *Pold = nullptr, *F = nullptr, *F2 = nullptr;
    double *C = nullptr, *eps = nullptr, *T1 = nullptr, *T2 = nullptr, *work = nullptr;
    int lwork = 0;
    int *info = nullptr;
    std::vector<double *> Fh, Eh;  // all buffers belong to the context's pool
};

// Device-resident results of the last SCF, kept per context.
struct ScfResident {
    int m = 0, nocc = 0;
    double *P = nullptr, *C = nullptr, *eps = nullptr;
    double *F = nullptr;    // the Fock matrix P is the projector density of (purification path)
    bool orbitals = false;  // C, eps hold the orbitals (eigensolver path)
    // unrestricted: P is the total density; Pa, Pb the spin densities, Fa, Fb the Fock matrices
    // whose projectors they are
    bool unrestricted = false;
    double *Pa = nullptr, *Pb = nullptr, *Fa = nullptr, *Fb = nullptr;
    double cx = 1.0;
    bool valid = false;
};

std::map<const pdg_context *, ScfResident> g_resident;  // node-based: references stay valid
std::mutex g_resident_mutex;

ScfResident &resident(const pdg_context *ctx) {
    std::lock_guard<std::mutex> lock(g_resident_mutex);
    return g_resident[ctx];
}

int gemm(pdg_context *ctx, cublasOperation_t ta, cublasOperation_t tb, int m, int n, int k, double alpha,
         const double *A, int lda, const double *B, int ldb, double beta, double *C, int ldc) {
    if (cublasDgemm(ctx->cublas, ta, tb, m, n, k, &alpha, A, lda, B, ldb, &beta, C, ldc) != CUBLAS_STATUS_SUCCESS) {
        pdg_set_error("cublasDgemm failed");
        return PDG_ERR_CUDA;
    }
    return PDG_OK;
}

// Symmetric eigen-decomposition in place (column-major, eigenvectors in columns, ascending).
int syevd(pdg_context *ctx, ScfState &st, double *A, double *w) {
    const int m = st.m;
    if (st.work == nullptr) {
        if (cusolverDnDsyevd_bufferSize(ctx->cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, m, A, m, w, &st.lwork) !=
            CUSOLVER_STATUS_SUCCESS) { pdg_set_error("syevd buffer query failed"); return PDG_ERR_CUDA; }
        st.work = (double *)pdg_pool(ctx, "scf.syevd_work", (size_t)st.lwork * sizeof(double));
        st.info = (int *)pdg_pool(ctx, "scf.syevd_info", sizeof(int));
        if (!st.work || !st.info) { pdg_set_error("SCF allocation failed"); return PDG_ERR_ALLOC; }
    }
    if (cusolverDnDsyevd(ctx->cusolver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, m, A, m, w, st.work, st.lwork, st.info) !=
        CUSOLVER_STATUS_SUCCESS) { pdg_set_error("cusolverDnDsyevd failed"); return PDG_ERR_CUDA; }
    return PDG_OK;
}

__global__ void scale_cols_kernel(int m, double *V, const double *w, double power, double cut) {
    const int j = blockIdx.y;
    const double s = w[j] > cut ? pow(w[j], power) : 0.0;
    for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < m; i += blockDim.x * gridDim.x) V[(long long)j * m + i] *= s;
}

__global__ void diff_sq_kernel(long long n, const double *a, const double *b, double *out) {
    __shared__ double sh[256];
    double s = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)blockDim.x * gridDim.x) {
        const double d = a[k] - b[k];
        s += d * d;
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(out, sh[0]);
}

__global__ void antisym_kernel(int m, const double *A, double *E) {
    const int i = blockIdx.y;
    for (int j = threadIdx.x + blockIdx.x * blockDim.x; j < m; j += blockDim.x * gridDim.x)
        E[(long long)i * m + j] = A[(long long)i * m + j] - A[(long long)j * m + i];
}

__global__ void add2_kernel(long long n, const double *a, const double *b, double *c) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)blockDim.x * gridDim.x) c[k] = a[k] + b[k];
}

dim3 rgrid(int m) { return dim3((m + 255) / 256 < 4 ? (m + 255) / 256 : 4, m); }

// Up to PDG_MAX_DIIS (16) dot products a_k . b_k and, optionally, max |x| of one more array, in one launch into
// dst[0..k-1] (and dst[k]) without a host synchronisation; the SCF reads them with its next copy.
struct DotBatch {
    const double *a[PDG_MAX_DIIS], *b[PDG_MAX_DIIS];
    int k = 0;
    const double *amax = nullptr;
    void add(const double *x, const double *y) {
        if (k < PDG_MAX_DIIS) { a[k] = x; b[k] = y; ++k; }
    }
};

__global__ void dot_batch_kernel(long long n, DotBatch d, double *dst) {
    __shared__ double sh[256];
    const int v = blockIdx.y;
    const bool isdot = v < d.k;
    const double *x = isdot ? d.a[v] : d.amax, *y = isdot ? d.b[v] : nullptr;
    double s = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)blockDim.x * gridDim.x)
        s = isdot ? s + x[k] * y[k] : fmax(s, fabs(x[k]));
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) sh[threadIdx.x] = isdot ? sh[threadIdx.x] + sh[threadIdx.x + o] : fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (isdot) atomicAdd(dst + v, sh[0]);
        else atomicMax((unsigned long long *)(dst + v), (unsigned long long)__double_as_longlong(sh[0]));  // >= 0
    }
}

// Zero dst[0..k] and launch the batch (stream-ordered, no synchronisation).
int dots_launch(pdg_context *ctx, long long n, const DotBatch &d, double *dst) {
    const int nv = d.k + (d.amax ? 1 : 0);
    if (nv == 0) return PDG_OK;
    PDG_CUDA(cudaMemsetAsync(dst, 0, nv * sizeof(double), ctx->stream));
    { dot_batch_kernel<<<dim3(74, nv), 256, 0, ctx->stream>>>(n, d, dst); pdg_count_launch(); }
    return PDG_OK;
}

// Copy cnt reduction results to the host (the one synchronisation).
int fetch(pdg_context *ctx, const double *dst, int cnt, double *host) {
    PDG_CUDA(cudaMemcpyAsync(host, dst, cnt * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    return PDG_OK;
}

bool solve_small(int n, std::vector<double> A, std::vector<double> &b) {
    // Gaussian elimination with partial pivoting, A row-major n x n.
    for (int c = 0; c < n; ++c) {
        int p = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(A[r * n + c]) > std::fabs(A[p * n + c])) p = r;
        if (std::fabs(A[p * n + c]) < 1e-300) return false;
        if (p != c) {
            for (int k = 0; k < n; ++k) std::swap(A[c * n + k], A[p * n + k]);
            std::swap(b[c], b[p]);
        }
        for (int r = c + 1; r < n; ++r) {
            const double f = A[r * n + c] / A[c * n + c];
            for (int k = c; k < n; ++k) A[r * n + k] -= f * A[c * n + k];
            b[r] -= f * b[c];
        }
    }
    for (int c = n - 1; c >= 0; --c) {
        double s = b[c];
        for (int k = c + 1; k < n; ++k) s -= A[c * n + k] * b[k];
        b[c] = s / A[c * n + c];
    }
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(b[i])) return false;
    return true;
}

__global__ void scale_columns_kernel(int m, int k, const double *C, const double *w, double *out) {
    const int j = blockIdx.y;
    if (j >= k) return;
    for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < m; i += blockDim.x * gridDim.x)
        out[(long long)j * m + i] = C[(long long)j * m + i] * w[j];
}

// Density P = 2 C_occ C_occ^T (column-major C, m x m), or sum_i occ_i C_i C_i^T when the context
// carries explicit occupations (fractional-occupation atomic runs of the density guess).
int make_density(pdg_context *ctx, ScfState &st, int nocc, double *P) {
    if (ctx->occ.empty())
        return gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_T, st.m, st.m, nocc, 2.0, st.C, st.m, st.C, st.m, 0.0, P, st.m);
    const int k = (int)std::min<size_t>(ctx->occ.size(), (size_t)st.m);
    PDG_CUDA(cudaMemcpyAsync(ctx->d_scal, ctx->occ.data(), k * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    { scale_columns_kernel<<<dim3((st.m + 255) / 256, k), 256, 0, ctx->stream>>>(st.m, k, st.C, ctx->d_scal, st.T1); pdg_count_launch(); }
    return gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_T, st.m, st.m, k, 1.0, st.T1, st.m, st.C, st.m, 0.0, P, st.m);
}

// Diagonalise F in the orthogonal basis: C = X eig(X^T F X).
int diagonalise(pdg_context *ctx, ScfState &st, const double *F) {
    const int m = st.m;
    PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, F, m, st.X, m, 0.0, st.T1, m));
    PDG_CHECK(gemm(ctx, CUBLAS_OP_T, CUBLAS_OP_N, m, m, m, 1.0, st.X, m, st.T1, m, 0.0, st.T2, m));
    PDG_CHECK(syevd(ctx, st, st.T2, st.eps));
    return gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, st.X, m, st.T2, m, 0.0, st.C, m);
}

// ---- density by canonical purification (Palser and Manolopoulos, Phys. Rev. B 58, 12704 (1998)) --
// In the orthogonal basis the closed-shell density is 2 x the projector on the nocc lowest
// eigenvectors of F' = X^T F X.  Starting from P0 = (lambda/m)(mu I - F') + (nocc/m) I, with the
// spectrum bounded by Gershgorin discs, the iteration
//   c = tr(P^2 - P^3) / tr(P - P^2),
//   P <- ((1+c) P^2 - P^3) / c               (c >= 1/2)
//   P <- ((1-2c) P + (1+c) P^2 - P^3) / (1-c) (c <  1/2)
// keeps the trace at nocc and converges to that projector; it needs only GEMMs, where a dense
// eigensolver of this size is bound by its serial tridiagonalisation.

// Gershgorin discs, one warp per row: rows[i] = F_ii - sum_j |F_ij|, rows[m + i] = F_ii + sum_j |F_ij|
// (j != i), rows[2m + i] = F_ii.
__global__ void gershgorin_kernel(int m, const double *__restrict__ F, double *__restrict__ rows) {
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (i >= m) return;
    double r = 0.0;
    for (int j = lane; j < m; j += 32)
        if (j != i) r += fabs(F[(long long)i * m + j]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
    if (lane == 0) {
        const double d = F[(long long)i * m + i];
        rows[i] = d - r;
        rows[m + i] = d + r;
        rows[2 * m + i] = d;
    }
}

// P0 = (lambda/m)(mu I - F') + (nocc/m) I from the spectrum bounds (every block reduces the
// per-row Gershgorin values itself: 3 m reads).
__global__ void purify_init_kernel(int m, const double *__restrict__ F, const double *__restrict__ rows, int nocc,
                                   double *__restrict__ P) {
    __shared__ double sl[256], sh[256], st[256];
    double lo = 1e300, hi = -1e300, tr = 0.0;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        lo = fmin(lo, rows[i]);
        hi = fmax(hi, rows[m + i]);
        tr += rows[2 * m + i];
    }
    sl[threadIdx.x] = lo; sh[threadIdx.x] = hi; st[threadIdx.x] = tr;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            sl[threadIdx.x] = fmin(sl[threadIdx.x], sl[threadIdx.x + o]);
            sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
            st[threadIdx.x] += st[threadIdx.x + o];
        }
        __syncthreads();
    }
    const double emin = sl[0], emax = sh[0];
    const double mu = st[0] / m;
    const double lam = fmin(nocc / fmax(emax - mu, 1e-300), (m - nocc) / fmax(mu - emin, 1e-300));
    const long long n = (long long)m * m;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)blockDim.x * gridDim.x) {
        const int i = (int)(k % m), j = (int)(k / m);
        P[k] = -(lam / m) * F[k] + (i == j ? (lam / m) * mu + (double)nocc / m : 0.0);
    }
}

// One purification step P' = f(P, P2, P3) into a separate array; every block forms the two traces
// t0 = tr(P - P2), t1 = tr(P2 - P3) from the diagonals itself (O(m)), and block 0 stores them for
// the convergence check.
__global__ void purify_step_kernel(int m, const double *__restrict__ P, const double *__restrict__ P2,
                                   const double *__restrict__ P3, double *__restrict__ Pn, double *__restrict__ t) {
    __shared__ double a[256], b[256];
    double x = 0.0, y = 0.0;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const long long d = (long long)i * m + i;
        x += P[d] - P2[d];
        y += P2[d] - P3[d];
    }
    a[threadIdx.x] = x; b[threadIdx.x] = y;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) { a[threadIdx.x] += a[threadIdx.x + o]; b[threadIdx.x] += b[threadIdx.x + o]; }
        __syncthreads();
    }
    const double t0 = a[0], t1 = b[0];
    if (blockIdx.x == 0 && threadIdx.x == 0) { t[0] = t0; t[1] = t1; }
    const long long n = (long long)m * m;
    const bool idem = !(fabs(t0) > 1e-300);  // already idempotent: copy
    const double c = idem ? 0.0 : t1 / t0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)blockDim.x * gridDim.x) {
        if (idem) Pn[k] = P[k];
        else if (c >= 0.5) Pn[k] = ((1.0 + c) * P2[k] - P3[k]) / c;
        else Pn[k] = ((1.0 - 2.0 * c) * P[k] + (1.0 + c) * P2[k] - P3[k]) / (1.0 - c);
    }
}

// Closed-shell density P = 2 X proj X^T of F by purification (falls back to the eigensolver when
// the iteration has not reached idempotency in 120 steps).
int purify_density(pdg_context *ctx, ScfState &st, const double *F, int nocc, double *P) {
    const int m = st.m;
    const size_t mm = (size_t)m * m * sizeof(double);
    double *Q = (double *)pdg_pool(ctx, "scf.pur.P", mm), *Q2 = (double *)pdg_pool(ctx, "scf.pur.P2", mm),
           *Q3 = (double *)pdg_pool(ctx, "scf.pur.P3", mm), *Qn = (double *)pdg_pool(ctx, "scf.pur.Pn", mm),
           *sc = (double *)pdg_pool(ctx, "scf.pur.s", 8 * sizeof(double)),
           *rows = (double *)pdg_pool(ctx, "scf.pur.rows", 3 * (size_t)m * sizeof(double));
    if (!Q || !Q2 || !Q3 || !Qn || !sc || !rows) { pdg_set_error("purification allocation failed"); return PDG_ERR_ALLOC; }
    PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, F, m, st.X, m, 0.0, st.T1, m));
    PDG_CHECK(gemm(ctx, CUBLAS_OP_T, CUBLAS_OP_N, m, m, m, 1.0, st.X, m, st.T1, m, 0.0, st.T2, m));
    { gershgorin_kernel<<<(m + 7) / 8, 256, 0, ctx->stream>>>(m, st.T2, rows); pdg_count_launch(); }
    const long long n = (long long)m * m;
    // few blocks: each re-reads the diagonals (or the Gershgorin rows) for its own reduction
    const int grid = (int)std::min<long long>(32, (n + 255) / 256);
    { purify_init_kernel<<<grid, 256, 0, ctx->stream>>>(m, st.T2, rows, nocc, Q); pdg_count_launch(); }
    bool done = false;
    for (int it = 0; it < 120 && !done; ++it) {
        PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, Q, m, Q, m, 0.0, Q2, m));
        PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, Q2, m, Q, m, 0.0, Q3, m));
        { purify_step_kernel<<<grid, 256, 0, ctx->stream>>>(m, Q, Q2, Q3, Qn, sc + 3); pdg_count_launch(); }
        std::swap(Q, Qn);
        if (it % 8 == 7) {  // idempotency check every 8 steps (one host read)
            double t[2];
            PDG_CUDA(cudaMemcpyAsync(t, sc + 3, 2 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
            PDG_CUDA(cudaStreamSynchronize(ctx->stream));
            done = std::fabs(t[0]) < 1e-12;
        }
    }
    if (!done) {  // slow (near-degenerate frontier): the eigensolver
        PDG_CHECK(diagonalise(ctx, st, F));
        return make_density(ctx, st, nocc, P);
    }
    // P = 2 X Q X^T
    PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, st.X, m, Q, m, 0.0, st.T1, m));
    return gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_T, m, m, m, 2.0, st.T1, m, st.X, m, 0.0, P, m);
}

// F = H + F2(P) (+ V_xc); returns the exchange-correlation energy and density integral, and
// launches tr(P H) and tr(P F2) into red[0], red[1] (read by the caller with its next copy).
int build_fock(pdg_context *ctx, ScfState &st, double cx, bool doJ, double *Exc, double *rho, double *red) {
    const int m = st.m;
    // Cartesian scaled density D' = N C^T P C N
    PDG_CHECK(pdg_out_to_cart(ctx, st.P, ctx->d_D));
    pdg_launch_scale_full(ctx, ctx->nbf, ctx->d_D, ctx->dbasis.bf_norm);
    PDG_CHECK(pdg_fock2_scf(ctx, cx, doJ, ctx->d_F));  // Cartesian normalised F2 in d_F (uses d_J, d_K)
    *Exc = 0.0;
    *rho = 0.0;
    if (pdg_dft_active(ctx)) PDG_CHECK(pdg_dft_fock_device(ctx, ctx->d_F, Exc, rho));
    PDG_CHECK(pdg_cart_to_out(ctx, ctx->d_F, st.F2));
    { add2_kernel<<<296, 256, 0, ctx->stream>>>((long long)m * m, st.H, st.F2, st.F); pdg_count_launch(); }
    DotBatch d;
    d.add(st.P, st.H);
    d.add(st.P, st.F2);
    PDG_CHECK(dots_launch(ctx, (long long)m * m, d, red));
    PDG_CUDA(cudaGetLastError());
    return PDG_OK;
}

}  // namespace

extern "C" int pdg_scf_run(pdg_context *ctx, const pdg_scf_options *opt, double *density, pdg_scf_result *res) {
    if (!ctx || !opt || !res) { pdg_set_error("pdg_scf_run: invalid argument"); return PDG_ERR_ARG; }
    if (ctx->nbf == 0 || !ctx->have_geometry) { pdg_set_error("pdg_scf_run: basis and geometry required"); return PDG_ERR_STATE; }
    if (opt->use_guess && !density) { pdg_set_error("pdg_scf_run: use_guess without density"); return PDG_ERR_ARG; }
    if (opt->maximum_history < 0 || opt->maximum_history > PDG_MAX_DIIS) {
        pdg_set_error("pdg_scf_run: maximum_history %d outside 0..%d", opt->maximum_history, PDG_MAX_DIIS);
        return PDG_ERR_ARG;
    }
    if (opt->use_guess) {
        // a non-finite guess is refused before any device work (it would only yield NaN)
        const size_t np = (size_t)ctx->nbf_out * (ctx->nbf_out + 1) / 2;
        for (size_t k = 0; k < np; ++k)
            if (!std::isfinite(density[k])) { pdg_set_error("pdg_scf_run: non-finite guess density"); return PDG_ERR_NAN; }
    }
    cudaSetDevice(ctx->device);
    *res = pdg_scf_result{};
    const int m = ctx->nbf_out;
    double nel = -opt->total_charge;
    for (double z : ctx->Z) nel += z;
    const int nocc = (int)std::lround(nel / 2.0);
    if (ctx->occ.empty() && (std::fabs(nel - 2.0 * nocc) > 1e-8 || nocc <= 0 || nocc > m)) {
        pdg_set_error("pdg_scf_run: %g electrons is not a closed shell in %d functions", nel, m);
        return PDG_ERR_ARG;
    }
    const double cx = pdg_dft_active(ctx) ? pdg_dft_exchange_scaling(ctx) : 1.0;
    const bool doJ = true;
    PDG_CHECK(pdg_ensure_pairs(ctx));
    PDG_CHECK(pdg_compute_one_electron(ctx));
    ctx->inc_count = -1;  // first build of this SCF is a full one
    ScfState st;
    st.m = m;
    const size_t mm = (size_t)m * m * sizeof(double);
    double **bufs[] = {&st.S, &st.H, &st.X, &st.P, &st.Pold, &st.F, &st.F2, &st.C, &st.T1, &st.T2};
    const char *names[] = {"scf.S", "scf.H", "scf.X", "scf.P", "scf.Pold", "scf.F", "scf.F2", "scf.C", "scf.T1", "scf.T2"};
    for (int k = 0; k < 10; ++k)
        if (!(*bufs[k] = (double *)pdg_pool(ctx, names[k], mm))) { pdg_set_error("SCF allocation failed"); return PDG_ERR_ALLOC; }
    if (!(st.eps = (double *)pdg_pool(ctx, "scf.eps", m * sizeof(double)))) { pdg_set_error("SCF allocation failed"); return PDG_ERR_ALLOC; }
    PDG_CHECK(pdg_cart_to_out(ctx, ctx->d_S, st.S));
    PDG_CHECK(pdg_cart_to_out(ctx, ctx->d_H, st.H));
    const double Enuc = pdg_nuclear_energy(ctx, nullptr);
    // X = S^-1/2 (symmetric)
    PDG_CUDA(cudaMemcpyAsync(st.T1, st.S, mm, cudaMemcpyDeviceToDevice, ctx->stream));
    PDG_CHECK(syevd(ctx, st, st.T1, st.eps));
    std::vector<double> sev(m);
    PDG_CUDA(cudaMemcpyAsync(sev.data(), st.eps, m * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    if (sev[0] <= 1e-10) {
        pdg_set_error("pdg_scf_run: overlap matrix is singular (smallest eigenvalue %g)", sev[0]);
        return PDG_ERR_UNSUPPORTED;
    }
    PDG_CUDA(cudaMemcpyAsync(st.T2, st.T1, mm, cudaMemcpyDeviceToDevice, ctx->stream));
    { scale_cols_kernel<<<rgrid(m), 256, 0, ctx->stream>>>(m, st.T2, st.eps, -0.5, 0.0); pdg_count_launch(); }
    PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_T, m, m, m, 1.0, st.T2, m, st.T1, m, 0.0, st.X, m));
    // initial density
    if (opt->use_guess) {
        const size_t np = (size_t)m * (m + 1) / 2;
        double *dpk = (double *)pdg_pool(ctx, "packed.tmp", np * sizeof(double));
        if (!dpk) { pdg_set_error("SCF allocation failed"); return PDG_ERR_ALLOC; }
        PDG_CUDA(cudaMemcpyAsync(dpk, density, np * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        pdg_launch_unpack(ctx, m, dpk, nullptr, st.P);
        PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    bool good_start = opt->use_guess != 0;  // a previous density or atomic densities: DIIS at once
    if (!opt->use_guess) {
        bool have = false;
        if (ctx->guess_sad && ctx->occ.empty()) {
            std::vector<double> Pg;
            if (pdg_sad_density(ctx, Pg) == PDG_OK && Pg.size() == (size_t)m * m) {
                PDG_CUDA(cudaMemcpyAsync(st.P, Pg.data(), mm, cudaMemcpyHostToDevice, ctx->stream));
                PDG_CUDA(cudaStreamSynchronize(ctx->stream));
                have = true;
                good_start = true;
            }
        }
        if (!have) {
            PDG_CHECK(diagonalise(ctx, st, st.H));
            PDG_CHECK(make_density(ctx, st, nocc, st.P));
        }
    }
    const int maxh = opt->maximum_history > 0 ? opt->maximum_history : 10;
    std::vector<std::vector<double>> B;  // DIIS overlaps (host)
    int hist_n = 0, hist_head = 0;
    for (int k = 0; k < maxh; ++k) {
        double *a = (double *)pdg_pool(ctx, ("scf.diisF." + std::to_string(k)).c_str(), mm);
        double *b = (double *)pdg_pool(ctx, ("scf.diisE." + std::to_string(k)).c_str(), mm);
        if (!a || !b) { pdg_set_error("DIIS allocation failed"); return PDG_ERR_ALLOC; }
        st.Fh.push_back(a);
        st.Eh.push_back(b);
    }
    std::vector<double> Bm(maxh * maxh, 0.0);
    double E1 = 0, E2 = 0, Exc = 0, rho = 0, Etot = 0, Eold = 0, rms = 0;
    int it = 0;
    bool converged = false;
    // reduction slots: 0..16 dot batches, RMS_SLOT the density change
    constexpr int RMS_SLOT = 20;
    double *red = (double *)pdg_pool(ctx, "scf.red", 24 * sizeof(double));
    if (!red) { pdg_set_error("SCF allocation failed"); return PDG_ERR_ALLOC; }
    double hv[24];
    // Fock and energy of the initial density
    PDG_CHECK(build_fock(ctx, st, cx, doJ, &Exc, &rho, red));
    {
        PDG_CHECK(fetch(ctx, red, 2, hv));
        E1 = hv[0];
        const double pvxc = pdg_dft_active(ctx) ? pdg_dft_last_vxc_trace(ctx) : 0.0;
        E2 = 0.5 * (hv[1] - pvxc);
        Etot = E1 + E2 + Exc + Enuc;
    }
    const int maxit = opt->maximum_iterations > 0 ? opt->maximum_iterations : 100;
    const bool trace = std::getenv("PDG_SCF_TRACE") != nullptr;
    std::vector<int> idx;
    // Optimal damping (ODA) until the DIIS error falls below the onset, then DIIS, as the reference's
    // converger does with its defaults (DIISSCFConverger.py:448-537: diisOnset 0.2, rcaOnset 0.8,
    // minimumMu 0.01).
    // From a core-Hamiltonian start the reference's onsets are used; from atomic densities or a
    // previous density DIIS is switched on at once (ODA only for a very large commutator).
    const double diis_onset = good_start ? 2.0 : 0.2, rca_onset = good_start ? 4.0 : 0.8, minimum_mu = 0.01;
    bool diis_on = false;
    double *Poda = (double *)pdg_pool(ctx, "scf.Poda", mm), *Foda = (double *)pdg_pool(ctx, "scf.Foda", mm);
    if (!Poda || !Foda) { pdg_set_error("ODA allocation failed"); return PDG_ERR_ALLOC; }
    double eOda = Etot;
    double best_err = 1e300;
    int best_it = 0, force_oda = 0;
    for (it = 1; it <= maxit; ++it) {
        // DIIS error e = X^T (F P S - S P F) X
        double *Fk = st.Fh[hist_head], *Ek = st.Eh[hist_head];
        PDG_CUDA(cudaMemcpyAsync(Fk, st.F, mm, cudaMemcpyDeviceToDevice, ctx->stream));
        PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, st.F, m, st.P, m, 0.0, st.T1, m));
        PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, st.T1, m, st.S, m, 0.0, st.T2, m));
        { antisym_kernel<<<rgrid(m), 256, 0, ctx->stream>>>(m, st.T2, st.T1); pdg_count_launch(); }
        PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, st.T1, m, st.X, m, 0.0, st.T2, m));
        PDG_CHECK(gemm(ctx, CUBLAS_OP_T, CUBLAS_OP_N, m, m, m, 1.0, st.X, m, st.T2, m, 0.0, Ek, m));
        const int slot = hist_head;
        hist_head = (hist_head + 1) % maxh;
        if (hist_n < maxh) ++hist_n;
        // the new row of the DIIS matrix and the largest error element, one host read
        DotBatch db;
        int cols[PDG_MAX_DIIS];
        for (int j = 0; j < maxh; ++j) {
            if (j >= hist_n && j != slot) continue;
            cols[db.k] = j;
            db.add(Ek, st.Eh[j]);
        }
        db.amax = Ek;
        PDG_CHECK(dots_launch(ctx, (long long)m * m, db, red));
        PDG_CHECK(fetch(ctx, red, db.k + 1, hv));
        for (int r = 0; r < db.k; ++r) Bm[slot * maxh + cols[r]] = Bm[cols[r] * maxh + slot] = hv[r];
        const double diis_err = hv[db.k];
        if (it > 1) {
            if (diis_on) diis_on = diis_err < rca_onset;
            else if (it > (good_start ? 1 : 2)) diis_on = diis_err < diis_onset;
        }
        // DIIS that has not lowered its error for 8 cycles (occupations sloshing in a small-gap
        // molecule) drops its history and hands over to optimal damping for a few cycles; the
        // first of them only records a consistent (density, Fock) pair for the damping model.
        bool skip_oda = false;
        if (diis_err < 0.95 * best_err) { best_err = diis_err; best_it = it; }
        if (diis_on && it - best_it >= 8) {
            hist_n = 0;
            force_oda = 4;
            skip_oda = true;
            best_err = diis_err;
            best_it = it;
        }
        if (force_oda > 0) { diis_on = false; --force_oda; }
        idx.clear();
        if (it > 1 && !diis_on && !skip_oda) {
            // ODA: cubic model of the energy between the saved (density, Fock) and the current one,
            // E(mu) = A mu^3 + B mu^2 + C mu + D with the end values and end slopes (ODAIterate).
            DotBatch od;
            od.add(st.P, st.F);
            od.add(Poda, st.F);
            od.add(st.P, Foda);
            od.add(Poda, Foda);
            PDG_CHECK(dots_launch(ctx, (long long)m * m, od, red));
            PDG_CHECK(fetch(ctx, red, 4, hv));
            const double tdf = hv[0], thf = hv[1], tdfh = hv[2], thfh = hv[3];
            const double D0 = eOda, C0 = tdfh - thfh;
            const double A0 = (tdf - thf) + C0 + 2.0 * (D0 - Etot);
            const double B0 = Etot - A0 - C0 - D0;
            double fmin = Etot, mu = 1.0;
            if (eOda < Etot) { fmin = eOda; mu = 0.0; }
            if (A0 == 0.0) {
                if (B0 != 0.0) {
                    const double mt = -C0 / (2.0 * B0);
                    if (B0 > 0.0 && mt > 0.0 && mt < 1.0) mu = mt;
                }
            } else {
                const double fac = B0 * B0 - 3.0 * A0 * C0;
                if (fac >= 0.0) {
                    const double roots[2] = {(-B0 + std::sqrt(fac)) / (3.0 * A0), (-B0 - std::sqrt(fac)) / (3.0 * A0)};
                    for (double mt : roots)
                        if (mt > 0.0 && mt < 1.0) {
                            const double fm = ((A0 * mt + B0) * mt + C0) * mt + D0;
                            if (fm < fmin) { fmin = fm; mu = mt; }
                        }
                }
            }
            mu = std::fmax(mu, minimum_mu);
            const double nu = 1.0 - mu;
            if (cublasDscal(ctx->cublas, m * m, &mu, st.P, 1) != CUBLAS_STATUS_SUCCESS ||
                cublasDaxpy(ctx->cublas, m * m, &nu, Poda, 1, st.P, 1) != CUBLAS_STATUS_SUCCESS ||
                cublasDscal(ctx->cublas, m * m, &mu, st.F, 1) != CUBLAS_STATUS_SUCCESS ||
                cublasDaxpy(ctx->cublas, m * m, &nu, Foda, 1, st.F, 1) != CUBLAS_STATUS_SUCCESS) {
                pdg_set_error("cuBLAS failed (ODA)");
                return PDG_ERR_CUDA;
            }
            Etot = ((A0 * mu + B0) * mu + C0) * mu + D0;
        }
        std::vector<double> coef;
        if (diis_on) {
        // solve, dropping the oldest entries while ill-conditioned
        for (int j = 0; j < hist_n; ++j) idx.push_back((hist_head - hist_n + j + maxh) % maxh);  // oldest first
        while (true) {
            const int k = (int)idx.size();
            if (k == 1) { coef = {1.0}; break; }
            std::vector<double> A((k + 1) * (k + 1), 0.0), b(k + 1, 0.0);
            double scale = 0.0;
            for (int r = 0; r < k; ++r) scale = std::fmax(scale, Bm[idx[r] * maxh + idx[r]]);
            if (scale <= 0.0) scale = 1.0;
            for (int r = 0; r < k; ++r) {
                for (int c = 0; c < k; ++c) A[r * (k + 1) + c] = Bm[idx[r] * maxh + idx[c]] / scale;
                A[r * (k + 1) + k] = -1.0;
                A[k * (k + 1) + r] = -1.0;
            }
            b[k] = -1.0;
            if (solve_small(k + 1, A, b)) { coef.assign(b.begin(), b.begin() + k); break; }
            idx.erase(idx.begin());
        }
        if (idx.size() > 1) {
            PDG_CUDA(cudaMemsetAsync(st.F, 0, mm, ctx->stream));
            for (size_t r = 0; r < idx.size(); ++r) {
                const double c = coef[r];
                if (cublasDaxpy(ctx->cublas, m * m, &c, st.Fh[idx[r]], 1, st.F, 1) != CUBLAS_STATUS_SUCCESS) {
                    pdg_set_error("cublasDaxpy failed"); return PDG_ERR_CUDA;
                }
            }
        }
        }  // diis_on
        // save the (possibly damped) density and Fock matrix and their energy for the next ODA step
        PDG_CUDA(cudaMemcpyAsync(Poda, st.P, mm, cudaMemcpyDeviceToDevice, ctx->stream));
        PDG_CUDA(cudaMemcpyAsync(Foda, st.F, mm, cudaMemcpyDeviceToDevice, ctx->stream));
        eOda = Etot;
        // new orbitals and density
        {
            ProfScope prof_diag(ctx, "scf_diag");
            PDG_CUDA(cudaMemcpyAsync(st.Pold, st.P, mm, cudaMemcpyDeviceToDevice, ctx->stream));
            if (ctx->occ.empty()) {
                PDG_CHECK(purify_density(ctx, st, st.F, nocc, st.P));
            } else {
                PDG_CHECK(diagonalise(ctx, st, st.F));
                PDG_CHECK(make_density(ctx, st, nocc, st.P));
            }
        }
        // density change (read with the energy traces after the Fock build)
        PDG_CUDA(cudaMemsetAsync(red + RMS_SLOT, 0, sizeof(double), ctx->stream));
        { diff_sq_kernel<<<296, 256, 0, ctx->stream>>>((long long)m * m, st.P, st.Pold, red + RMS_SLOT); pdg_count_launch(); }
        // Fock and energy of the new density
        Eold = Etot;
        PDG_CHECK(build_fock(ctx, st, cx, doJ, &Exc, &rho, red));
        PDG_CHECK(fetch(ctx, red, RMS_SLOT + 1, hv));
        rms = std::sqrt(hv[RMS_SLOT] / ((double)m * m));
        E1 = hv[0];
        const double pvxc = pdg_dft_active(ctx) ? pdg_dft_last_vxc_trace(ctx) : 0.0;
        E2 = 0.5 * (hv[1] - pvxc);
        Etot = E1 + E2 + Exc + Enuc;
        if (!std::isfinite(Etot)) { pdg_set_error("pdg_scf_run: non-finite energy"); return PDG_ERR_NAN; }
        if (trace)
            fprintf(stderr, "scf %3d E %.12f dE %+.3e rms %.3e err %.3e %s %zu\n", it, Etot, Etot - Eold, rms, diis_err,
                    diis_on ? "diis" : "oda", idx.size());
        if (rms <= opt->density_tolerance && (Etot - Eold) <= opt->energy_tolerance) { converged = true; break; }
    }
    res->energy_total = Etot;
    res->energy_one = E1;
    res->energy_two = E2;
    res->energy_xc = Exc;
    res->energy_nuclear = Enuc;
    res->rho_integral = rho;
    res->rms_density = rms;
    res->iterations = converged ? it : maxit;
    res->converged = converged ? 1 : 0;
    res->quartets = ctx->last_quartets;
    // keep P resident with what the weighted density needs (copies in pool buffers of their own: the
    // SCF buffers are reused): the orbitals of the eigensolver path, or, on the purification path,
    // the Fock matrix (saved in Foda) whose occupied projector P is, since there W = 1/2 P F P
    ScfResident &r = resident(ctx);
    r.unrestricted = false;
    r.orbitals = !ctx->occ.empty();
    r.P = (double *)pdg_pool(ctx, "scf.res.P", mm);
    if (r.orbitals) {
        r.C = (double *)pdg_pool(ctx, "scf.res.C", mm);
        r.eps = (double *)pdg_pool(ctx, "scf.res.eps", m * sizeof(double));
    } else {
        r.F = (double *)pdg_pool(ctx, "scf.res.F", mm);
    }
    if (!r.P || (r.orbitals ? (!r.C || !r.eps) : !r.F)) { r.valid = false; pdg_set_error("SCF allocation failed"); return PDG_ERR_ALLOC; }
    PDG_CUDA(cudaMemcpyAsync(r.P, st.P, mm, cudaMemcpyDeviceToDevice, ctx->stream));
    if (r.orbitals) {
        PDG_CUDA(cudaMemcpyAsync(r.C, st.C, mm, cudaMemcpyDeviceToDevice, ctx->stream));
        PDG_CUDA(cudaMemcpyAsync(r.eps, st.eps, m * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    } else {
        PDG_CUDA(cudaMemcpyAsync(r.F, Foda, mm, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    r.m = m;
    r.nocc = nocc;
    r.cx = cx;
    r.valid = true;
    if (density) PDG_CHECK(pdg_store_packed(ctx, r.P, density));
    if (!converged) { pdg_set_error("Too many iterations."); return PDG_ERR_NOCONV; }
    return PDG_OK;
}

// ---- unrestricted Hartree-Fock -------------------------------------------------------------------
// The reference's spin-unrestricted path (two densities and Fock matrices, FockConstruction.c:258-264;
// per-spin DIIS frames and the larger of the two RMS density changes, DIISSCFConverger.py:77-108,
// 438-446) for Hartree-Fock: F_s = H + J(P_a + P_b) - cx K(P_s).  J is linear in the density, so
// one J+K pass per spin density gives both K_s and, summed, J.  Densities by purification of each
// spin's Fock matrix (occupation one), DIIS on the joint error (B_ij = e_a,i.e_a,j + e_b,i.e_b,j)
// from the atomic-density (or core) guess; full density-screened builds every cycle.
namespace {

struct UhfBuffers {
    double *Pa, *Pb, *Pa_old, *Pb_old, *Fa, *Fb, *F2a, *F2b, *Fa_used, *Fb_used;
    double *Db, *Kb, *dmaxb, *Fc;
};

int uhf_fock(pdg_context *ctx, ScfState &st, UhfBuffers &u, double cx, double *red) {
    const int n = ctx->nbf, m = st.m;
    const size_t nn = (size_t)n * n * sizeof(double);
    PDG_CHECK(pdg_out_to_cart(ctx, u.Pa, ctx->d_D));
    pdg_launch_scale_full(ctx, n, ctx->d_D, ctx->dbasis.bf_norm);
    PDG_CHECK(pdg_out_to_cart(ctx, u.Pb, u.Db));
    pdg_launch_scale_full(ctx, n, u.Db, ctx->dbasis.bf_norm);
    PDG_CUDA(cudaMemsetAsync(ctx->d_J, 0, nn, ctx->stream));
    PDG_CUDA(cudaMemsetAsync(ctx->d_K, 0, nn, ctx->stream));
    PDG_CUDA(cudaMemsetAsync(u.Kb, 0, nn, ctx->stream));
    const bool doK = cx != 0.0;
    PDG_CHECK(pdg_shell_pair_dmax(ctx, ctx->d_D, ctx->d_dmax));
    PDG_CHECK(pdg_eri_jk_screened(ctx, ctx->d_D, ctx->d_J, ctx->d_K, true, doK, ctx->d_dmax, pdg_fock_dcut(ctx)));
    PDG_CHECK(pdg_shell_pair_dmax(ctx, u.Db, u.dmaxb));
    PDG_CHECK(pdg_eri_jk_screened(ctx, u.Db, ctx->d_J, u.Kb, true, doK, u.dmaxb, pdg_fock_dcut(ctx)));
    pdg_launch_sym_combine2(ctx, n, ctx->d_J, doK ? ctx->d_K : nullptr, 1.0, -cx, ctx->dbasis.bf_norm, u.Fc);
    PDG_CHECK(pdg_cart_to_out(ctx, u.Fc, u.F2a));
    pdg_launch_sym_combine2(ctx, n, ctx->d_J, doK ? u.Kb : nullptr, 1.0, -cx, ctx->dbasis.bf_norm, u.Fc);
    PDG_CHECK(pdg_cart_to_out(ctx, u.Fc, u.F2b));
    { add2_kernel<<<296, 256, 0, ctx->stream>>>((long long)m * m, st.H, u.F2a, u.Fa); pdg_count_launch(); }
    { add2_kernel<<<296, 256, 0, ctx->stream>>>((long long)m * m, st.H, u.F2b, u.Fb); pdg_count_launch(); }
    // E = sum_s tr(P_s H) + 1/2 sum_s tr(P_s F2_s)
    DotBatch d;
    d.add(u.Pa, st.H);
    d.add(u.Pb, st.H);
    d.add(u.Pa, u.F2a);
    d.add(u.Pb, u.F2b);
    PDG_CHECK(dots_launch(ctx, (long long)m * m, d, red));
    PDG_CUDA(cudaGetLastError());
    return PDG_OK;
}

// P_s = projector on the n_s lowest orbitals of F_s (occupation one), or zero.
int uhf_density(pdg_context *ctx, ScfState &st, const double *F, int n_s, double *P) {
    const int m = st.m;
    if (n_s == 0) {
        PDG_CUDA(cudaMemsetAsync(P, 0, (size_t)m * m * sizeof(double), ctx->stream));
        return PDG_OK;
    }
    PDG_CHECK(purify_density(ctx, st, F, n_s, P));  // 2 x projector
    const double half = 0.5;
    if (cublasDscal(ctx->cublas, m * m, &half, P, 1) != CUBLAS_STATUS_SUCCESS) { pdg_set_error("cublasDscal failed"); return PDG_ERR_CUDA; }
    return PDG_OK;
}

// DIIS error X^T (F P S - S P F) X of one spin into E.
int uhf_error(pdg_context *ctx, ScfState &st, const double *F, const double *P, double *E) {
    const int m = st.m;
    PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, F, m, P, m, 0.0, st.T1, m));
    PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, st.T1, m, st.S, m, 0.0, st.T2, m));
    { antisym_kernel<<<rgrid(m), 256, 0, ctx->stream>>>(m, st.T2, st.T1); pdg_count_launch(); }
    PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, st.T1, m, st.X, m, 0.0, st.T2, m));
    return gemm(ctx, CUBLAS_OP_T, CUBLAS_OP_N, m, m, m, 1.0, st.X, m, st.T2, m, 0.0, E, m);
}

}  // namespace

extern "C" int pdg_uscf_run(pdg_context *ctx, const pdg_scf_options *opt, int n_alpha, int n_beta, double *density_alpha,
                            double *density_beta, pdg_scf_result *res) {
    if (!ctx || !opt || !res || n_alpha < 0 || n_beta < 0) { pdg_set_error("pdg_uscf_run: invalid argument"); return PDG_ERR_ARG; }
    if (ctx->nbf == 0 || !ctx->have_geometry) { pdg_set_error("pdg_uscf_run: basis and geometry required"); return PDG_ERR_STATE; }
    if (pdg_dft_active(ctx)) { pdg_set_error("pdg_uscf_run: unrestricted Kohn-Sham is not supported (Hartree-Fock only)"); return PDG_ERR_UNSUPPORTED; }
    if (opt->use_guess && (!density_alpha || !density_beta)) { pdg_set_error("pdg_uscf_run: use_guess without densities"); return PDG_ERR_ARG; }
    if (opt->maximum_history < 0 || opt->maximum_history > PDG_MAX_DIIS) {
        pdg_set_error("pdg_uscf_run: maximum_history %d outside 0..%d", opt->maximum_history, PDG_MAX_DIIS);
        return PDG_ERR_ARG;
    }
    if (opt->use_guess) {
        const size_t np = (size_t)ctx->nbf_out * (ctx->nbf_out + 1) / 2;
        for (size_t k = 0; k < np; ++k)
            if (!std::isfinite(density_alpha[k]) || !std::isfinite(density_beta[k])) {
                pdg_set_error("pdg_uscf_run: non-finite guess density");
                return PDG_ERR_NAN;
            }
    }
    cudaSetDevice(ctx->device);
    *res = pdg_scf_result{};
    const int m = ctx->nbf_out;
    double nel = -opt->total_charge;
    for (double z : ctx->Z) nel += z;
    if (std::fabs(nel - (n_alpha + n_beta)) > 1e-8 || n_alpha > m || n_beta > m || n_alpha + n_beta == 0) {
        pdg_set_error("pdg_uscf_run: %d + %d electrons for a molecule with %g", n_alpha, n_beta, nel);
        return PDG_ERR_ARG;
    }
    const double cx = 1.0;
    PDG_CHECK(pdg_ensure_pairs(ctx));
    PDG_CHECK(pdg_compute_one_electron(ctx));
    ctx->inc_count = -1;
    ScfState st;
    st.m = m;
    const size_t mm = (size_t)m * m * sizeof(double), nn = (size_t)ctx->nbf * ctx->nbf * sizeof(double);
    double **bufs[] = {&st.S, &st.H, &st.X, &st.P, &st.Pold, &st.F, &st.F2, &st.C, &st.T1, &st.T2};
    const char *names[] = {"scf.S", "scf.H", "scf.X", "scf.P", "scf.Pold", "scf.F", "scf.F2", "scf.C", "scf.T1", "scf.T2"};
    for (int k = 0; k < 10; ++k)
        if (!(*bufs[k] = (double *)pdg_pool(ctx, names[k], mm))) { pdg_set_error("SCF allocation failed"); return PDG_ERR_ALLOC; }
    if (!(st.eps = (double *)pdg_pool(ctx, "scf.eps", m * sizeof(double)))) { pdg_set_error("SCF allocation failed"); return PDG_ERR_ALLOC; }
    UhfBuffers u;
    double **ub[] = {&u.Pa, &u.Pb, &u.Pa_old, &u.Pb_old, &u.Fa, &u.Fb, &u.F2a, &u.F2b, &u.Fa_used, &u.Fb_used};
    const char *un[] = {"uscf.Pa", "uscf.Pb", "uscf.Pa0", "uscf.Pb0", "uscf.Fa", "uscf.Fb", "uscf.F2a", "uscf.F2b", "uscf.Fau", "uscf.Fbu"};
    for (int k = 0; k < 10; ++k)
        if (!(*ub[k] = (double *)pdg_pool(ctx, un[k], mm))) { pdg_set_error("SCF allocation failed"); return PDG_ERR_ALLOC; }
    const int ns = (int)ctx->shells.size();
    u.Db = (double *)pdg_pool(ctx, "uscf.Db", nn);
    u.Kb = (double *)pdg_pool(ctx, "uscf.Kb", nn);
    u.Fc = (double *)pdg_pool(ctx, "uscf.Fc", nn);
    u.dmaxb = (double *)pdg_pool(ctx, "uscf.dmaxb", (size_t)ns * ns * sizeof(double));
    if (!u.Db || !u.Kb || !u.Fc || !u.dmaxb) { pdg_set_error("SCF allocation failed"); return PDG_ERR_ALLOC; }
    PDG_CHECK(pdg_cart_to_out(ctx, ctx->d_S, st.S));
    PDG_CHECK(pdg_cart_to_out(ctx, ctx->d_H, st.H));
    const double Enuc = pdg_nuclear_energy(ctx, nullptr);
    // X = S^-1/2
    PDG_CUDA(cudaMemcpyAsync(st.T1, st.S, mm, cudaMemcpyDeviceToDevice, ctx->stream));
    PDG_CHECK(syevd(ctx, st, st.T1, st.eps));
    std::vector<double> sev(m);
    PDG_CUDA(cudaMemcpyAsync(sev.data(), st.eps, m * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    if (sev[0] <= 1e-10) { pdg_set_error("pdg_uscf_run: overlap matrix is singular (smallest eigenvalue %g)", sev[0]); return PDG_ERR_UNSUPPORTED; }
    PDG_CUDA(cudaMemcpyAsync(st.T2, st.T1, mm, cudaMemcpyDeviceToDevice, ctx->stream));
    { scale_cols_kernel<<<rgrid(m), 256, 0, ctx->stream>>>(m, st.T2, st.eps, -0.5, 0.0); pdg_count_launch(); }
    PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_T, m, m, m, 1.0, st.T2, m, st.T1, m, 0.0, st.X, m));
    // initial spin densities: given, atomic densities halved, or the core Hamiltonian's orbitals
    const size_t np = (size_t)m * (m + 1) / 2;
    if (opt->use_guess) {
        double *dpk = (double *)pdg_pool(ctx, "packed.tmp", np * sizeof(double));
        if (!dpk) { pdg_set_error("SCF allocation failed"); return PDG_ERR_ALLOC; }
        PDG_CUDA(cudaMemcpyAsync(dpk, density_alpha, np * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        pdg_launch_unpack(ctx, m, dpk, nullptr, u.Pa);
        PDG_CUDA(cudaMemcpyAsync(dpk, density_beta, np * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        pdg_launch_unpack(ctx, m, dpk, nullptr, u.Pb);
        PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    } else {
        bool have = false;
        if (ctx->guess_sad && ctx->occ.empty()) {
            std::vector<double> Pg;
            if (pdg_sad_density(ctx, Pg) == PDG_OK && Pg.size() == (size_t)m * m) {
                for (double &v : Pg) v *= 0.5;
                PDG_CUDA(cudaMemcpyAsync(u.Pa, Pg.data(), mm, cudaMemcpyHostToDevice, ctx->stream));
                PDG_CUDA(cudaMemcpyAsync(u.Pb, Pg.data(), mm, cudaMemcpyHostToDevice, ctx->stream));
                PDG_CUDA(cudaStreamSynchronize(ctx->stream));
                have = true;
            }
        }
        if (!have) {
            PDG_CHECK(uhf_density(ctx, st, st.H, n_alpha, u.Pa));
            PDG_CHECK(uhf_density(ctx, st, st.H, n_beta, u.Pb));
        }
    }
    const int maxh = opt->maximum_history > 0 ? opt->maximum_history : 10;
    std::vector<double *> Fah, Fbh, Eah, Ebh;
    for (int k = 0; k < maxh; ++k) {
        const std::string s = std::to_string(k);
        double *a = (double *)pdg_pool(ctx, ("uscf.dFa." + s).c_str(), mm), *b = (double *)pdg_pool(ctx, ("uscf.dFb." + s).c_str(), mm);
        double *c = (double *)pdg_pool(ctx, ("uscf.dEa." + s).c_str(), mm), *d = (double *)pdg_pool(ctx, ("uscf.dEb." + s).c_str(), mm);
        if (!a || !b || !c || !d) { pdg_set_error("DIIS allocation failed"); return PDG_ERR_ALLOC; }
        Fah.push_back(a); Fbh.push_back(b); Eah.push_back(c); Ebh.push_back(d);
    }
    double *red = (double *)pdg_pool(ctx, "scf.red", 48 * sizeof(double));
    if (!red) { pdg_set_error("SCF allocation failed"); return PDG_ERR_ALLOC; }
    double hv[48];
    constexpr int RMS_A = 40, RMS_B = 41;
    PDG_CHECK(uhf_fock(ctx, st, u, cx, red));
    PDG_CHECK(fetch(ctx, red, 4, hv));
    double E1 = hv[0] + hv[1], E2 = 0.5 * (hv[2] + hv[3]);
    double Etot = E1 + E2 + Enuc, Eold = Etot, rms = 0.0;
    std::vector<double> Bm(maxh * maxh, 0.0);
    int hist_n = 0, hist_head = 0, it = 0;
    bool converged = false;
    const int maxit = opt->maximum_iterations > 0 ? opt->maximum_iterations : 100;
    for (it = 1; it <= maxit; ++it) {
        // errors of both spins into the history, the new DIIS row and the largest element
        const int slot = hist_head;
        PDG_CUDA(cudaMemcpyAsync(Fah[slot], u.Fa, mm, cudaMemcpyDeviceToDevice, ctx->stream));
        PDG_CUDA(cudaMemcpyAsync(Fbh[slot], u.Fb, mm, cudaMemcpyDeviceToDevice, ctx->stream));
        PDG_CHECK(uhf_error(ctx, st, u.Fa, u.Pa, Eah[slot]));
        PDG_CHECK(uhf_error(ctx, st, u.Fb, u.Pb, Ebh[slot]));
        hist_head = (hist_head + 1) % maxh;
        if (hist_n < maxh) ++hist_n;
        DotBatch da, db;
        int cols[PDG_MAX_DIIS];
        for (int j = 0; j < maxh; ++j) {
            if (j >= hist_n && j != slot) continue;
            cols[da.k] = j;
            da.add(Eah[slot], Eah[j]);
            db.add(Ebh[slot], Ebh[j]);
        }
        da.amax = Eah[slot];
        db.amax = Ebh[slot];
        PDG_CHECK(dots_launch(ctx, (long long)m * m, da, red));
        PDG_CHECK(dots_launch(ctx, (long long)m * m, db, red + 20));
        PDG_CHECK(fetch(ctx, red, 20 + db.k + 1, hv));
        for (int r = 0; r < da.k; ++r) Bm[slot * maxh + cols[r]] = Bm[cols[r] * maxh + slot] = hv[r] + hv[20 + r];
        const double diis_err = std::fmax(hv[da.k], hv[20 + db.k]);
        // DIIS extrapolation of both Fock matrices with the joint coefficients
        std::vector<int> idx;
        for (int j = 0; j < hist_n; ++j) idx.push_back((hist_head - hist_n + j + maxh) % maxh);
        std::vector<double> coef;
        while (idx.size() > 1) {
            const int k = (int)idx.size();
            std::vector<double> A((k + 1) * (k + 1), 0.0), b(k + 1, 0.0);
            double scale = 0.0;
            for (int r = 0; r < k; ++r) scale = std::fmax(scale, Bm[idx[r] * maxh + idx[r]]);
            if (scale <= 0.0) scale = 1.0;
            for (int r = 0; r < k; ++r) {
                for (int c = 0; c < k; ++c) A[r * (k + 1) + c] = Bm[idx[r] * maxh + idx[c]] / scale;
                A[r * (k + 1) + k] = -1.0;
                A[k * (k + 1) + r] = -1.0;
            }
            b[k] = -1.0;
            if (solve_small(k + 1, A, b)) { coef.assign(b.begin(), b.begin() + k); break; }
            idx.erase(idx.begin());
        }
        if (idx.size() > 1) {
            PDG_CUDA(cudaMemsetAsync(u.Fa, 0, mm, ctx->stream));
            PDG_CUDA(cudaMemsetAsync(u.Fb, 0, mm, ctx->stream));
            for (size_t r = 0; r < idx.size(); ++r) {
                const double c = coef[r];
                if (cublasDaxpy(ctx->cublas, m * m, &c, Fah[idx[r]], 1, u.Fa, 1) != CUBLAS_STATUS_SUCCESS ||
                    cublasDaxpy(ctx->cublas, m * m, &c, Fbh[idx[r]], 1, u.Fb, 1) != CUBLAS_STATUS_SUCCESS) {
                    pdg_set_error("cublasDaxpy failed"); return PDG_ERR_CUDA;
                }
            }
        }
        // new spin densities from the (extrapolated) Fock matrices, kept for the weighted density
        {
            ProfScope prof_diag(ctx, "scf_diag");
            PDG_CUDA(cudaMemcpyAsync(u.Fa_used, u.Fa, mm, cudaMemcpyDeviceToDevice, ctx->stream));
            PDG_CUDA(cudaMemcpyAsync(u.Fb_used, u.Fb, mm, cudaMemcpyDeviceToDevice, ctx->stream));
            PDG_CUDA(cudaMemcpyAsync(u.Pa_old, u.Pa, mm, cudaMemcpyDeviceToDevice, ctx->stream));
            PDG_CUDA(cudaMemcpyAsync(u.Pb_old, u.Pb, mm, cudaMemcpyDeviceToDevice, ctx->stream));
            PDG_CHECK(uhf_density(ctx, st, u.Fa_used, n_alpha, u.Pa));
            PDG_CHECK(uhf_density(ctx, st, u.Fb_used, n_beta, u.Pb));
        }
        PDG_CUDA(cudaMemsetAsync(red + RMS_A, 0, 2 * sizeof(double), ctx->stream));
        { diff_sq_kernel<<<296, 256, 0, ctx->stream>>>((long long)m * m, u.Pa, u.Pa_old, red + RMS_A); pdg_count_launch(); }
        { diff_sq_kernel<<<296, 256, 0, ctx->stream>>>((long long)m * m, u.Pb, u.Pb_old, red + RMS_B); pdg_count_launch(); }
        Eold = Etot;
        PDG_CHECK(uhf_fock(ctx, st, u, cx, red));
        PDG_CHECK(fetch(ctx, red, RMS_B + 1, hv));
        rms = std::sqrt(std::fmax(hv[RMS_A], hv[RMS_B]) / ((double)m * m));
        E1 = hv[0] + hv[1];
        E2 = 0.5 * (hv[2] + hv[3]);
        Etot = E1 + E2 + Enuc;
        if (!std::isfinite(Etot)) { pdg_set_error("pdg_uscf_run: non-finite energy"); return PDG_ERR_NAN; }
        if (std::getenv("PDG_SCF_TRACE"))
            fprintf(stderr, "uscf %3d E %.12f dE %+.3e rms %.3e err %.3e %zu\n", it, Etot, Etot - Eold, rms, diis_err, idx.size());
        if (rms <= opt->density_tolerance && (Etot - Eold) <= opt->energy_tolerance) { converged = true; break; }
    }
    // <S^2> = Sz (Sz + 1) + n_beta - tr(Pa S Pb S); with symmetric Pa, Pb, S the trace is the
    // elementwise dot of Pa S with S Pb = (Pb S)^T
    PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, u.Pa, m, st.S, m, 0.0, st.T1, m));
    PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, st.S, m, u.Pb, m, 0.0, st.T2, m));
    {
        DotBatch d;
        d.add(st.T1, st.T2);
        PDG_CHECK(dots_launch(ctx, (long long)m * m, d, red));
        PDG_CHECK(fetch(ctx, red, 1, hv));
    }
    const double sz = 0.5 * (n_alpha - n_beta);
    res->s2 = sz * (sz + 1.0) + n_beta - hv[0];
    res->energy_total = Etot;
    res->energy_one = E1;
    res->energy_two = E2;
    res->energy_nuclear = Enuc;
    res->rms_density = rms;
    res->iterations = converged ? it : maxit;
    res->converged = converged ? 1 : 0;
    res->quartets = ctx->last_quartets;
    ScfResident &r = resident(ctx);
    r.unrestricted = true;
    r.orbitals = false;
    r.P = (double *)pdg_pool(ctx, "scf.res.P", mm);
    r.Pa = (double *)pdg_pool(ctx, "scf.res.Pa", mm);
    r.Pb = (double *)pdg_pool(ctx, "scf.res.Pb", mm);
    r.Fa = (double *)pdg_pool(ctx, "scf.res.Fa", mm);
    r.Fb = (double *)pdg_pool(ctx, "scf.res.Fb", mm);
    if (!r.P || !r.Pa || !r.Pb || !r.Fa || !r.Fb) { r.valid = false; pdg_set_error("SCF allocation failed"); return PDG_ERR_ALLOC; }
    { add2_kernel<<<296, 256, 0, ctx->stream>>>((long long)m * m, u.Pa, u.Pb, r.P); pdg_count_launch(); }
    PDG_CUDA(cudaMemcpyAsync(r.Pa, u.Pa, mm, cudaMemcpyDeviceToDevice, ctx->stream));
    PDG_CUDA(cudaMemcpyAsync(r.Pb, u.Pb, mm, cudaMemcpyDeviceToDevice, ctx->stream));
    PDG_CUDA(cudaMemcpyAsync(r.Fa, u.Fa_used, mm, cudaMemcpyDeviceToDevice, ctx->stream));
    PDG_CUDA(cudaMemcpyAsync(r.Fb, u.Fb_used, mm, cudaMemcpyDeviceToDevice, ctx->stream));
    r.m = m;
    r.nocc = n_alpha;
    r.cx = cx;
    r.valid = true;
    if (density_alpha) PDG_CHECK(pdg_store_packed(ctx, r.Pa, density_alpha));
    if (density_beta) PDG_CHECK(pdg_store_packed(ctx, r.Pb, density_beta));
    if (!converged) { pdg_set_error("Too many iterations."); return PDG_ERR_NOCONV; }
    return PDG_OK;
}

namespace {
__global__ void weighted_coef_kernel(int m, int nocc, const double *C, const double *eps, double *Cw) {
    // Cw[:, i] = C[:, i] * 2 eps_i (column-major)
    const int j = blockIdx.y;
    for (int i = threadIdx.x + blockIdx.x * blockDim.x; i < m; i += blockDim.x * gridDim.x)
        Cw[(long long)j * m + i] = j < nocc ? 2.0 * eps[j] * C[(long long)j * m + i] : 0.0;
}

// Standard-convention weighted density W = sum_occ 2 e_i C_i C_i^T into out (m x m).  Without
// orbitals: P = 2 C_o C_o^T is the occupied projector density of F (C^T F C = e, C^T S C = 1), so
// P F P = 4 C_o e_o C_o^T and W = 1/2 P F P.
int weighted_density(pdg_context *ctx, ScfResident &r, double *tmp, double *out) {
    const int m = r.m;
    if (r.unrestricted) {  // W = sum_s P_s F_s P_s (each P_s the occupation-one projector of F_s)
        PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, r.Fa, m, r.Pa, m, 0.0, tmp, m));
        PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, r.Pa, m, tmp, m, 0.0, out, m));
        PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, r.Fb, m, r.Pb, m, 0.0, tmp, m));
        return gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, r.Pb, m, tmp, m, 1.0, out, m);
    }
    if (!r.orbitals) {
        PDG_CHECK(gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 1.0, r.F, m, r.P, m, 0.0, tmp, m));
        return gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_N, m, m, m, 0.5, r.P, m, tmp, m, 0.0, out, m);
    }
    { weighted_coef_kernel<<<dim3((m + 255) / 256 < 4 ? (m + 255) / 256 : 4, r.nocc), 256, 0, ctx->stream>>>(m, r.nocc, r.C, r.eps, tmp); pdg_count_launch(); }
    return gemm(ctx, CUBLAS_OP_N, CUBLAS_OP_T, m, m, r.nocc, 1.0, tmp, m, r.C, m, 0.0, out, m);
}
}  // namespace

// The last SCF's density (output basis, full m x m, device), or null.
const double *pdg_scf_resident_density(const pdg_context *ctx) {
    ScfResident &r = resident(ctx);
    return r.valid ? r.P : nullptr;
}

void pdg_scf_release(const pdg_context *ctx) {
    std::lock_guard<std::mutex> lock(g_resident_mutex);
    auto it = g_resident.find(ctx);
    if (it == g_resident.end()) return;
    g_resident.erase(it);  // its buffers belong to the context's pool
}

extern "C" int pdg_scf_weighted_density(pdg_context *ctx, double *wd) {
    if (!ctx || !wd) { pdg_set_error("pdg_scf_weighted_density: invalid argument"); return PDG_ERR_ARG; }
    ScfResident &r = resident(ctx);
    if (!r.valid) { pdg_set_error("pdg_scf_weighted_density: no SCF result"); return PDG_ERR_STATE; }
    cudaSetDevice(ctx->device);
    PDG_CHECK(weighted_density(ctx, r, ctx->d_Fout, ctx->d_Dout));
    const double m2 = -2.0;  // reference convention: -2 x standard
    const int m = r.m;
    if (cublasDscal(ctx->cublas, m * m, &m2, ctx->d_Dout, 1) != CUBLAS_STATUS_SUCCESS) { pdg_set_error("cublasDscal failed"); return PDG_ERR_CUDA; }
    return pdg_store_packed(ctx, ctx->d_Dout, wd);
}

extern "C" int pdg_scf_gradients(pdg_context *ctx, double *gradients3) {
    if (!ctx || !gradients3) { pdg_set_error("pdg_scf_gradients: invalid argument"); return PDG_ERR_ARG; }
    ScfResident &r = resident(ctx);
    if (!r.valid) { pdg_set_error("pdg_scf_gradients: no SCF result"); return PDG_ERR_STATE; }
    cudaSetDevice(ctx->device);
    // W' = N C^T W C N
    PDG_CHECK(weighted_density(ctx, r, ctx->d_Fout, ctx->d_Dout));
    PDG_CHECK(pdg_out_to_cart(ctx, ctx->d_Dout, ctx->d_W));
    pdg_launch_scale_full(ctx, ctx->nbf, ctx->d_W, ctx->dbasis.bf_norm);
    PDG_CHECK(pdg_out_to_cart(ctx, r.P, ctx->d_D));
    pdg_launch_scale_full(ctx, ctx->nbf, ctx->d_D, ctx->dbasis.bf_norm);
    if (r.unrestricted) {
        // one-electron terms and Coulomb from the total density; exchange per spin density, whose
        // Gamma -cx/2 sum_s P_s,ac P_s,bd is the restricted form with 2 cx
        const int na = ctx->natom;
        PDG_CUDA(cudaMemsetAsync(ctx->d_grad, 0, 3 * na * sizeof(double), ctx->stream));
        PDG_CHECK(pdg_oneint_grad(ctx, ctx->d_D, ctx->d_W, ctx->d_grad));
        PDG_CHECK(pdg_eri_grad(ctx, ctx->d_D, 0.0, true, ctx->d_grad));
        for (const double *Ps : {r.Pa, r.Pb}) {
            PDG_CHECK(pdg_out_to_cart(ctx, Ps, ctx->d_D));
            pdg_launch_scale_full(ctx, ctx->nbf, ctx->d_D, ctx->dbasis.bf_norm);
            PDG_CHECK(pdg_eri_grad(ctx, ctx->d_D, 2.0 * r.cx, false, ctx->d_grad));
        }
        std::vector<double> h(3 * na);
        PDG_CUDA(cudaMemcpyAsync(h.data(), ctx->d_grad, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        PDG_CUDA(cudaStreamSynchronize(ctx->stream));
        pdg_nuclear_energy(ctx, &h);
        for (int k = 0; k < 3 * na; ++k) gradients3[k] += h[k];
        return PDG_OK;
    }
    std::vector<double> g(3 * ctx->natom, 0.0);
    PDG_CHECK(pdg_gradients_device(ctx, r.cx, true, g));
    if (pdg_dft_active(ctx)) {
        PDG_CUDA(cudaMemsetAsync(ctx->d_grad, 0, 3 * ctx->natom * sizeof(double), ctx->stream));
        PDG_CHECK(pdg_dft_grad_device(ctx, ctx->d_grad));
        std::vector<double> h(3 * ctx->natom);
        PDG_CUDA(cudaMemcpyAsync(h.data(), ctx->d_grad, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        PDG_CUDA(cudaStreamSynchronize(ctx->stream));
        for (size_t k = 0; k < h.size(); ++k) g[k] += h[k];
    }
    for (int k = 0; k < 3 * ctx->natom; ++k) gradients3[k] += g[k];
    return PDG_OK;
}
