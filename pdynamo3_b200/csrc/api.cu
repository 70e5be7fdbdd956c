// C-ABI entry points: context, basis, geometry, one-electron, two-electron Fock and gradients.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <vector>

#include "context.h"

static thread_local char g_err[1024] = "";

void pdg_set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

extern "C" int pdg_version(void) { return 100; }
extern "C" const char *pdg_last_error(void) { return g_err; }

static std::atomic<long long> g_launches{0};
void pdg_count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

extern "C" int pdg_launch_count(long long *count) {
    if (!count) return PDG_ERR_ARG;
    *count = g_launches.load();
    return PDG_OK;
}

void *pdg_pool(pdg_context *ctx, const char *name, size_t bytes) {
    auto &e = ctx->pool[name];
    if (e.first && e.second >= bytes) return e.first;
    cudaFree(e.first);
    e.first = nullptr;
    e.second = 0;
    const size_t want = bytes + bytes / 8 + 256;  // headroom so small growth does not reallocate
    if (cudaMalloc(&e.first, want) != cudaSuccess) {
        e.first = nullptr;
        return nullptr;
    }
    e.second = want;
    return e.first;
}

static void clear_pool(pdg_context *ctx) {
    for (auto &kv : ctx->pool) cudaFree(kv.second.first);
    ctx->pool.clear();
}

static void clear_profile(pdg_context *ctx) {
    for (auto &m : ctx->prof_marks) { cudaEventDestroy(m.a); cudaEventDestroy(m.b); }
    ctx->prof_marks.clear();
}

extern "C" int pdg_profile_enable(pdg_context *ctx, int enable) {
    if (!ctx) return PDG_ERR_ARG;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    clear_profile(ctx);
    ctx->prof = enable != 0;
    return PDG_OK;
}

extern "C" int pdg_profile_region(pdg_context *ctx, const char *name, int *count, double *total_ms) {
    if (!ctx || !name || !count || !total_ms) return PDG_ERR_ARG;
    cudaSetDevice(ctx->device);
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    int c = 0;
    double t = 0.0;
    for (auto &m : ctx->prof_marks) {
        if (std::strcmp(m.name, name) != 0) continue;
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, m.a, m.b) == cudaSuccess) { t += ms; ++c; }
    }
    *count = c;
    *total_ms = t;
    return PDG_OK;
}

// ------------------------------------------------------------------------------------------
// small device helpers
// ------------------------------------------------------------------------------------------
namespace {

__global__ void unpack_scale_kernel(int n, const double *__restrict__ packed, const double *__restrict__ norm,
                                    double *__restrict__ full) {
    const int i = blockIdx.y;
    for (int j = threadIdx.x + blockIdx.x * blockDim.x; j < n; j += blockDim.x * gridDim.x) {
        const int hi = i > j ? i : j, lo = i > j ? j : i;
        const double v = packed[(long long)hi * (hi + 1) / 2 + lo];
        full[(long long)i * n + j] = norm ? v * norm[i] * norm[j] : v;
    }
}

__global__ void pack_scale_kernel(int n, const double *__restrict__ full, const double *__restrict__ norm,
                                  double *__restrict__ packed) {
    const int i = blockIdx.y;
    for (int j = threadIdx.x + blockIdx.x * blockDim.x; j <= i; j += blockDim.x * gridDim.x) {
        const double v = full[(long long)i * n + j];
        packed[(long long)i * (i + 1) / 2 + j] = norm ? v * norm[i] * norm[j] : v;
    }
}

// F[i][j] = cJ (J + J^T) + cK (K + K^T), optionally scaled by norm_i norm_j
__global__ void sym_combine_kernel(int n, const double *__restrict__ J, const double *__restrict__ K, double cJ,
                                   double cK, const double *__restrict__ norm, double *__restrict__ F) {
    const int i = blockIdx.y;
    for (int j = threadIdx.x + blockIdx.x * blockDim.x; j < n; j += blockDim.x * gridDim.x) {
        double v = 0.0;
        if (J) v += cJ * (J[(long long)i * n + j] + J[(long long)j * n + i]);
        if (K) v += cK * (K[(long long)i * n + j] + K[(long long)j * n + i]);
        F[(long long)i * n + j] = norm ? v * norm[i] * norm[j] : v;
    }
}

__global__ void scale_full_kernel(int n, double *__restrict__ M, const double *__restrict__ norm) {
    const int i = blockIdx.y;
    for (int j = threadIdx.x + blockIdx.x * blockDim.x; j < n; j += blockDim.x * gridDim.x)
        M[(long long)i * n + j] *= norm[i] * norm[j];
}

__global__ void add_kernel(long long n, const double *__restrict__ a, double *__restrict__ b) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)blockDim.x * gridDim.x)
        b[k] += a[k];
}

double odd_factorial(int n) {  // (-1)!! = 1
    double f = 1.0;
    for (int i = 3; i <= n; i += 2) f *= i;
    return f;
}

}  // namespace

dim3 row_grid(int n) { return dim3((n + 255) / 256 < 4 ? (n + 255) / 256 : 4, n); }

void pdg_launch_unpack(pdg_context *ctx, int n, const double *packed_dev, const double *norm, double *full) {
    { unpack_scale_kernel<<<row_grid(n), 256, 0, ctx->stream>>>(n, packed_dev, norm, full); pdg_count_launch(); }
}
void pdg_launch_pack(pdg_context *ctx, int n, const double *full, const double *norm, double *packed_dev) {
    { pack_scale_kernel<<<row_grid(n), 256, 0, ctx->stream>>>(n, full, norm, packed_dev); pdg_count_launch(); }
}
void pdg_launch_sym_combine2(pdg_context *ctx, int n, const double *J, const double *K, double cJ, double cK,
                             const double *norm, double *F) {
    { sym_combine_kernel<<<row_grid(n), 256, 0, ctx->stream>>>(n, J, K, cJ, cK, norm, F); pdg_count_launch(); }
}
void pdg_launch_scale_full(pdg_context *ctx, int n, double *M, const double *norm) {
    { scale_full_kernel<<<row_grid(n), 256, 0, ctx->stream>>>(n, M, norm); pdg_count_launch(); }
}
void pdg_launch_add(pdg_context *ctx, long long n, const double *a, double *b) {
    { add_kernel<<<296, 256, 0, ctx->stream>>>(n, a, b); pdg_count_launch(); }
}

// ------------------------------------------------------------------------------------------
// context
// ------------------------------------------------------------------------------------------
// The basis and work arrays are the context's pool buffers ("basis.*", "work.*"): forgetting them
// frees nothing, so a context that serves one molecule after another allocates and frees no
// device memory once it has met the largest (no cudaFree synchronising the other slots' streams).
static void free_basis(pdg_context *ctx) {
    ctx->dbasis = DeviceBasis{};
    ctx->d_c2s = nullptr;
}

static void free_work(pdg_context *ctx) {
    double **bufs[] = {&ctx->d_D, &ctx->d_J, &ctx->d_K, &ctx->d_F, &ctx->d_W, &ctx->d_grad, &ctx->d_scal,
                       &ctx->d_H, &ctx->d_S, &ctx->d_Dout, &ctx->d_Fout, &ctx->d_Dprev, &ctx->d_F2prev, &ctx->d_dmax};
    for (double **p : bufs) *p = nullptr;
    ctx->d_status = nullptr;
    ctx->inc_count = -1;
}

extern "C" int pdg_context_create(int device, pdg_context **out) {
    if (!out) { pdg_set_error("pdg_context_create: null output"); return PDG_ERR_ARG; }
    *out = nullptr;
    int ndev = 0;
    PDG_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) { pdg_set_error("pdg_context_create: device %d of %d", device, ndev); return PDG_ERR_ARG; }
    PDG_CUDA(cudaSetDevice(device));
    pdg_context *ctx = new pdg_context();
    ctx->device = device;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx; pdg_set_error("stream creation failed"); return PDG_ERR_CUDA;
    }
    if (cublasCreate(&ctx->cublas) != CUBLAS_STATUS_SUCCESS) { delete ctx; pdg_set_error("cublasCreate failed"); return PDG_ERR_CUDA; }
    cublasSetStream(ctx->cublas, ctx->stream);
    if (cusolverDnCreate(&ctx->cusolver) != CUSOLVER_STATUS_SUCCESS) { delete ctx; pdg_set_error("cusolverDnCreate failed"); return PDG_ERR_CUDA; }
    cusolverDnSetStream(ctx->cusolver, ctx->stream);
    *out = ctx;
    return PDG_OK;
}

extern "C" int pdg_context_destroy(pdg_context *ctx) {
    if (!ctx) return PDG_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    clear_profile(ctx);
    pdg_scf_release(ctx);
    pdg_free_pairs(ctx);
    pdg_release_dft(ctx);
    free_basis(ctx);
    free_work(ctx);
    clear_pool(ctx);
    if (ctx->cublas) cublasDestroy(ctx->cublas);
    if (ctx->cusolver) cusolverDnDestroy(ctx->cusolver);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return PDG_OK;
}

// Stream-ordered upload into the context's pool buffer `name` on its non-blocking stream, complete
// on return.
template <typename T>
static int upload_vec(pdg_context *ctx, const char *name, T **dst, const std::vector<T> &src) {
    *dst = nullptr;
    if (src.empty()) return PDG_OK;
    *dst = (T *)pdg_pool(ctx, name, src.size() * sizeof(T));
    if (!*dst) { pdg_set_error("device allocation failed (%s)", name); return PDG_ERR_ALLOC; }
    PDG_CUDA(cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    return PDG_OK;
}

// Real solid harmonics from normalised Cartesians for l <= 2, order m = 0, 1c, 1s, 2c, 2s
// (GaussianBasis.c:191-193).  Rows: spherical, columns: Cartesian (xx, xy, yy, xz, yz, zz).
static void c2s_block(int l, std::vector<double> &M) {
    if (l == 0) { M = {1.0}; return; }
    if (l == 1) { M = {0, 0, 1, 1, 0, 0, 0, 1, 0}; return; }
    const double s3 = std::sqrt(3.0);
    M.assign(5 * 6, 0.0);
    // d0 = zz - (xx + yy)/2
    M[0 * 6 + 5] = 1.0; M[0 * 6 + 0] = -0.5; M[0 * 6 + 2] = -0.5;
    // d1c = xz, d1s = yz
    M[1 * 6 + 3] = 1.0;
    M[2 * 6 + 4] = 1.0;
    // d2c = sqrt(3)/2 (xx - yy), d2s = xy
    M[3 * 6 + 0] = 0.5 * s3; M[3 * 6 + 2] = -0.5 * s3;
    M[4 * 6 + 1] = 1.0;
}

extern "C" int pdg_basis_upload(pdg_context *ctx, int n_atoms, const double *Z, int n_shells, const int *shell_atom,
                                const int *l_low, const int *l_high, const int *nprim, const double *exponents,
                                const double *coefficients, int normalized, int spherical) {
    if (!ctx || n_atoms <= 0 || n_shells <= 0 || !Z || !shell_atom || !l_low || !l_high || !nprim || !exponents ||
        !coefficients) {
        pdg_set_error("pdg_basis_upload: invalid argument");
        return PDG_ERR_ARG;
    }
    cudaSetDevice(ctx->device);
    pdg_free_pairs(ctx);
    pdg_free_dft(ctx);
    free_basis(ctx);
    free_work(ctx);
    ctx->natom = n_atoms;
    ctx->Z.assign(Z, Z + n_atoms);
    ctx->shells.clear();
    ctx->prim_exp.clear();
    ctx->prim_coef.clear();
    ctx->bf_norm.clear();
    ctx->bf_atom.clear();
    ctx->bf_l.clear();
    ctx->spherical = spherical ? 1 : 0;
    // keep each atom's shells as given, for the atomic-density guess
    ctx->raw_atom.assign(n_atoms, pdg_context::RawAtomBasis{});
    ctx->raw_normalized = normalized ? 1 : 0;
    ctx->sad.clear();
    {
        size_t e0 = 0, c0 = 0;
        for (int s = 0; s < n_shells; ++s) {
            if (shell_atom[s] < 0 || shell_atom[s] >= n_atoms || nprim[s] <= 0 || l_high[s] < l_low[s]) break;
            auto &ra = ctx->raw_atom[shell_atom[s]];
            ra.llo.push_back(l_low[s]);
            ra.lhi.push_back(l_high[s]);
            ra.np.push_back(nprim[s]);
            ra.ex.insert(ra.ex.end(), exponents + e0, exponents + e0 + nprim[s]);
            const size_t nc = (size_t)(l_high[s] - l_low[s] + 1) * nprim[s];
            ra.co.insert(ra.co.end(), coefficients + c0, coefficients + c0 + nc);
            e0 += nprim[s];
            c0 += nc;
        }
    }
    ctx->lmax = 0;
    const double PI32 = 5.568327996831708;  // pi^(3/2)
    size_t eoff = 0, coff = 0;
    int bf = 0, nout = 0;
    std::vector<std::vector<double>> c2s_blocks;
    std::vector<int> c2s_l;
    for (int s = 0; s < n_shells; ++s) {
        if (shell_atom[s] < 0 || shell_atom[s] >= n_atoms || l_low[s] < 0 || l_high[s] < l_low[s] || nprim[s] <= 0) {
            pdg_set_error("pdg_basis_upload: bad shell %d", s);
            return PDG_ERR_ARG;
        }
        if (l_high[s] > PDG_LMAX) {
            pdg_set_error("pdg_basis_upload: angular momentum %d above the supported maximum %d", l_high[s], PDG_LMAX);
            return PDG_ERR_UNSUPPORTED;
        }
        for (int l = l_low[s]; l <= l_high[s]; ++l) {
            HostShell hs;
            hs.l = l;
            hs.atom = shell_atom[s];
            hs.bf = bf;
            hs.np = nprim[s];
            hs.poff = (int)ctx->prim_exp.size();
            for (int p = 0; p < nprim[s]; ++p) {
                const double e = exponents[eoff + p];
                double c = coefficients[coff + (size_t)(l - l_low[s]) * nprim[s] + p];
                if (normalized) {
                    const double e2 = 2.0 * e;
                    double fac = PI32 / (e2 * std::sqrt(e2));
                    for (int i = 1; i <= l; ++i) fac *= (double)(2 * i - 1) / (2.0 * e2);
                    c /= std::sqrt(fac);
                }
                ctx->prim_exp.push_back(e);
                ctx->prim_coef.push_back(c);
            }
            ctx->shells.push_back(hs);
            for (int i = 0; i < ncart(l); ++i) {
                const int x = cart_x(l, i), y = cart_y(l, i), z = cart_z(l, i);
                ctx->bf_norm.push_back(std::sqrt(odd_factorial(2 * l - 1) /
                                                 (odd_factorial(2 * x - 1) * odd_factorial(2 * y - 1) * odd_factorial(2 * z - 1))));
                ctx->bf_atom.push_back(shell_atom[s]);
                ctx->bf_l.push_back(l);
            }
            bf += ncart(l);
            nout += spherical ? 2 * l + 1 : ncart(l);
            if (l > ctx->lmax) ctx->lmax = l;
            std::vector<double> blk;
            c2s_block(l, blk);
            c2s_blocks.push_back(blk);
            c2s_l.push_back(l);
        }
        eoff += nprim[s];
        coff += (size_t)(l_high[s] - l_low[s] + 1) * nprim[s];
    }
    ctx->nbf = bf;
    ctx->nbf_out = nout;
    ctx->c2s.clear();
    if (spherical) {
        ctx->c2s.assign((size_t)nout * bf, 0.0);
        int r0 = 0, c0 = 0;
        for (size_t k = 0; k < c2s_blocks.size(); ++k) {
            const int l = c2s_l[k], nr = 2 * l + 1, nc = ncart(l);
            for (int r = 0; r < nr; ++r)
                for (int c = 0; c < nc; ++c) ctx->c2s[(size_t)(r0 + r) * bf + c0 + c] = c2s_blocks[k][r * nc + c];
            r0 += nr;
            c0 += nc;
        }
    }
    // device copies
    std::vector<int> sl, sa, sb, sn, so;
    for (const auto &h : ctx->shells) { sl.push_back(h.l); sa.push_back(h.atom); sb.push_back(h.bf); sn.push_back(h.np); so.push_back(h.poff); }
    DeviceBasis &db = ctx->dbasis;
    db.nshell = (int)ctx->shells.size();
    db.nbf = bf;
    db.natom = n_atoms;
    PDG_CHECK(upload_vec(ctx, "basis.sh_l", &db.sh_l, sl));
    PDG_CHECK(upload_vec(ctx, "basis.sh_atom", &db.sh_atom, sa));
    PDG_CHECK(upload_vec(ctx, "basis.sh_bf", &db.sh_bf, sb));
    PDG_CHECK(upload_vec(ctx, "basis.sh_np", &db.sh_np, sn));
    PDG_CHECK(upload_vec(ctx, "basis.sh_poff", &db.sh_poff, so));
    PDG_CHECK(upload_vec(ctx, "basis.prim_exp", &db.prim_exp, ctx->prim_exp));
    PDG_CHECK(upload_vec(ctx, "basis.prim_coef", &db.prim_coef, ctx->prim_coef));
    PDG_CHECK(upload_vec(ctx, "basis.atom_Z", &db.atom_Z, ctx->Z));
    PDG_CHECK(upload_vec(ctx, "basis.bf_norm", &db.bf_norm, ctx->bf_norm));
    PDG_CHECK(upload_vec(ctx, "basis.bf_atom", &db.bf_atom, ctx->bf_atom));
    {
        std::vector<int> bsh;
        for (size_t k = 0; k < ctx->shells.size(); ++k)
            for (int i = 0; i < ncart(ctx->shells[k].l); ++i) bsh.push_back((int)k);
        PDG_CHECK(upload_vec(ctx, "basis.bf_shell", &db.bf_shell, bsh));
    }
    if (spherical) PDG_CHECK(upload_vec(ctx, "basis.c2s", &ctx->d_c2s, ctx->c2s));
    db.atom_xyz = (double *)pdg_pool(ctx, "basis.atom_xyz", 3 * n_atoms * sizeof(double));
    if (!db.atom_xyz) { pdg_set_error("device allocation failed (basis.atom_xyz)"); return PDG_ERR_ALLOC; }
    ctx->have_geometry = false;
    return pdg_alloc_work(ctx);
}

int pdg_alloc_work(pdg_context *ctx) {
    free_work(ctx);
    const size_t nn = (size_t)ctx->nbf * ctx->nbf * sizeof(double);
    const size_t no = (size_t)ctx->nbf_out * ctx->nbf_out * sizeof(double);
    double **bufs[] = {&ctx->d_D, &ctx->d_J, &ctx->d_K, &ctx->d_F, &ctx->d_W, &ctx->d_H, &ctx->d_S, &ctx->d_Dprev, &ctx->d_F2prev};
    const char *names[] = {"work.D", "work.J", "work.K", "work.F", "work.W", "work.H", "work.S", "work.Dprev", "work.F2prev"};
    for (int k = 0; k < 9; ++k)
        if (!(*bufs[k] = (double *)pdg_pool(ctx, names[k], nn))) { pdg_set_error("device allocation of %zu bytes failed", nn); return PDG_ERR_ALLOC; }
    const size_t ns = ctx->shells.size();
    ctx->d_dmax = (double *)pdg_pool(ctx, "work.dmax", std::max<size_t>(1, ns * ns) * sizeof(double));
    ctx->d_Dout = (double *)pdg_pool(ctx, "work.Dout", no);
    ctx->d_Fout = (double *)pdg_pool(ctx, "work.Fout", no);
    ctx->d_grad = (double *)pdg_pool(ctx, "work.grad", 3 * ctx->natom * sizeof(double));
    ctx->d_scal = (double *)pdg_pool(ctx, "work.scal", 64 * sizeof(double));
    ctx->d_status = (int *)pdg_pool(ctx, "work.status", 16 * sizeof(int));
    if (!ctx->d_dmax || !ctx->d_Dout || !ctx->d_Fout || !ctx->d_grad || !ctx->d_scal || !ctx->d_status) {
        pdg_set_error("device allocation failed");
        return PDG_ERR_ALLOC;
    }
    PDG_CUDA(cudaMemsetAsync(ctx->d_status, 0, 16 * sizeof(int), ctx->stream));
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    return PDG_OK;
}

extern "C" int pdg_basis_size(const pdg_context *ctx, int *n_functions, int *n_cartesian) {
    if (!ctx) return PDG_ERR_ARG;
    if (n_functions) *n_functions = ctx->nbf_out;
    if (n_cartesian) *n_cartesian = ctx->nbf;
    return PDG_OK;
}

extern "C" int pdg_geometry_set(pdg_context *ctx, const double *xyz) {
    if (!ctx || !xyz) { pdg_set_error("pdg_geometry_set: invalid argument"); return PDG_ERR_ARG; }
    if (ctx->nbf == 0) { pdg_set_error("pdg_geometry_set: no basis"); return PDG_ERR_STATE; }
    for (int k = 0; k < 3 * ctx->natom; ++k)
        if (!std::isfinite(xyz[k])) { pdg_set_error("pdg_geometry_set: non-finite coordinate"); return PDG_ERR_NAN; }
    cudaSetDevice(ctx->device);
    ctx->xyz.assign(xyz, xyz + 3 * ctx->natom);
    PDG_CUDA(cudaMemcpyAsync(ctx->dbasis.atom_xyz, xyz, 3 * ctx->natom * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    pdg_free_pairs(ctx);
    pdg_free_dft(ctx);
    ctx->have_geometry = true;
    ctx->inc_count = -1;
    return PDG_OK;
}

extern "C" int pdg_set_eri_options(pdg_context *ctx, double schwarz_cut, double tei_underflow, int precision_mode,
                                   double mixed_cut) {
    if (!ctx || schwarz_cut < 0.0 || tei_underflow < 0.0 || precision_mode < 0 || precision_mode > 1 || mixed_cut < 0.0) {
        pdg_set_error("pdg_set_eri_options: invalid argument");
        return PDG_ERR_ARG;
    }
    ctx->schwarz_cut = schwarz_cut;
    ctx->tei_underflow = tei_underflow;
    ctx->precision_mode = precision_mode;
    ctx->mixed_cut = mixed_cut;
    ctx->blocks_thr = -1.0;
    return PDG_OK;
}

static int require_ready(pdg_context *ctx, const char *who) {
    if (!ctx) { pdg_set_error("%s: null context", who); return PDG_ERR_ARG; }
    if (ctx->nbf == 0) { pdg_set_error("%s: no basis", who); return PDG_ERR_STATE; }
    if (!ctx->have_geometry) { pdg_set_error("%s: no geometry", who); return PDG_ERR_STATE; }
    cudaSetDevice(ctx->device);
    return PDG_OK;
}

double pdg_nuclear_energy(const pdg_context *ctx, std::vector<double> *grad) {
    double e = 0.0;
    for (int i = 0; i < ctx->natom; ++i)
        for (int j = 0; j < i; ++j) {
            const double dx = ctx->xyz[3 * i] - ctx->xyz[3 * j], dy = ctx->xyz[3 * i + 1] - ctx->xyz[3 * j + 1],
                         dz = ctx->xyz[3 * i + 2] - ctx->xyz[3 * j + 2];
            const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
            const double zz = ctx->Z[i] * ctx->Z[j];
            e += zz / r;
            if (grad) {
                const double f = -zz / (r * r * r);
                (*grad)[3 * i] += f * dx; (*grad)[3 * i + 1] += f * dy; (*grad)[3 * i + 2] += f * dz;
                (*grad)[3 * j] -= f * dx; (*grad)[3 * j + 1] -= f * dy; (*grad)[3 * j + 2] -= f * dz;
            }
        }
    return e;
}

// Cartesian normalised S and H (full, nbf x nbf) into ctx->d_S / ctx->d_H.
int pdg_qcmm_add_potentials(pdg_context *ctx, double *Vc);

int pdg_compute_one_electron(pdg_context *ctx) {
    PDG_CHECK(pdg_ensure_pairs(ctx));
    const int n = ctx->nbf;
    PDG_CHECK(pdg_oneint(ctx, ctx->d_S, ctx->d_J, ctx->d_K));
    PDG_CHECK(pdg_qcmm_add_potentials(ctx, ctx->d_K));  // MM point charges, when set
    // H = T + V
    pdg_launch_add(ctx, (long long)n * n, ctx->d_J, ctx->d_K);
    PDG_CUDA(cudaMemcpyAsync(ctx->d_H, ctx->d_K, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    pdg_launch_scale_full(ctx, n, ctx->d_S, ctx->dbasis.bf_norm);
    pdg_launch_scale_full(ctx, n, ctx->d_H, ctx->dbasis.bf_norm);
    PDG_CUDA(cudaGetLastError());
    return PDG_OK;
}

// Output-basis (spherical or Cartesian) full matrix from a Cartesian one: M_out = C M C^T.
int pdg_cart_to_out(pdg_context *ctx, const double *Mc, double *Mo) {
    const int n = ctx->nbf, m = ctx->nbf_out;
    if (!ctx->spherical) {
        PDG_CUDA(cudaMemcpyAsync(Mo, Mc, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        return PDG_OK;
    }
    // Row-major C (m x n) is column-major C^T (n x m).  tmp(col-major n x m) = Mc * C^T ; Mo = C * tmp
    double *tmp = ctx->d_F;  // n*n >= n*m
    const double one = 1.0, zero = 0.0;
    if (cublasDgemm(ctx->cublas, CUBLAS_OP_N, CUBLAS_OP_N, n, m, n, &one, Mc, n, ctx->d_c2s, n, &zero, tmp, n) != CUBLAS_STATUS_SUCCESS ||
        cublasDgemm(ctx->cublas, CUBLAS_OP_T, CUBLAS_OP_N, m, m, n, &one, ctx->d_c2s, n, tmp, n, &zero, Mo, m) != CUBLAS_STATUS_SUCCESS) {
        pdg_set_error("cublasDgemm failed (c2s)");
        return PDG_ERR_CUDA;
    }
    return PDG_OK;
}

// Cartesian full matrix from an output-basis one (density-like): M_c = C^T M_o C.
int pdg_out_to_cart(pdg_context *ctx, const double *Mo, double *Mc) {
    const int n = ctx->nbf, m = ctx->nbf_out;
    if (!ctx->spherical) {
        PDG_CUDA(cudaMemcpyAsync(Mc, Mo, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        return PDG_OK;
    }
    double *tmp = ctx->d_F;
    const double one = 1.0, zero = 0.0;
    // tmp (col-major m x n) = Mo * C ; Mc (n x n) = C^T * tmp
    if (cublasDgemm(ctx->cublas, CUBLAS_OP_N, CUBLAS_OP_T, m, n, m, &one, Mo, m, ctx->d_c2s, n, &zero, tmp, m) != CUBLAS_STATUS_SUCCESS ||
        cublasDgemm(ctx->cublas, CUBLAS_OP_N, CUBLAS_OP_N, n, n, m, &one, ctx->d_c2s, n, tmp, m, &zero, Mc, n) != CUBLAS_STATUS_SUCCESS) {
        pdg_set_error("cublasDgemm failed (s2c)");
        return PDG_ERR_CUDA;
    }
    return PDG_OK;
}

extern "C" int pdg_one_electron(pdg_context *ctx, double *overlap, double *core, double *e_nuclear) {
    PDG_CHECK(require_ready(ctx, "pdg_one_electron"));
    PDG_CHECK(pdg_compute_one_electron(ctx));
    const int m = ctx->nbf_out;
    const size_t np = (size_t)m * (m + 1) / 2;
    double *dpk = (double *)pdg_pool(ctx, "packed.tmp", np * sizeof(double));
    if (!dpk) { pdg_set_error("device buffer allocation failed"); return PDG_ERR_ALLOC; }
    int st = PDG_OK;
    if (overlap) {
        st = pdg_cart_to_out(ctx, ctx->d_S, ctx->d_Dout);
        if (st == PDG_OK) {
            pdg_launch_pack(ctx, m, ctx->d_Dout, nullptr, dpk);
            if (cudaMemcpyAsync(overlap, dpk, np * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) st = PDG_ERR_CUDA;
            cudaStreamSynchronize(ctx->stream);
        }
    }
    if (core && st == PDG_OK) {
        st = pdg_cart_to_out(ctx, ctx->d_H, ctx->d_Dout);
        if (st == PDG_OK) {
            pdg_launch_pack(ctx, m, ctx->d_Dout, nullptr, dpk);
            if (cudaMemcpyAsync(core, dpk, np * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess) st = PDG_ERR_CUDA;
        }
    }
    cudaStreamSynchronize(ctx->stream);
    if (st != PDG_OK) return st;
    PDG_CUDA(cudaGetLastError());
    if (e_nuclear) *e_nuclear = pdg_nuclear_energy(ctx, nullptr);
    return PDG_OK;
}

// Upload a packed output-basis density and produce the scaled Cartesian D' = N C^T D C N in ctx->d_D.
int pdg_load_density(pdg_context *ctx, const double *packed_host) {
    const int m = ctx->nbf_out;
    const size_t np = (size_t)m * (m + 1) / 2;
    double *dpk = (double *)pdg_pool(ctx, "packed.tmp", np * sizeof(double));
    if (!dpk) { pdg_set_error("device buffer allocation failed"); return PDG_ERR_ALLOC; }
    if (cudaMemcpyAsync(dpk, packed_host, np * sizeof(double), cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess) {
        pdg_set_error("density upload failed"); return PDG_ERR_CUDA;
    }
    pdg_launch_unpack(ctx, m, dpk, nullptr, ctx->d_Dout);
    cudaStreamSynchronize(ctx->stream);
    PDG_CHECK(pdg_out_to_cart(ctx, ctx->d_Dout, ctx->d_D));
    pdg_launch_scale_full(ctx, ctx->nbf, ctx->d_D, ctx->dbasis.bf_norm);
    PDG_CUDA(cudaGetLastError());
    return PDG_OK;
}

// Two-electron Fock from the scaled Cartesian density already in ctx->d_D; the normalised
// Cartesian F2 goes to d_F2 (full nbf x nbf).
int pdg_fock2_device(pdg_context *ctx, double cx, bool doJ, double *d_F2) {
    const int n = ctx->nbf;
    const size_t nn = (size_t)n * n * sizeof(double);
    const bool doK = cx != 0.0;
    if (doJ) PDG_CUDA(cudaMemsetAsync(ctx->d_J, 0, nn, ctx->stream));
    if (doK) PDG_CUDA(cudaMemsetAsync(ctx->d_K, 0, nn, ctx->stream));
    if (doJ || doK) PDG_CHECK(pdg_eri_jk(ctx, ctx->d_D, ctx->d_J, ctx->d_K, doJ, doK));
    pdg_launch_sym_combine2(ctx, n, doJ ? ctx->d_J : nullptr, doK ? ctx->d_K : nullptr, 1.0, -0.5 * cx,
                            ctx->dbasis.bf_norm, d_F2);
    PDG_CUDA(cudaGetLastError());
    return PDG_OK;
}

namespace {
__global__ void diff_kernel(long long n, const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ c) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)blockDim.x * gridDim.x)
        c[k] = a[k] - b[k];
}
}  // namespace

// SCF Fock build of the two-electron part.  After a full build the next ones are difference
// builds F2 = F2_prev + G(D' - D'_prev), with quartets skipped when Q_AB Q_CD max|dD'| < inc_cut
// (mixed mode: mixed_dcut when larger, the same bound for the full builds);
// G is linear in the density (the underflow drop depends only on the integral), so the sum equals
// a full build up to the skipped contributions.  A full build is made again every inc_rebuild steps.
int pdg_fock2_scf(pdg_context *ctx, double cx, bool doJ, double *d_F2) {
    const int n = ctx->nbf;
    const size_t nn = (size_t)n * n * sizeof(double);
    const bool doK = cx != 0.0;
    const bool full = !ctx->incremental || ctx->inc_count < 0 || ctx->inc_count >= ctx->inc_rebuild;
    if (full) {
        // full build, density-screened at the difference builds' bound (J and K parts separately)
        if (doJ) PDG_CUDA(cudaMemsetAsync(ctx->d_J, 0, nn, ctx->stream));
        if (doK) PDG_CUDA(cudaMemsetAsync(ctx->d_K, 0, nn, ctx->stream));
        PDG_CHECK(pdg_shell_pair_dmax(ctx, ctx->d_D, ctx->d_dmax));
        if (doJ || doK) PDG_CHECK(pdg_eri_jk_screened(ctx, ctx->d_D, ctx->d_J, ctx->d_K, doJ, doK, ctx->d_dmax, pdg_fock_dcut(ctx)));
        pdg_launch_sym_combine2(ctx, n, doJ ? ctx->d_J : nullptr, doK ? ctx->d_K : nullptr, 1.0, -0.5 * cx,
                                ctx->dbasis.bf_norm, d_F2);
        ctx->inc_count = 0;
    } else {
        // dD' in d_W (free during the SCF)
        { diff_kernel<<<296, 256, 0, ctx->stream>>>((long long)n * n, ctx->d_D, ctx->d_Dprev, ctx->d_W); pdg_count_launch(); }
        PDG_CHECK(pdg_shell_pair_dmax(ctx, ctx->d_W, ctx->d_dmax));
        if (doJ) PDG_CUDA(cudaMemsetAsync(ctx->d_J, 0, nn, ctx->stream));
        if (doK) PDG_CUDA(cudaMemsetAsync(ctx->d_K, 0, nn, ctx->stream));
        if (doJ || doK) PDG_CHECK(pdg_eri_jk_screened(ctx, ctx->d_W, ctx->d_J, ctx->d_K, doJ, doK, ctx->d_dmax, pdg_fock_dcut(ctx)));
        pdg_launch_sym_combine2(ctx, n, doJ ? ctx->d_J : nullptr, doK ? ctx->d_K : nullptr, 1.0, -0.5 * cx,
                                ctx->dbasis.bf_norm, d_F2);
        pdg_launch_add(ctx, (long long)n * n, ctx->d_F2prev, d_F2);
        ++ctx->inc_count;
    }
    PDG_CUDA(cudaMemcpyAsync(ctx->d_F2prev, d_F2, nn, cudaMemcpyDeviceToDevice, ctx->stream));
    PDG_CUDA(cudaMemcpyAsync(ctx->d_Dprev, ctx->d_D, nn, cudaMemcpyDeviceToDevice, ctx->stream));
    PDG_CUDA(cudaGetLastError());
    return PDG_OK;
}

extern "C" int pdg_set_incremental(pdg_context *ctx, int enable, double density_cut, int rebuild_period) {
    if (!ctx || density_cut < 0.0 || rebuild_period < 0) { pdg_set_error("pdg_set_incremental: invalid argument"); return PDG_ERR_ARG; }
    ctx->incremental = enable ? 1 : 0;
    ctx->inc_cut = density_cut;
    ctx->inc_rebuild = rebuild_period;
    ctx->inc_count = -1;
    return PDG_OK;
}

// Pack an output-basis full matrix to host.
int pdg_store_packed(pdg_context *ctx, const double *d_full_out, double *packed_host) {
    const int m = ctx->nbf_out;
    const size_t np = (size_t)m * (m + 1) / 2;
    double *dpk = (double *)pdg_pool(ctx, "packed.tmp", np * sizeof(double));
    if (!dpk) { pdg_set_error("device buffer allocation failed"); return PDG_ERR_ALLOC; }
    pdg_launch_pack(ctx, m, d_full_out, nullptr, dpk);
    cudaError_t e = cudaMemcpyAsync(packed_host, dpk, np * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) { pdg_set_error("packed download failed"); return PDG_ERR_CUDA; }
    return PDG_OK;
}

static double packed_trace_product(int m, const double *a, const double *b) {
    double t = 0.0;
    for (int i = 0; i < m; ++i) {
        const size_t r = (size_t)i * (i + 1) / 2;
        for (int j = 0; j < i; ++j) t += 2.0 * a[r + j] * b[r + j];
        t += a[r + i] * b[r + i];
    }
    return t;
}

extern "C" int pdg_fock_two_electron(pdg_context *ctx, const double *density, double cx, int do_coulomb, double *fock,
                                     double *e2) {
    PDG_CHECK(require_ready(ctx, "pdg_fock_two_electron"));
    if (!density || !fock) { pdg_set_error("pdg_fock_two_electron: null array"); return PDG_ERR_ARG; }
    PDG_CHECK(pdg_ensure_pairs(ctx));
    PDG_CHECK(pdg_load_density(ctx, density));
    PDG_CHECK(pdg_fock2_device(ctx, cx, do_coulomb != 0, ctx->d_F));
    PDG_CHECK(pdg_cart_to_out(ctx, ctx->d_F, ctx->d_Fout));
    PDG_CHECK(pdg_store_packed(ctx, ctx->d_Fout, fock));
    PDG_CUDA(cudaGetLastError());
    if (e2) *e2 = 0.5 * packed_trace_product(ctx->nbf_out, density, fock);
    return PDG_OK;
}

// Gradient of nuclear, one-electron and two-electron terms from device-resident scaled
// Cartesian D' (ctx->d_D) and W' (ctx->d_W, standard convention sum n e C C^T).
int pdg_gradients_device(pdg_context *ctx, double cx, bool doJ, std::vector<double> &g) {
    const int na = ctx->natom;
    PDG_CUDA(cudaMemsetAsync(ctx->d_grad, 0, 3 * na * sizeof(double), ctx->stream));
    PDG_CHECK(pdg_oneint_grad(ctx, ctx->d_D, ctx->d_W, ctx->d_grad));
    if (doJ || cx != 0.0) PDG_CHECK(pdg_eri_grad(ctx, ctx->d_D, cx, doJ, ctx->d_grad));
    std::vector<double> h(3 * na);
    PDG_CUDA(cudaMemcpyAsync(h.data(), ctx->d_grad, 3 * na * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    pdg_nuclear_energy(ctx, &h);
    for (int k = 0; k < 3 * na; ++k) g[k] += h[k];
    return PDG_OK;
}

extern "C" int pdg_gradients(pdg_context *ctx, const double *density, const double *wdensity, double cx, int do_coulomb,
                             double *gradients3) {
    PDG_CHECK(require_ready(ctx, "pdg_gradients"));
    if (!density || !wdensity || !gradients3) { pdg_set_error("pdg_gradients: null array"); return PDG_ERR_ARG; }
    PDG_CHECK(pdg_ensure_pairs(ctx));
    // W' = N C^T (-W_ref / 2) C N
    PDG_CHECK(pdg_load_density(ctx, wdensity));
    PDG_CUDA(cudaMemcpyAsync(ctx->d_W, ctx->d_D, (size_t)ctx->nbf * ctx->nbf * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
    const double mhalf = -0.5;
    if (cublasDscal(ctx->cublas, ctx->nbf * ctx->nbf, &mhalf, ctx->d_W, 1) != CUBLAS_STATUS_SUCCESS) {
        pdg_set_error("cublasDscal failed"); return PDG_ERR_CUDA;
    }
    PDG_CHECK(pdg_load_density(ctx, density));
    std::vector<double> g(3 * ctx->natom, 0.0);
    PDG_CHECK(pdg_gradients_device(ctx, cx, do_coulomb != 0, g));
    for (int k = 0; k < 3 * ctx->natom; ++k) gradients3[k] += g[k];
    return PDG_OK;
}
