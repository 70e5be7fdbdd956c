// Library context: device-resident basis, geometry, shell-pair lists and work buffers.
#pragma once
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <map>
#include <string>
#include <vector>

#include "common.cuh"

struct HostShell {          // one split shell (a single angular momentum)
    int l, atom, bf, np, poff;
};

// One (bra class, ket class) block of the screened shell-quartet work list, split by the
// primitive-count bucket of the ket pair.
struct QuartetBlock {
    int cb, ck;             // pair classes
    long long total;        // number of quartets (all buckets)
    int nsub;               // non-empty ket buckets
    struct Sub {
        long long total;    // quartets with a ket of this bucket
        long long *offs;    // device prefix sums over bra pairs (bra.n + 1)
        int *cbra;          // device: bra pair of quartet min(4k, total-1), k = 0 .. (total-1)/4 + 1
        int k0, nk;         // the bucket's kets: [k0, k0 + nk) of the ket class list
        int bucket;
    } sub[PDG_NBUCKET];
};

struct GridData;            // DFT grid (dft.cu)
struct XCData;              // functional + per-point buffers (dft.cu)

struct pdg_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    cublasHandle_t cublas = nullptr;
    cusolverDnHandle_t cusolver = nullptr;

    // ---- basis (host copy) ----
    int natom = 0, nbf = 0, nbf_out = 0, spherical = 0;
    std::vector<double> Z;                 // nuclear charges
    std::vector<int> atomic_numbers;
    std::vector<HostShell> shells;         // split shells
    std::vector<double> prim_exp, prim_coef;
    std::vector<double> bf_norm;           // per Cartesian function
    std::vector<int> bf_atom;
    std::vector<int> bf_l;
    std::vector<double> c2s;               // nbf_out x nbf (row-major), only if spherical
    int lmax = 0;
    DeviceBasis dbasis{};
    double *d_c2s = nullptr;

    // ---- geometry ----
    std::vector<double> xyz;               // natom*3 bohr
    bool have_geometry = false;

    // ---- shell pairs ----
    PairList pairs[PDG_NPAIRCLASS]{};      // device arrays
    std::vector<double> hostQ[PDG_NPAIRCLASS];     // per class, ordered by bucket then Q descending
    std::vector<int> bucket_start[PDG_NPAIRCLASS]; // per class: first pair of each bucket (PDG_NBUCKET + 1)
    std::vector<int> hostPoff[PDG_NPAIRCLASS], hostNp[PDG_NPAIRCLASS];  // sorted pair -> primitive pairs
    std::vector<double> hostArg;                                        // primitive-pair exponent arguments
    PrimPairs pp{};
    int npp = 0;
    double qmax[PDG_NPAIRCLASS]{};
    std::vector<QuartetBlock> blocks;      // energy work list
    double blocks_thr = -1.0;

    // ---- options ----
    double schwarz_cut = 1.0e-13;          // quartet bound below which the quartet is skipped
    double tei_underflow = 1.0e-12;        // reference storage underflow (BlockStorage)
    int precision_mode = 0;                // 0 = FP64, 1 = mixed
    double mixed_cut = 1.0e-6;             // Schwarz x density bound below which FP32 is used
    double mixed_drop = 1.0e-10;           // mixed mode: gradient quartets with Schwarz x |Gamma| below are skipped
    double mixed_dcut = 1.0e-11;           // mixed mode: SCF Fock-build quartets with Schwarz x density below are skipped

    // ---- incremental Fock builds in the SCF: F2_k = F2_{k-1} + G(D_k - D_{k-1}) ----
    int incremental = 1;
    double inc_cut = 1.0e-13;              // density-screening bound for the difference builds
    int inc_rebuild = 16;                  // full rebuild after this many difference builds
    double *d_Dprev = nullptr, *d_F2prev = nullptr, *d_dmax = nullptr;
    int inc_count = -1;                    // < 0: no valid previous build

    // ---- QC/MM: MM point charges (x, y, z, q per charge, bohr) ----
    int nmm = 0;
    double *d_mm = nullptr;                // pool buffer "qcmm.charges"

    // ---- work buffers (nbf x nbf, Cartesian) ----
    double *d_D = nullptr, *d_J = nullptr, *d_K = nullptr, *d_F = nullptr, *d_W = nullptr;
    double *d_grad = nullptr;              // natom*3
    double *d_scal = nullptr;              // small scalars
    double *d_H = nullptr, *d_S = nullptr; // Cartesian one-electron matrices (normalised)
    double *d_Dout = nullptr;              // nbf_out x nbf_out scratch
    double *d_Fout = nullptr;
    int *d_status = nullptr;

    // ---- superposition-of-atomic-densities guess ----
    int guess_sad = 1;
    std::vector<double> occ;               // orbital occupations overriding 2 x nocc (atomic runs only)
    struct RawAtomBasis {
        std::vector<int> llo, lhi, np;
        std::vector<double> ex, co;
    };
    std::vector<RawAtomBasis> raw_atom;    // each atom's shells as uploaded
    int raw_normalized = 1;
    std::map<int, std::vector<double>> sad;  // element -> packed atomic density (output basis)

    // ---- named device buffers kept across geometries (grown, never shrunk) ----
    std::map<std::string, std::pair<void *, size_t>> pool;

    // ---- DFT ----
    GridData *grid = nullptr;
    XCData *xc = nullptr;

    // ---- statistics of the last Fock build ----
    long long last_quartets = 0;
    unsigned long long *d_count32 = nullptr;  // running count of shell quartets evaluated in FP32
    // screening of the last two-electron gradient (pdg_eri_grad), for its work estimate: the
    // shell-pair density maxima stay in the pool buffer "grad_dmax"
    bool grad_valid = false;
    int grad_doJ = 0;
    double grad_cx = 0.0, grad_gcut = 0.0;

    // ---- optional per-region device timing (CUDA events on the context stream) ----
    struct ProfMark {
        const char *name;
        cudaEvent_t a, b;
    };
    bool prof = false;
    std::vector<ProfMark> prof_marks;
};

// Brackets the kernels issued in its lifetime with CUDA events when profiling is enabled.
struct ProfScope {
    pdg_context *c;
    int idx = -1;
    ProfScope(pdg_context *ctx, const char *name) : c(ctx) {
        if (!c->prof) return;
        pdg_context::ProfMark m{name, nullptr, nullptr};
        if (cudaEventCreate(&m.a) != cudaSuccess || cudaEventCreate(&m.b) != cudaSuccess) return;
        cudaEventRecord(m.a, c->stream);
        c->prof_marks.push_back(m);
        idx = (int)c->prof_marks.size() - 1;
    }
    ~ProfScope() {
        if (idx >= 0) cudaEventRecord(c->prof_marks[idx].b, c->stream);
    }
};

// Density-screening bound of the SCF's Fock builds (full and difference): inc_cut, raised to
// mixed_dcut in the mixed mode.
inline double pdg_fock_dcut(const pdg_context *ctx) {
    return (ctx->precision_mode == 1 && ctx->mixed_dcut > ctx->inc_cut) ? ctx->mixed_dcut : ctx->inc_cut;
}

// Kernel view of a work-list block: lanes[bucket] lanes per quartet in 128-thread CTAs, the buckets'
// CTAs one after another.  Returns the number of CTAs of the launch.
inline long long pdg_fill_work(WorkList &w, const QuartetBlock &b, const int (&lanes)[PDG_NBUCKET]) {
    long long cta = 0;
    w.nsub = b.nsub;
    for (int k = 0; k < PDG_NBUCKET; ++k) {
        if (k < b.nsub) {
            const auto &s = b.sub[k];
            const int l = lanes[s.bucket];
            w.sub[k] = WorkSub{s.offs, s.cbra, s.total, cta, s.k0, l};
            cta += (s.total * l + 127) / 128;
        } else {
            w.sub[k] = WorkSub{nullptr, nullptr, 0, cta, 0, 1};
        }
    }
    return cta;
}

int pdg_ensure_pairs(pdg_context *ctx);
int pdg_build_blocks(pdg_context *ctx, double thr);
// Number of kets of [k0, k0 + nk) of class ck with Q >= need (the bucket is sorted by Q descending),
// limited to ket index <= bra for a same-class block; the rule the work lists and the work
// estimate share.
long long pdg_ket_count(const pdg_context *ctx, int cb, int ck, int ib, int k0, int nk, double thr);
int pdg_alloc_work(pdg_context *ctx);
void pdg_free_pairs(pdg_context *ctx);
void pdg_free_dft(pdg_context *ctx);
void pdg_release_dft(pdg_context *ctx);
int pdg_xc_kind(const char *name, int *kind);  // functional name -> xc::Kind (dft.cu)

// Cartesian <-> output-basis helpers (util.cu)
int pdg_unpack_density(pdg_context *ctx, const double *packed_host, double *d_full_cart_scaled);
int pdg_pack_fock(pdg_context *ctx, const double *d_full_cart, double *packed_host);
void pdg_launch_sym_combine(pdg_context *ctx, double cJ, double cK, bool doK);

// Kernel drivers
int pdg_eri_jk(pdg_context *ctx, const double *d_Dscaled, double *d_J, double *d_K, bool doJ, bool doK);
int pdg_eri_jk_screened(pdg_context *ctx, const double *d_Dscaled, double *d_J, double *d_K, bool doJ, bool doK,
                        const double *d_dmax, double dcut);
int pdg_shell_pair_dmax(pdg_context *ctx, const double *d_D, double *d_dmax);
int pdg_eri_grad(pdg_context *ctx, const double *d_Dscaled, double cx, bool doJ, double *d_grad);
int pdg_oneint(pdg_context *ctx, double *d_S, double *d_T, double *d_V);
int pdg_oneint_grad(pdg_context *ctx, const double *d_Dscaled, const double *d_Wscaled, double *d_grad);

// Device buffer `name` of at least `bytes` bytes owned by the context (api.cu); nullptr on failure.
void *pdg_pool(pdg_context *ctx, const char *name, size_t bytes);

// SCF helpers (scf.cu, sad.cu)
void pdg_scf_release(const pdg_context *ctx);
int pdg_sad_density(pdg_context *ctx, std::vector<double> &full_out);  // m x m guess density
