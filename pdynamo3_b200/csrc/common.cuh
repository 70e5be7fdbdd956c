// Shared definitions for the pdgpu Fock-build library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include "../../include/pdgpu.h"

#define PDG_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            pdg_set_error("%s:%d: %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
            return PDG_ERR_CUDA;                                                         \
        }                                                                                \
    } while (0)

#define PDG_CHECK(call)                  \
    do {                                 \
        int s_ = (call);                 \
        if (s_ != PDG_OK) return s_;     \
    } while (0)

void pdg_set_error(const char *fmt, ...);

// Raises a kernel's dynamic shared-memory limit to the device's opt-in maximum.  The limit is a
// process-wide attribute of the function: setting it to the size of each launch would race when
// server slots (host threads) launch the kernel with different sizes at once; every caller setting
// the same maximum does not, and each launch still asks only for what it uses.
template <typename K>
inline cudaError_t pdg_allow_max_smem(K kernel) {
    int dev = 0, mx = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&mx, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    return e;
}
void pdg_count_launch();  // process-wide count of kernel launches made by this library

// Largest angular momentum of a (split) shell handled by the integral kernels: d.
#define PDG_LMAX 2
#define PDG_NPAIRCLASS 6  // (0,0) (1,0) (1,1) (2,0) (2,1) (2,2)
#define PDG_MAX_DIIS 16   // largest DIIS history of the SCF drivers (one batched reduction per cycle)

// Primitive-pair cut of the reference: exp(-arg) below 1e-18 is dropped
// (GaussianBases/__extensions__/cinclude/GaussianBasis.h:24,58, applied at
// GaussianBasisIntegrals_f2Xf2.c:693,712).
#define PDG_PRIMITIVE_CUT (2.30258509299405e+00 * 18.0)

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int pair_class(int la, int lb) { return la * (la + 1) / 2 + lb; }  // la >= lb

// Cartesian component powers in the reference order: for z in 0..l, for y in 0..l-z, x = l-y-z
// (GaussianBasis.c:184-190, :590-627).
__host__ __device__ constexpr int cart_x(int l, int i) {
    return (l == 0) ? 0 : (l == 1) ? (i == 0 ? 1 : 0)
         : (i == 0 ? 2 : i == 1 ? 1 : i == 2 ? 0 : i == 3 ? 1 : 0);
}
__host__ __device__ constexpr int cart_y(int l, int i) {
    return (l == 0) ? 0 : (l == 1) ? (i == 1 ? 1 : 0)
         : (i == 1 ? 1 : i == 2 ? 2 : i == 4 ? 1 : 0);
}
__host__ __device__ constexpr int cart_z(int l, int i) { return l - cart_x(l, i) - cart_y(l, i); }

// Shell pair data for one pair class, structure of arrays, sorted by Schwarz bound (descending).
struct PairList {
    int n;            // number of shell pairs
    int *shA, *shB;   // shell indices (l(A) >= l(B))
    int *poff, *np;   // primitive-pair offset / count
    double *Q;        // Schwarz bound sqrt(max |(ab|ab)|), true normalisation
};

// Primitive-pair data (all pair classes share one set of arrays).
struct PrimPairs {
    double *a, *b;            // exponents of the A and B primitives
    double *Px, *Py, *Pz;     // Gaussian product centre
    double *K;                // exp(-ab/p |AB|^2) * cA * cB
    double *arg;              // ab/p |AB|^2 (for the quartet cut)
    double *Kp;               // K / p: the quartet prefactor 2 pi^(5/2) K_ab K_cd / (p q sqrt(p+q)) is
                              // then 2 pi^(5/2) Kp_ab Kp_cd rsqrt(p+q), with 1/(p+q) = rsqrt^2
    double *hp;               // 1 / (2p)
    const double2 *rec;       // the same per pair packed for 16-byte loads: {p, Px}, {Py, Pz}, {Kp, hp}, {arg, a}
    const float4 *rec32;      // single precision for the FP32 quartets: {p, P-A}, {Kp, hp, arg, 0}, with A
                              // the pair's first centre (differences, so no absolute coordinate is rounded)
};

// A primitive pair's record in registers (three 16-byte loads of PrimPairs::rec).
struct PairRec {
    double p, Px, Py, Pz, Kp, hp;
};
__device__ __forceinline__ PairRec load_rec(const double2 *__restrict__ rec, int i) {
    const double2 a = __ldg(rec + 4 * i), b = __ldg(rec + 4 * i + 1), c = __ldg(rec + 4 * i + 2);
    return PairRec{a.x, a.y, b.x, b.y, c.x, c.y};
}
__device__ __forceinline__ double load_arg(const double2 *__restrict__ rec, int i) { return __ldg(rec + 4 * i + 3).x; }
// {cut argument, exponent of the pair's first primitive} in one 16-byte load (the second exponent
// is p - a).
__device__ __forceinline__ double2 load_arg_a(const double2 *__restrict__ rec, int i) { return __ldg(rec + 4 * i + 3); }

// A primitive pair's single-precision record (two 16-byte loads of PrimPairs::rec32).
struct PairRec32 {
    float p, PAx, PAy, PAz, Kp, hp, arg;
};
__device__ __forceinline__ PairRec32 load_rec32(const float4 *__restrict__ rec, int i) {
    const float4 a = __ldg(rec + 2 * i), b = __ldg(rec + 2 * i + 1);
    return PairRec32{a.x, a.y, a.z, a.w, b.x, b.y, b.z};
}

struct DeviceBasis {
    int nshell, nbf, natom;
    int *sh_l, *sh_atom, *sh_bf, *sh_np, *sh_poff;  // split shells
    double *prim_exp, *prim_coef;
    double *atom_xyz;   // natom*3, bohr
    double *atom_Z;     // nuclear charges
    double *bf_norm;    // per Cartesian function: sqrt((2l-1)!!/((2x-1)!!(2y-1)!!(2z-1)!!))
    int *bf_atom;
    int *bf_shell;      // split shell of each Cartesian function
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Primitive-pair-count buckets of a shell-pair class.  Each class list is ordered by bucket, then
// by Schwarz bound (descending) inside the bucket, and the work lists split the kets by bucket: the
// quartets next to each other in a launch (one bra pair, consecutive kets) then have the same
// number of primitive quartets, so the lanes of a warp finish together.
#define PDG_NBUCKET 5
__host__ __device__ constexpr int np_bucket(int np) { return np <= 1 ? 0 : np <= 4 ? 1 : np <= 9 ? 2 : np <= 18 ? 3 : 4; }

// One ket bucket of a (bra class, ket class) work list as a kernel sees it.
struct WorkSub {
    const long long *offs;   // prefix sums over bra pairs of their surviving kets in this bucket
    const int *cbra;         // bra pair of every fourth quartet (bra_of)
    long long total;         // quartets
    long long cta0;          // first CTA of the launch working on this bucket
    int k0;                  // first ket pair of the bucket in the ket class list
    int lanes;               // lanes per quartet (a power of two, <= 32)
};
struct WorkList {
    int nsub;
    WorkSub sub[PDG_NBUCKET];
};

// The bucket of this CTA (static indices only, so the parameter array stays in constant space).
__device__ __forceinline__ WorkSub pick_sub(const WorkList &w) {
    WorkSub s = w.sub[0];
#pragma unroll
    for (int k = 1; k < PDG_NBUCKET; ++k)
        if (k < w.nsub && (long long)blockIdx.x >= w.sub[k].cta0) s = w.sub[k];
    return s;
}

// Mask of the `lanes` lanes (a power of two) that share a quartet with the calling lane.
__device__ __forceinline__ unsigned lane_group_mask(int lanes) {
    if (lanes >= 32) return 0xffffffffu;
    return ((1u << lanes) - 1u) << ((threadIdx.x & 31) & ~(lanes - 1));
}

// Bra pair of work item t from the prefix sums offs over bra pairs and the precomputed map cbra
// (cbra[k] = bra pair of item 4k): the search runs between cbra[t/4] and cbra[t/4 + 1] only, with no
// block barrier.
__device__ __forceinline__ int bra_of(const long long *__restrict__ offs, const int *__restrict__ cbra, long long t) {
    const long long k = t >> 2;
    int lo = cbra[k], hi = cbra[k + 1] + 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (offs[mid] <= t) lo = mid; else hi = mid;
    }
    return lo;
}

