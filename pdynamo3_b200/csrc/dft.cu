// DFT grid integrator: Becke-partitioned atomic grids, basis functions on grid blocks, density,
// exchange-correlation Fock matrix and gradients (including grid-weight derivatives).
//
// Replaces the reference's grid and integrator:
//   DFTGrid_Construct / _Atom_Parameters / _Radial_Points (pMolecule/QCModel/__extensions__/csource/
//   DFTGrid.c:105-263,474-576), DFTGridWeights_Weight / _Derivatives (DFTGridWeights.c:98-215,220-258),
//   DFTIntegrator_Integrate with its Fock and gradient helpers (DFTIntegrator.c:159-1018),
//   GaussianBasisContainerIntegrals_f1Op1ir123 + GridFunctionDataBlock_FilterValues
//   (GaussianBasisContainerIntegrals_f1Op1.c:71-161, GridFunctionDataBlock.c:130).
// The point set, its order, the 128-point blocks per atom, the basis-value filter (functions whose
// largest |value| over a block is <= the accuracy's bfTolerance are dropped) and the block skip on
// max rho <= rhoTolerance follow the reference, so the quadrature is the same sum.
//
// Layout on the device: points as (x, y, z, w) quadruples; per block the list of surviving
// Cartesian functions and, resident for the whole SCF, their values and first derivatives
// [4][nfun][128] (in-core; the reference recomputes them every cycle).  Per Fock build one kernel
// forms X = D B, rho, grad rho and evaluates the functional per point; a second forms the block
// contribution B Z^T + Z B^T to V_xc.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "context.h"
#include "xc.cuh"
#include "lebedev_table.inc"

namespace {

constexpr int BLK = 128;  // points per block (DFTGrid.c:82)
constexpr double PI = 3.14159265358979323846;

// Bragg radii in angstroms (DFTGrid.c:29-40), converted with the reference's bohr radius.
const double kBragg[] = {0.75, 0.35, 0.35, 1.45, 1.05, 0.85, 0.70, 0.65, 0.60, 0.50, 0.50, 1.80, 1.50, 1.25, 1.10, 1.00,
                         1.00, 1.00, 1.00, 2.20, 1.80, 1.60, 1.40, 1.35, 1.40, 1.40, 1.40, 1.35, 1.35, 1.35, 1.35, 1.30,
                         1.25, 1.15, 1.15, 1.15, 1.15};
const double kAngToBohr = 1.0e-10 / 5.291772083e-11;
const double kBfTol[5] = {1.0e-8, 1.0e-9, 1.0e-10, 1.0e-12, 1.0e-15};
const double kRhoTol[5] = {1.0e-13, 1.0e-14, 1.0e-15, 1.0e-17, 1.0e-20};

double bragg(int z) {
    const int n = (int)(sizeof(kBragg) / sizeof(kBragg[0]));
    if (z < 0) z = 0;
    const double r = z < n ? kBragg[z] : 1.55;
    return r * kAngToBohr;
}

// Per-element radial count, Lebedev order and maximum radius (DFTGrid.c:474-523).
void atom_parameters(int acc, int z, int *nR, int *l, double *rmax) {
    switch (acc) {
        case 0: *nR = z < 11 ? 21 : z < 19 ? 42 : z < 37 ? 75 : 84; *rmax = 20.0; *l = 23; break;
        case 1: *nR = z < 11 ? 35 : z < 19 ? 70 : z < 37 ? 95 : 104; *rmax = 25.0; *l = 35; break;
        case 2: *nR = z < 11 ? 49 : z < 19 ? 88 : z < 37 ? 112 : 123; *rmax = 30.0; *l = z < 11 ? 35 : 41; break;
        case 3:
            *nR = z < 11 ? 70 : z < 19 ? 123 : z < 37 ? 130 : 155; *rmax = 35.0;
            *l = z < 11 ? 41 : z < 19 ? 47 : z < 89 ? 53 : 59;
            break;
        default: *nR = z < 11 ? 100 : z < 19 ? 125 : z < 37 ? 160 : 205; *rmax = 35.0; *l = 65; break;
    }
}

int leb_index_for_order(int l) {  // smallest tabulated order >= l
    for (int k = 0; k < LEB_NORDERS; ++k)
        if (leb_order[k] >= l) return k;
    return LEB_NORDERS - 1;
}
int leb_index_for_count(int n) {  // smallest grid with at least n points (LebedevLaikov_Angular_Momentum_Value)
    for (int k = 0; k < LEB_NORDERS; ++k)
        if (leb_count[k] >= n) return k;
    return LEB_NORDERS - 1;
}

// The partition polynomial of DFTGridWeights.c:21-35: s(nu) = 1/2 - APASC sum_t XPASC[t] nu^(2t+1).
__constant__ double c_xpasc[11] = {1.000000000000000e+00, -3.333333333333333e+00, 9.000000000000000e+00,
                                   -17.142857142857142e+00, 23.333333333333332e+00, -22.909090909090910e+00,
                                   16.153846153846153e+00, -8.000000000000000e+00, 2.647058823529412e+00,
                                   -0.526315789473684e+00, 0.047619047619048e+00};
constexpr double APASC = 1.850069046020527e+00;

// Horner form in nu^2.
__device__ __forceinline__ double pasc_sum(double nu) {
    const double nu2 = nu * nu;
    double acc = c_xpasc[10];
#pragma unroll
    for (int t = 9; t >= 0; --t) acc = fma(acc, nu2, c_xpasc[t]);
    return acc * nu;
}
__device__ __forceinline__ double pasc_s(double nu) { return 0.5 - APASC * pasc_sum(nu); }
// d/dnu of pasc_sum: sum_t XPASC[t] (2t+1) nu^(2t) = sum_t C(10,t) (-nu^2)^t = (1 - nu^2)^10.
__device__ __forceinline__ double pasc_ds(double nu) {
    const double t = 1.0 - nu * nu, t2 = t * t, t4 = t2 * t2;
    return t4 * t4 * t2;
}

constexpr double CELL_REL = 1.0e-30;  // cell functions below this fraction of the grid atom's are cut short

// Unnormalised cell function A_k(r) = prod_{j != k} s(nu_kj) at distances R[j * rs] (atoms k, j).
// Every factor has magnitude at most one (a factor at |nu| = 1 can round to a tiny negative value),
// so the product's magnitude only falls; once it is below tiny the rest of the factors are not
// formed (tiny = 0: the full product).
__device__ __forceinline__ double cell_factor(int k, int n, const double *R, int rs, const double *rinv, const double *aij,
                                              double tiny = 0.0) {
    double prod = 1.0;
    const double Rk = R[k * rs];
    for (int j = 0; j < n && !(fabs(prod) < tiny); ++j) {
        if (j == k) continue;
        const double mu = (Rk - R[j * rs]) * rinv[k * n + j];
        const double nu = mu + aij[k * n + j] * (1.0 - mu * mu);
        prod *= pasc_s(nu);
    }
    return prod;
}

// Basis function (raw Cartesian) value and derivatives up to second order at a point.
// out: 0 value, 1-3 x y z, 4-9 xx xy xz yy yz zz.
template <int ORDER>
__device__ __forceinline__ void basis_eval(const DeviceBasis &bs, int f, double px, double py, double pz, double *out) {
    const int sh = bs.bf_shell[f];
    const int l = bs.sh_l[sh];
    const int comp = f - bs.sh_bf[sh];
    int lx, ly, lz;
    if (l == 0) { lx = ly = lz = 0; }
    else if (l == 1) { lx = comp == 0; ly = comp == 1; lz = comp == 2; }
    else { lx = cart_x(2, comp); ly = cart_y(2, comp); lz = cart_z(2, comp); }
    const int at = bs.sh_atom[sh];
    const double dx = px - bs.atom_xyz[3 * at], dy = py - bs.atom_xyz[3 * at + 1], dz = pz - bs.atom_xyz[3 * at + 2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    // powers
    auto pw = [](double x, int n) { return n == 0 ? 1.0 : n == 1 ? x : n == 2 ? x * x : n == 3 ? x * x * x : x * x * x * x; };
    const double X0 = pw(dx, lx), Y0 = pw(dy, ly), Z0 = pw(dz, lz);
    const double Xm = lx >= 1 ? pw(dx, lx - 1) : 0.0, Ym = ly >= 1 ? pw(dy, ly - 1) : 0.0, Zm = lz >= 1 ? pw(dz, lz - 1) : 0.0;
    const double Xmm = lx >= 2 ? pw(dx, lx - 2) : 0.0, Ymm = ly >= 2 ? pw(dy, ly - 2) : 0.0, Zmm = lz >= 2 ? pw(dz, lz - 2) : 0.0;
    double v = 0, vx = 0, vy = 0, vz = 0, vxx = 0, vxy = 0, vxz = 0, vyy = 0, vyz = 0, vzz = 0;
    const int p0 = bs.sh_poff[sh], np = bs.sh_np[sh];
    for (int k = p0; k < p0 + np; ++k) {
        const double a = bs.prim_exp[k];
        const double ar2 = a * r2;
        if (ar2 > 740.0) continue;
        const double g = bs.prim_coef[k] * exp(-ar2);
        v += g * X0 * Y0 * Z0;
        if (ORDER >= 1) {
            const double ta = 2.0 * a;
            const double X1 = lx * Xm - ta * X0 * dx, Y1 = ly * Ym - ta * Y0 * dy, Z1 = lz * Zm - ta * Z0 * dz;
            vx += g * X1 * Y0 * Z0;
            vy += g * X0 * Y1 * Z0;
            vz += g * X0 * Y0 * Z1;
            if (ORDER >= 2) {
                const double X2 = lx * (lx - 1) * Xmm - ta * (2 * lx + 1) * X0 + ta * ta * X0 * dx * dx;
                const double Y2 = ly * (ly - 1) * Ymm - ta * (2 * ly + 1) * Y0 + ta * ta * Y0 * dy * dy;
                const double Z2 = lz * (lz - 1) * Zmm - ta * (2 * lz + 1) * Z0 + ta * ta * Z0 * dz * dz;
                vxx += g * X2 * Y0 * Z0;
                vyy += g * X0 * Y2 * Z0;
                vzz += g * X0 * Y0 * Z2;
                vxy += g * X1 * Y1 * Z0;
                vxz += g * X1 * Y0 * Z1;
                vyz += g * X0 * Y1 * Z1;
            }
        }
    }
    out[0] = v;
    if (ORDER >= 1) { out[1] = vx; out[2] = vy; out[3] = vz; }
    if (ORDER >= 2) { out[4] = vxx; out[5] = vxy; out[6] = vxz; out[7] = vyy; out[8] = vyz; out[9] = vzz; }
}

// Resident basis values [4][nfun][128] per block.
__global__ void basis_values_kernel(int nblk, const int *__restrict__ bstart, const int *__restrict__ bcount,
                                    const long long *__restrict__ foff, const int *__restrict__ fun,
                                    const long long *__restrict__ voff, const double *__restrict__ pts, DeviceBasis bs,
                                    double *__restrict__ bval) {
    const int b = blockIdx.x;
    const int p = threadIdx.x;
    const int np = bcount[b];
    const int nf = (int)(foff[b + 1] - foff[b]);
    double px = 0, py = 0, pz = 0;
    if (p < np) {
        const long long q = bstart[b] + p;
        px = pts[4 * q]; py = pts[4 * q + 1]; pz = pts[4 * q + 2];
    }
    double *V = bval + voff[b];
    for (int i = 0; i < nf; ++i) {
        double o[4] = {0, 0, 0, 0};
        if (p < np) basis_eval<1>(bs, fun[foff[b] + i], px, py, pz, o);
        V[(0 * nf + i) * BLK + p] = o[0];
        V[(1 * nf + i) * BLK + p] = o[1];
        V[(2 * nf + i) * BLK + p] = o[2];
        V[(3 * nf + i) * BLK + p] = o[3];
    }
}

struct RhoArgs {
    int nblk;
    const int *bstart, *bcount;
    const long long *foff, *voff;
    const int *fun;
    const double *pts, *bval, *D;  // D: scaled Cartesian density D' (n x n)
    int n, kind, chunk;
    double rho_tol;
    double *pcoef, *pF, *red;  // red[0] += E_xc, red[1] += integrated rho
    int *skip;
};

constexpr int XT = 256;  // threads of the XC contraction kernels

struct VxcArgs {
    const int *bcount, *bstart;
    const long long *foff, *voff;
    const int *fun;
    const double *bval, *pcoef;
    const int *skip;
    int n;
    double c0scale;  // Z = c0scale c0 B + c . grad B: 1/2 for V_xc, 0 for the gradient's Zg
    double *Z;  // scratch rows beside B: Z_mu(p) of each block at foff[b] * BLK
    double *V;  // raw Cartesian V_xc, lower triangle (row >= col) accumulated
};

// ---- FP64 tensor-core forms of the XC contractions ---------------------------------------------
// mma.sync m8n8k4 FP64 (DMMA): one instruction does an 8x8x4 block (256 FMAs) where the SIMT
// form needs 8 FFMA per lane, so the contractions stop being bound by instruction issue.
// Fragment layout (PTX ISA, m8n8k4 .f64): A (8x4, row) a0 = A[l/4][l%4]; B (4x8, col)
// b0 = B[l%4][l/4]; C (8x8) c{0,1} = C[l/4][2(l%4)+{0,1}], l = lane.
__device__ __forceinline__ void dmma_8x8x4(double &c0, double &c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

// Row strides (doubles) of the staged slices, both = 4 mod 16: in a fragment read lane (g, q) reads
// D' row g, column q, or basis row q, column g, so each half-warp's four rows land 8 banks apart
// (conflict-free), and 16-byte copies into the basis rows stay aligned.
constexpr int XS = 20, XB = 132;

// Asynchronous global -> shared copies (cp.async, sm_80+): the copy bypasses registers and is
// waited on per commit group, so the next slice streams in while the tensor cores work on this one.
// A copy whose source size is 0 writes zeros (ragged edges) and reads nothing.
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 8 : 0) : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Shared memory of the density kernel: two stages of the D' and basis slices, the per-warp-row
// partial sums, the block's function list.
struct RhoSmem {
    double Ds[2][64][XS];  // Ds[s][m][k] = D'[fun[m0+m]][fun[k0+k]]
    double Bs[2][16][XB];  // Bs[s][k][p] = B[k0+k][p]
    double part[2][4][BLK];
    double red[3][XT / 32];
    int skip_blk;
};
inline size_t rho_smem(int max_nf) { return sizeof(RhoSmem) + (size_t)std::max(1, max_nf) * sizeof(int); }

// X = D'_red B on DMMA: CTA tile 64 functions x 128 points, 8 warps as 2 x 4, warp tile 32 x 32
// (4 x 4 DMMA blocks), 16-deep slices double-buffered through cp.async; then rho = sum_mu B_mu X_mu
// and grad rho = 2 sum_mu grad B_mu X_mu (DFTIntegrator.c:814-877), the block skip, the functional
// and the per-point coefficients.
__global__ void __launch_bounds__(XT, 2) rho_xc_dmma_kernel(RhoArgs a) {
    extern __shared__ __align__(16) unsigned char rho_raw[];
    RhoSmem &S = *reinterpret_cast<RhoSmem *>(rho_raw);
    int *sfun = reinterpret_cast<int *>(rho_raw + sizeof(RhoSmem));
    const int b = blockIdx.x, t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int wm = warp >> 2, wp = warp & 3, g = lane >> 2, q = lane & 3;
    const int np = a.bcount[b];
    const int nf = (int)(a.foff[b + 1] - a.foff[b]);
    const int *fun = a.fun + a.foff[b];
    const double *B = a.bval + a.voff[b];
    const double *Bx = B + (long long)nf * BLK, *By = Bx + (long long)nf * BLK, *Bz = By + (long long)nf * BLK;
    for (int e = t; e < 8 * BLK; e += XT) (&S.part[0][0][0])[e] = 0.0;
    for (int e = t; e < nf; e += XT) sfun[e] = fun[e];
    __syncthreads();
    const int nk = (nf + 15) >> 4;
    // slice kk of the panel at row m0 into stage s: 1024 gathered D' elements (8-byte copies), 16
    // basis rows of 128 points (16-byte copies); rows past nf are zero-filled
    auto load = [&](int s, int m0, int kk) {
        const int k0 = kk << 4;
        for (int e = t; e < 16 * 64; e += XT) {
            const int m = e >> 4, k = e & 15, mu = m0 + m, nu = k0 + k;
            const bool ok = mu < nf && nu < nf;
            cp_async8(&S.Ds[s][m][k], ok ? a.D + (long long)sfun[mu] * a.n + sfun[nu] : a.D, ok);
        }
        for (int e = t; e < 16 * (BLK / 2); e += XT) {
            const int k = e >> 6, c = (e & 63) << 1;
            const bool ok = k0 + k < nf;
            cp_async16(&S.Bs[s][k][c], ok ? B + (long long)(k0 + k) * BLK + c : B, ok);
        }
        cp_async_commit();
    };
    if (nf > 0) load(0, 0, 0);
    for (int m0 = 0; m0 < nf; m0 += 64) {
        double acc[4][4][2];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
        for (int kk = 0; kk < nk; ++kk) {
            const int s = kk & 1;
            cp_async_wait_all();
            __syncthreads();  // stage s has landed for everyone; stage s^1 is no longer read
            if (kk + 1 < nk) load(s ^ 1, m0, kk + 1);
            if (m0 + wm * 32 >= nf) continue;  // this warp's rows are all padding
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const int k = 4 * ks + q;
                double av[4], bv[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) av[i] = S.Ds[s][wm * 32 + 8 * i + g][k];
#pragma unroll
                for (int j = 0; j < 4; ++j) bv[j] = S.Bs[s][k][wp * 32 + 8 * j + g];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], av[i], bv[j]);
            }
        }
        __syncthreads();  // no stage is read any more: the next panel's first slice streams in
        if (m0 + 64 < nf) load(0, m0 + 64, 0);  // under this panel's contraction below
        // this lane holds X[mu][p] for mu = m0 + 32 wm + 8 i + g and p = 32 wp + 8 j + 2 q + c
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int p = wp * 32 + 8 * j + 2 * q + c;
                double r = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int mu = m0 + wm * 32 + 8 * i + g;
                    if (mu < nf) {
                        const long long o = (long long)mu * BLK + p;
                        const double x = acc[i][j][c];
                        r += B[o] * x;
                        gx += Bx[o] * x;
                        gy += By[o] * x;
                        gz += Bz[o] * x;
                    }
                }
#pragma unroll
                for (int o = 4; o <= 16; o <<= 1) {  // over g: the 8 lanes that share q
                    r += __shfl_xor_sync(0xffffffffu, r, o);
                    gx += __shfl_xor_sync(0xffffffffu, gx, o);
                    gy += __shfl_xor_sync(0xffffffffu, gy, o);
                    gz += __shfl_xor_sync(0xffffffffu, gz, o);
                }
                if (g == 0) {  // one writer per (wm, p): deterministic order
                    S.part[wm][0][p] += r;
                    S.part[wm][1][p] += gx;
                    S.part[wm][2][p] += gy;
                    S.part[wm][3][p] += gz;
                }
            }
    }
    __syncthreads();
    const int p = t;
    double rho = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
    if (p < BLK) {
        rho = S.part[0][0][p] + S.part[1][0][p];
        gx = 2.0 * (S.part[0][1][p] + S.part[1][1][p]);
        gy = 2.0 * (S.part[0][2][p] + S.part[1][2][p]);
        gz = 2.0 * (S.part[0][3][p] + S.part[1][3][p]);
    }
    double m = (p < np) ? fabs(rho) : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) S.red[0][warp] = m;
    __syncthreads();
    if (t == 0) {
        double mm = S.red[0][0];
        for (int w = 1; w < XT / 32; ++w) mm = fmax(mm, S.red[0][w]);
        S.skip_blk = mm <= a.rho_tol;
        a.skip[b] = S.skip_blk;
    }
    __syncthreads();
    const bool skip_blk = S.skip_blk;
    double f = 0, vr = 0, vs = 0, w = 0;
    const long long qq = (long long)a.bstart[b] + p;
    if (p < np && !skip_blk) {
        w = a.pts[4 * qq + 3];
        xc::evaluate(a.kind, rho, gx * gx + gy * gy + gz * gz, &f, &vr, &vs);
    }
    if (p < np) {
        a.pcoef[4 * qq] = w * vr;
        a.pcoef[4 * qq + 1] = 2.0 * w * vs * gx;
        a.pcoef[4 * qq + 2] = 2.0 * w * vs * gy;
        a.pcoef[4 * qq + 3] = 2.0 * w * vs * gz;
        a.pF[qq] = skip_blk ? 0.0 : f;
    }
    double e = w * f, r = (skip_blk || p >= np) ? 0.0 : w * rho;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_xor_sync(0xffffffffu, e, o);
        r += __shfl_xor_sync(0xffffffffu, r, o);
    }
    if (lane == 0) { S.red[1][warp] = e; S.red[2][warp] = r; }
    __syncthreads();
    if (t == 0) {
        double es = 0, rs = 0;
        for (int k = 0; k < XT / 32; ++k) { es += S.red[1][k]; rs += S.red[2][k]; }
        atomicAdd(&a.red[0], es);
        atomicAdd(&a.red[1], rs);
    }
}

// Shared memory of the V_xc kernel: two stages of [function][point] slices (16 points, rows padded
// to 20 doubles so the fragment reads are conflict-free and 16-byte copies stay aligned) of B and Z
// for the row tile (m) and the column tile (n).
constexpr int VS = 20;
struct VxcSmem {
    double Bm[2][64][VS], Zm[2][64][VS], Bn[2][64][VS], Zn[2][64][VS];
};

// Z_mu(p) = s c0(p) B_mu(p) + c(p) . grad B_mu(p) (s = 1/2 for V_xc, 0 for the gradient) for every
// function row of every live block, into
// scratch rows beside B (one CTA per block; B, and so Z, is zero at the padding points p >= np).
__global__ void __launch_bounds__(XT) xc_z_kernel(VxcArgs a) {
    const int b = blockIdx.x;
    if (a.skip[b]) return;
    __shared__ double coef[4][BLK];
    const int nf = (int)(a.foff[b + 1] - a.foff[b]);
    const int np = a.bcount[b];
    const double *B = a.bval + a.voff[b];
    const double *Bx = B + (long long)nf * BLK, *By = Bx + (long long)nf * BLK, *Bz = By + (long long)nf * BLK;
    double *Z = a.Z + a.foff[b] * BLK;
    for (int e = threadIdx.x; e < 4 * BLK; e += XT) {
        const int k = e / BLK, p = e - k * BLK;
        coef[k][p] = p < np ? a.pcoef[4 * ((long long)a.bstart[b] + p) + k] : 0.0;
    }
    __syncthreads();
#pragma unroll 4
    for (int e = threadIdx.x; e < nf * BLK; e += XT) {
        const int p = e & (BLK - 1);
        Z[e] = a.c0scale * coef[0][p] * B[e] + coef[1][p] * Bx[e] + coef[2][p] * By[e] + coef[3][p] * Bz[e];
    }
}

// V_red = B Z^T + Z B^T on DMMA with Z_mu(p) = 1/2 c0 B_mu + c . grad B_mu (DFTIntegrator.c:515-621)
// from xc_z_kernel: the lower-triangle 64 x 64 tiles run over 16-point slices of B and Z, double-buffered through
// cp.async across tile boundaries; 8 warps as 2 x 4, warp tile 32 x 16 (4 x 2 DMMA blocks, two
// products each).
__global__ void __launch_bounds__(XT, 2) vxc_dmma_kernel(VxcArgs a) {
    const int b = blockIdx.x;
    if (a.skip[b]) return;
    extern __shared__ __align__(16) unsigned char vxc_raw[];
    VxcSmem &S = *reinterpret_cast<VxcSmem *>(vxc_raw);
    const int nf = (int)(a.foff[b + 1] - a.foff[b]);
    const int np = a.bcount[b];
    const int *fun = a.fun + a.foff[b];
    const double *B = a.bval + a.voff[b];
    const double *Z = a.Z + a.foff[b] * BLK;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int wm = warp >> 2, wn = warp & 3, g = lane >> 2, q = lane & 3;
    const int ntile = (nf + 63) >> 6, nk = (np + 15) >> 4;
    if (ntile == 0 || nk == 0) return;
    auto load = [&](int s, int ti, int tj, int kk) {
        const int p0 = kk << 4;
        for (int e = t; e < 64 * 8; e += XT) {
            const int r = e >> 3, c = (e & 7) << 1;
            const int mu = ti * 64 + r;
            const bool okm = mu < nf;
            const long long om = okm ? (long long)mu * BLK + p0 + c : 0;
            cp_async16(&S.Bm[s][r][c], B + om, okm);
            cp_async16(&S.Zm[s][r][c], Z + om, okm);
            if (ti != tj) {
                const int nu = tj * 64 + r;
                const bool okn = nu < nf;
                const long long on = okn ? (long long)nu * BLK + p0 + c : 0;
                cp_async16(&S.Bn[s][r][c], B + on, okn);
                cp_async16(&S.Zn[s][r][c], Z + on, okn);
            }
        }
        cp_async_commit();
    };
    // (tile pair, slice) steps in order: pairs (ti, tj <= ti) row by row, nk slices each
    const int total = ntile * (ntile + 1) / 2 * nk;
    int ti = 0, tj = 0, kk = 0;       // step being computed
    int pi = 0, pj = 0, pk = 0;       // step being prefetched
    auto advance = [&](int &i, int &j, int &k) {
        if (++k == nk) { k = 0; if (++j > i) { ++i; j = 0; } }
    };
    load(0, 0, 0, 0);
    advance(pi, pj, pk);
    double acc[4][2][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    for (int step = 0; step < total; ++step) {
        const int s = step & 1;
        cp_async_wait_all();
        __syncthreads();  // stage s has landed for everyone; stage s^1 is no longer read
        if (step + 1 < total) { load(s ^ 1, pi, pj, pk); advance(pi, pj, pk); }
        const bool diag = ti == tj;
        const double(*Bn)[VS] = diag ? S.Bm[s] : S.Bn[s];
        const double(*Zn)[VS] = diag ? S.Zm[s] : S.Zn[s];
        // a warp whose rows or columns are all padding, or whose sub-tile lies above the diagonal of
        // a diagonal tile, has no lower-triangle entry to form
        const bool work = ti * 64 + wm * 32 < nf && tj * 64 + wn * 16 < nf && !(diag && wn * 16 > wm * 32 + 31);
#pragma unroll
        for (int ks = 0; ks < 4 && work; ++ks) {
            const int k = 4 * ks + q;
            double bmv[4], zmv[4], bnv[2], znv[2];
#pragma unroll
            for (int i = 0; i < 4; ++i) { bmv[i] = S.Bm[s][wm * 32 + 8 * i + g][k]; zmv[i] = S.Zm[s][wm * 32 + 8 * i + g][k]; }
#pragma unroll
            for (int j = 0; j < 2; ++j) { bnv[j] = Bn[wn * 16 + 8 * j + g][k]; znv[j] = Zn[wn * 16 + 8 * j + g][k]; }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    dmma_8x8x4(acc[i][j][0], acc[i][j][1], bmv[i], znv[j]);
                    dmma_8x8x4(acc[i][j][0], acc[i][j][1], zmv[i], bnv[j]);
                }
        }
        if (kk == nk - 1 && work) {  // tile pair done: lower-triangle entries to V
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int mu = ti * 64 + wm * 32 + 8 * i + g;
#pragma unroll
                for (int j = 0; j < 2; ++j)
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        const int nu = tj * 64 + wn * 16 + 8 * j + 2 * q + c;
                        if (mu < nf && nu < nf && nu <= mu) atomicAdd(&a.V[(long long)fun[mu] * a.n + fun[nu]], acc[i][j][c]);
                        acc[i][j][c] = 0.0;
                    }
            }
        }
        advance(ti, tj, kk);
    }
}

// V (lower triangle raw) -> F_true += N (V + V^T - diag) N ; also returns tr(D' V) pieces.
__global__ void vxc_finish_kernel(int n, const double *__restrict__ V, const double *__restrict__ norm,
                                  const double *__restrict__ Ds, double *__restrict__ F, double *__restrict__ trace) {
    const int i = blockIdx.y;
    double s = 0.0;
    for (int j = threadIdx.x + blockIdx.x * blockDim.x; j < n; j += blockDim.x * gridDim.x) {
        const double v = i >= j ? V[(long long)i * n + j] : V[(long long)j * n + i];
        F[(long long)i * n + j] += v * norm[i] * norm[j];
        s += Ds[(long long)i * n + j] * v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(trace, s);
}

struct GradArgs {
    const int *bstart, *bcount, *batom;
    const long long *foff, *voff;
    const int *fun;
    const double *pts, *bval, *pcoef, *D;
    const double *Z;  // Zg rows of each block at foff[b] * BLK
    const int *skip;
    DeviceBasis bs;
    int n, chunk;
    double *grad;
};

// Shared memory of the XC-gradient kernel: two stages of the D' slice and of the basis and Zg
// slices, the block's points and coefficients, per-warp-column partial gradients of the panel's
// functions, the block's function list.
struct XcGradSmem {
    double Ds[2][64][XS];
    double Bs[2][16][XB];  // B[k0+k][p]
    double Ws[2][16][XB];  // Zg[k0+k][p] = c(p) . grad B[k0+k](p)
    double pt[3][BLK], cf[4][BLK];
    double gpart[4][64][3];
};
inline size_t xcgrad_smem(int max_nf) { return sizeof(XcGradSmem) + (size_t)std::max(1, max_nf) * sizeof(int); }

// Basis-function part of the XC gradient (DFTIntegrator_Gradients / _GradientsSigma and
// UGradientContributions, DFTIntegrator.c:643-809,909-940): for each function mu on atom c,
// g_mu = sum_p [2 X (a grad phi + sum_b c_b grad d_b phi) + 2 W grad phi]_mu(p) with X = D' B and
// W = D' Zg (Zg = c . grad B, from xc_z_kernel); the gradient of c decreases by g_mu and that of the
// block's grid atom increases by g_mu.  X and W are one DMMA pass (CTA tile 64 functions x 128
// points, 8 warps as 2 x 4, warp tile 32 x 32 of each), slices double-buffered through cp.async as in
// the density kernel; the second derivatives of the basis are evaluated in the epilogue.
__global__ void __launch_bounds__(XT, 1) xc_grad_dmma_kernel(GradArgs a) {
    const int b = blockIdx.x;
    if (a.skip[b]) return;
    extern __shared__ __align__(16) unsigned char xg_raw[];
    XcGradSmem &S = *reinterpret_cast<XcGradSmem *>(xg_raw);
    int *sfun = reinterpret_cast<int *>(xg_raw + sizeof(XcGradSmem));
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    const int wm = warp >> 2, wp = warp & 3, g = lane >> 2, q = lane & 3;
    const int np = a.bcount[b];
    const int nf = (int)(a.foff[b + 1] - a.foff[b]);
    const int gatom = a.batom[b];
    const int *fun = a.fun + a.foff[b];
    const double *B = a.bval + a.voff[b];
    const double *Bx = B + (long long)nf * BLK, *By = Bx + (long long)nf * BLK, *Bz = By + (long long)nf * BLK;
    const double *Zg = a.Z + a.foff[b] * BLK;
    for (int e = t; e < BLK; e += XT) {
        const long long qq = (long long)a.bstart[b] + e;
        const bool ok = e < np;
        S.pt[0][e] = ok ? a.pts[4 * qq] : 0.0;
        S.pt[1][e] = ok ? a.pts[4 * qq + 1] : 0.0;
        S.pt[2][e] = ok ? a.pts[4 * qq + 2] : 0.0;
        for (int k = 0; k < 4; ++k) S.cf[k][e] = ok ? a.pcoef[4 * qq + k] : 0.0;
    }
    for (int e = t; e < nf; e += XT) sfun[e] = fun[e];
    __syncthreads();
    const int nk = (nf + 15) >> 4;
    auto load = [&](int s, int m0, int kk) {
        const int k0 = kk << 4;
        for (int e = t; e < 16 * 64; e += XT) {
            const int m = e >> 4, k = e & 15, mu = m0 + m, nu = k0 + k;
            const bool ok = mu < nf && nu < nf;
            cp_async8(&S.Ds[s][m][k], ok ? a.D + (long long)sfun[mu] * a.n + sfun[nu] : a.D, ok);
        }
        for (int e = t; e < 16 * (BLK / 2); e += XT) {
            const int k = e >> 6, c = (e & 63) << 1;
            const bool ok = k0 + k < nf;
            const long long o = ok ? (long long)(k0 + k) * BLK + c : 0;
            cp_async16(&S.Bs[s][k][c], B + o, ok);
            cp_async16(&S.Ws[s][k][c], Zg + o, ok);
        }
        cp_async_commit();
    };
    if (nf > 0) load(0, 0, 0);
    for (int m0 = 0; m0 < nf; m0 += 64) {
        double ax[4][4][2], aw[4][4][2];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) ax[i][j][0] = ax[i][j][1] = aw[i][j][0] = aw[i][j][1] = 0.0;
        const bool rows = m0 + wm * 32 < nf;  // this warp has a function row in the panel
        for (int kk = 0; kk < nk; ++kk) {
            const int s = kk & 1;
            cp_async_wait_all();
            __syncthreads();
            if (kk + 1 < nk) load(s ^ 1, m0, kk + 1);
            if (!rows) continue;
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const int k = 4 * ks + q;
                double av[4], bv[4], wv[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) av[i] = S.Ds[s][wm * 32 + 8 * i + g][k];
#pragma unroll
                for (int j = 0; j < 4; ++j) { bv[j] = S.Bs[s][k][wp * 32 + 8 * j + g]; wv[j] = S.Ws[s][k][wp * 32 + 8 * j + g]; }
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        dmma_8x8x4(ax[i][j][0], ax[i][j][1], av[i], bv[j]);
                        dmma_8x8x4(aw[i][j][0], aw[i][j][1], av[i], wv[j]);
                    }
            }
        }
        __syncthreads();  // no stage is read any more: the next panel's first slice streams in
        if (m0 + 64 < nf) load(0, m0 + 64, 0);
        // this lane holds X, W [mu][p] for mu = m0 + 32 wm + 8 i + g, p = 32 wp + 8 j + 2 q + c; the W
        // terms first (they need only the stored gradient), so W's registers are free for the
        // second-derivative evaluations of the X terms
        double gs[4][3];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            gs[i][0] = gs[i][1] = gs[i][2] = 0.0;
            const int mu = m0 + wm * 32 + 8 * i + g;
            if (mu >= nf) continue;
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const int p = wp * 32 + 8 * j + 2 * q + c;
                    const long long o = (long long)mu * BLK + p;
                    const double W = aw[i][j][c];
                    gs[i][0] += Bx[o] * W; gs[i][1] += By[o] * W; gs[i][2] += Bz[o] * W;
                }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int mu = m0 + wm * 32 + 8 * i + g;
            if (mu >= nf) continue;
            const int f = sfun[mu];
#pragma unroll
            for (int jc = 0; jc < 8; ++jc) {
                const int j = jc >> 1, c = jc & 1;
                const int p = wp * 32 + 8 * j + 2 * q + c;
                if (p >= np) continue;
                const double X = ax[i][j][c];
                const double ca = S.cf[0][p], cx = S.cf[1][p], cy = S.cf[2][p], cz = S.cf[3][p];
                double h[10];
                basis_eval<2>(a.bs, f, S.pt[0][p], S.pt[1][p], S.pt[2][p], h);
                gs[i][0] += (ca * h[1] + cx * h[4] + cy * h[5] + cz * h[6]) * X;
                gs[i][1] += (ca * h[2] + cx * h[5] + cy * h[7] + cz * h[8]) * X;
                gs[i][2] += (ca * h[3] + cx * h[6] + cy * h[8] + cz * h[9]) * X;
            }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {  // over q: the 4 lanes that share (i, g)
                gs[i][d] += __shfl_xor_sync(0xffffffffu, gs[i][d], 1);
                gs[i][d] += __shfl_xor_sync(0xffffffffu, gs[i][d], 2);
            }
            if (q == 0) {
                const int r = wm * 32 + 8 * i + g;
                S.gpart[wp][r][0] = gs[i][0]; S.gpart[wp][r][1] = gs[i][1]; S.gpart[wp][r][2] = gs[i][2];
            }
        }
        __syncthreads();
        if (t < 64 && m0 + t < nf) {
            double gx = 0.0, gy = 0.0, gz = 0.0;
            for (int w = 0; w < 4; ++w) { gx += S.gpart[w][t][0]; gy += S.gpart[w][t][1]; gz += S.gpart[w][t][2]; }
            gx *= 2.0; gy *= 2.0; gz *= 2.0;
            const int c = a.bs.bf_atom[sfun[m0 + t]];
            if (c != gatom && (gx != 0.0 || gy != 0.0 || gz != 0.0)) {
                atomicAdd(&a.grad[3 * c], -gx); atomicAdd(&a.grad[3 * c + 1], -gy); atomicAdd(&a.grad[3 * c + 2], -gz);
                atomicAdd(&a.grad[3 * gatom], gx); atomicAdd(&a.grad[3 * gatom + 1], gy); atomicAdd(&a.grad[3 * gatom + 2], gz);
            }
        }
        // gpart is rewritten only after the next panel's k loop, whose barriers order it after this read
    }
}

// Grid-weight derivative term (DFTGridWeights_Derivatives, DFTGridWeights.c:98-215), one thread per
// point.  The point's atom distances live in shared memory, one column per thread ([atom][thread],
// conflict-free), so the atoms^2 pair loops read no local memory.  Pass 1 forms each cell function
// A_i = prod_j s_ij as its smallest factor times the product of the rest; since d A_i / d mu_ij =
// (prod_{k != i,j} s_ik) ds_ij and that product never exceeds the rest-product, a row i whose
// rest-product x max|ds| x |fac_i| is below WG_TINY contributes nothing above WG_TINY and is skipped
// by the whole warp.  For the rows kept, the i and g parts are kept in registers, the j part is
// summed over the warp with shuffles and added once per warp to a per-block shared array, which is
// flushed with one global atomic per atom.
__device__ __forceinline__ double warp_allsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

constexpr double WG_TINY = 1.0e-18;
constexpr double WG_DSMAX = 2.0 * APASC;  // max |ds/dmu| = APASC (1-nu^2)^10 |1 - 2 a mu| with |a|, |mu| <= 1/2, 1

// threads per block of the weight-gradient kernel: 128 (one grid block) while the distance columns
// fit in shared memory, else 64 (the grid block in two halves)
inline int wg_threads(int natom) { return natom <= 200 ? 128 : 64; }
inline size_t wg_smem(int natom) { return (size_t)(6 + wg_threads(natom)) * natom * sizeof(double); }

__global__ void __launch_bounds__(128) weight_grad_kernel(const int *__restrict__ bstart, const int *__restrict__ bcount,
                                                          const int *__restrict__ batom, const int *__restrict__ skip,
                                                          const double *__restrict__ pts, const double *__restrict__ pF,
                                                          int natom, const double *__restrict__ xyz,
                                                          const double *__restrict__ rinv, const double *__restrict__ aij,
                                                          double *__restrict__ grad) {
    extern __shared__ double wsh[];  // gradient 3*natom | coordinates 3*natom | distances natom*tpb
    const int tpb = blockDim.x;
    double *gsh = wsh, *sxyz = wsh + 3 * natom, *sR = wsh + 6 * natom;
    const int b = blockIdx.x, p = threadIdx.x, lane = p & 31;
    for (int e = p; e < 3 * natom; e += tpb) { gsh[e] = 0.0; sxyz[e] = xyz[e]; }
    __syncthreads();
    const int np = bcount[b];
    const int g = batom[b];
    double *Rp = sR + p;  // this thread's column: Rp[i * tpb] (private, so no block barriers below)
    for (int base = 0; !skip[b] && base < np; base += tpb) {
        if (base + (p & ~31) >= np) break;  // the whole warp is past the end of the block
        const bool active = base + p < np;
        const long long q = (long long)bstart[b] + (active ? base + p : 0);
        const double gx = pts[4 * q], gy = pts[4 * q + 1], gz = pts[4 * q + 2], w = pts[4 * q + 3];
        const double ef = active ? pF[q] : 0.0;
        for (int i = 0; i < natom; ++i) {
            const double dx = sxyz[3 * i] - gx, dy = sxyz[3 * i + 1] - gy, dz = sxyz[3 * i + 2] - gz;
            Rp[i * tpb] = sqrt(dx * dx + dy * dy + dz * dz);
        }
        // pass 1: A_i = smin_i * srest_i, smin_i the smallest factor of the row
        double smin[256], srest[256];
        // the grid atom's row first; another row's rest-product (which only falls) is formed down to
        // 1e-30 A_g: below that the row changes the sum by less than 1e-30 A_g and is dead in pass 2
        // (rest x |fac| <= 1e-30 A_g x ef w / A_g), and its stored rest-product bounds the true one
        double sum = 0.0, ag = 0.0, tiny = 0.0;
        for (int ii = -1; ii < natom; ++ii) {
            const int i = ii < 0 ? g : ii;
            if (ii >= 0 && i == g) continue;
            const double Ri = Rp[i * tpb];
            const double *ri = rinv + (size_t)i * natom, *ai = aij + (size_t)i * natom;
            double mn = 1.0, rest = 1.0;
            for (int j = 0; j < natom && !(fabs(rest) < tiny); ++j) {
                if (j == i) continue;
                const double mu = (Ri - Rp[j * tpb]) * ri[j];
                const double s = pasc_s(mu + ai[j] * (1.0 - mu * mu));
                if (s < mn) { rest *= mn; mn = s; } else rest *= s;
            }
            smin[i] = mn; srest[i] = rest;
            const double A = mn * rest;
            sum += A;
            if (ii < 0) { ag = A; tiny = CELL_REL * A; }
        }
        const double pg = ag / sum;
        const bool live = active && ef != 0.0 && pg > 0.0;
        if (!__any_sync(0xffffffffu, live)) continue;
        const double ew = live ? ef * w / (pg * sum) : 0.0;
        double ggx = 0.0, ggy = 0.0, ggz = 0.0;
        for (int i = 0; i < natom; ++i) {
            const double fac = (i == g) ? ew * (1.0 - pg) : -ew * pg;
            const double mn = smin[i], rest = srest[i];
            const bool rowlive = live && rest * WG_DSMAX * fabs(fac) > WG_TINY;
            if (!__any_sync(0xffffffffu, rowlive)) continue;
            const double Ri = Rp[i * tpb], iRi = 1.0 / Ri;
            const double xi = sxyz[3 * i], yi = sxyz[3 * i + 1], zi = sxyz[3 * i + 2];
            const double *ri = rinv + (size_t)i * natom, *ai = aij + (size_t)i * natom;
            double gix = 0.0, giy = 0.0, giz = 0.0;
            for (int j = 0; j < natom; ++j) {
                if (j == i) continue;
                double ifac = 0.0, rij = 0.0, mu = 0.0, Rj = 0.0;
                bool sig = false;
                if (rowlive) {
                    rij = ri[j];
                    Rj = Rp[j * tpb];
                    mu = (Ri - Rj) * rij;
                    const double aa = ai[j];
                    const double nu = mu + aa * (1.0 - mu * mu);
                    const double dsij = -APASC * pasc_ds(nu) * (1.0 - 2.0 * aa * mu);
                    const double dsf = dsij * fac;
                    // prod_{k != i,j} s_ik: the rest-product when s_ij is the smallest factor (or ties
                    // it), else rest * smin / s_ij (s_ij > smin >= 0 and a factor of the rest)
                    if (fabs(dsf) * rest > WG_TINY) {
                        const double s = pasc_s(nu);
                        ifac = (s == mn ? rest : rest * (mn / s)) * dsf;
                        sig = fabs(ifac) > WG_TINY;
                    }
                }
                if (!__any_sync(0xffffffffu, sig)) continue;  // the whole warp's terms are negligible
                double dxj = 0.0, dyj = 0.0, dzj = 0.0;
                if (sig) {
                    const double xj = sxyz[3 * j], yj = sxyz[3 * j + 1], zj = sxyz[3 * j + 2];
                    const double fi = rij * iRi, fj = rij / Rj;
                    double dxi = (xi - gx) * fi, dyi = (yi - gy) * fi, dzi = (zi - gz) * fi;
                    dxj = -(xj - gx) * fj; dyj = -(yj - gy) * fj; dzj = -(zj - gz) * fj;
                    const double dxg = -(dxi + dxj), dyg = -(dyi + dyj), dzg = -(dzi + dzj);
                    const double m2 = mu * rij * rij;
                    const double tx = (xi - xj) * m2, ty = (yi - yj) * m2, tz = (zi - zj) * m2;
                    dxi -= tx; dyi -= ty; dzi -= tz;
                    dxj += tx; dyj += ty; dzj += tz;
                    gix += ifac * dxi; giy += ifac * dyi; giz += ifac * dzi;
                    ggx += ifac * dxg; ggy += ifac * dyg; ggz += ifac * dzg;
                } else {
                    ifac = 0.0;
                }
                const double cx = warp_allsum(ifac * dxj), cy = warp_allsum(ifac * dyj), cz = warp_allsum(ifac * dzj);
                if (lane == 0 && (cx != 0.0 || cy != 0.0 || cz != 0.0)) {
                    atomicAdd(&gsh[3 * j], cx); atomicAdd(&gsh[3 * j + 1], cy); atomicAdd(&gsh[3 * j + 2], cz);
                }
            }
            gix = warp_allsum(gix); giy = warp_allsum(giy); giz = warp_allsum(giz);
            if (lane == 0) { atomicAdd(&gsh[3 * i], gix); atomicAdd(&gsh[3 * i + 1], giy); atomicAdd(&gsh[3 * i + 2], giz); }
        }
        ggx = warp_allsum(ggx); ggy = warp_allsum(ggy); ggz = warp_allsum(ggz);
        if (lane == 0) { atomicAdd(&gsh[3 * g], ggx); atomicAdd(&gsh[3 * g + 1], ggy); atomicAdd(&gsh[3 * g + 2], ggz); }
    }
    __syncthreads();
    for (int e = p; e < 3 * natom; e += tpb)
        if (gsh[e] != 0.0) atomicAdd(&grad[e], gsh[e]);
}

__global__ void xc_eval_kernel(int kind, int n, const double *rho, const double *sigma, double *f, double *vr, double *vs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) xc::evaluate(kind, rho[i], sigma[i], &f[i], &vr[i], &vs[i]);
}

template <typename T>
int pupload(pdg_context *ctx, const char *name, T **dst, const std::vector<T> &src) {
    *dst = (T *)pdg_pool(ctx, name, std::max<size_t>(1, src.size()) * sizeof(T));
    if (!*dst) { pdg_set_error("device allocation failed (%s)", name); return PDG_ERR_ALLOC; }
    if (!src.empty()) PDG_CUDA(cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    return PDG_OK;
}

}  // namespace

struct GridData {
    long long npts = 0;
    int nblk = 0, max_nf = 0;
    double bf_tol = 0, rho_tol = 0;
    double *pts = nullptr;
    int *bstart = nullptr, *bcount = nullptr, *batom = nullptr, *fun = nullptr, *skip = nullptr;
    long long *foff = nullptr, *voff = nullptr;
    double *bval = nullptr;
    double *rinv = nullptr, *aij = nullptr;
    long long nfun_total = 0;
    std::vector<long long> h_foff;  // host copies for work accounting
    std::vector<int> h_bcount;
    // device arrays are borrowed from the context's buffer pool and outlive the grid
};

struct XCData {
    int kind = 0;
    double cx = 1.0;
    int accuracy = 3, nr = 0, lq = 0;
    double *pcoef = nullptr, *pF = nullptr, *V = nullptr, *red = nullptr;
    long long cap = 0;
    double last_vxc_trace = 0.0;
    bool have_coef = false;
    // the buffers are the context's pool buffers ("xc.*"), released with the context
};

void pdg_free_dft(pdg_context *ctx) {
    delete ctx->grid;
    ctx->grid = nullptr;
    if (ctx->xc) ctx->xc->have_coef = false;
}

// Host state of the DFT path at context destruction (its device buffers are pool buffers).
void pdg_release_dft(pdg_context *ctx) {
    delete ctx->grid;
    ctx->grid = nullptr;
    delete ctx->xc;
    ctx->xc = nullptr;
}

bool pdg_dft_active(const pdg_context *ctx) { return ctx->xc != nullptr && ctx->xc->kind != xc::NONE; }
double pdg_dft_exchange_scaling(const pdg_context *ctx) { return ctx->xc ? ctx->xc->cx : 1.0; }
double pdg_dft_last_vxc_trace(const pdg_context *ctx) { return ctx->xc ? ctx->xc->last_vxc_trace : 0.0; }

static int functional_kind(const char *name, int *kind, double *cx) {
    std::string s(name);
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    if (s == "hf") { *kind = xc::NONE; *cx = 1.0; }
    else if (s == "pbe") { *kind = xc::PBE; *cx = 0.0; }
    else if (s == "blyp") { *kind = xc::BLYP; *cx = 0.0; }
    else if (s == "b3lyp") { *kind = xc::B3LYP; *cx = 0.2; }
    else return PDG_ERR_UNSUPPORTED;
    return PDG_OK;
}

// Functional kind of a name accepted by the point-evaluation entry points: the combinations of
// pdg_set_functional ("hf" evaluates to zero) and the single terms.
int pdg_xc_kind(const char *name, int *kind) {
    std::string s(name);
    for (auto &c : s) c = (char)std::tolower((unsigned char)c);
    const char *single[] = {"lda_x", "pw92", "vwn_rpa", "lyp", "b88", "pbe_x", "pbe_c"};
    const int skind[] = {xc::LDA_X_ONLY, xc::PW92_ONLY, xc::VWNRPA_ONLY, xc::LYP_ONLY, xc::B88_ONLY, xc::PBEX_ONLY, xc::PBEC_ONLY};
    for (int k = 0; k < 7; ++k)
        if (s == single[k]) { *kind = skind[k]; return PDG_OK; }
    double cx;
    return functional_kind(name, kind, &cx);
}

extern "C" int pdg_set_functional(pdg_context *ctx, const char *name, double *cx) {
    if (!ctx || !name) { pdg_set_error("pdg_set_functional: invalid argument"); return PDG_ERR_ARG; }
    int kind;
    double c;
    if (functional_kind(name, &kind, &c) != PDG_OK) {
        pdg_set_error("pdg_set_functional: functional '%s' is not implemented (hf, pbe, blyp, b3lyp)", name);
        return PDG_ERR_UNSUPPORTED;
    }
    if (!ctx->xc) ctx->xc = new XCData();
    ctx->xc->kind = kind;
    ctx->xc->cx = c;
    ctx->xc->have_coef = false;
    if (cx) *cx = c;
    return PDG_OK;
}

extern "C" int pdg_xc_evaluate(const char *name, int n, const double *rho, const double *sigma, double *f, double *vrho,
                               double *vsigma) {
    if (!name || n < 0 || (n > 0 && (!rho || !sigma || !f || !vrho || !vsigma))) {
        pdg_set_error("pdg_xc_evaluate: invalid argument");
        return PDG_ERR_ARG;
    }
    int kind;
    if (pdg_xc_kind(name, &kind) != PDG_OK) {
        pdg_set_error("pdg_xc_evaluate: unknown functional '%s'", name);
        return PDG_ERR_UNSUPPORTED;
    }
    if (n == 0) return PDG_OK;
    double *d = nullptr;
    PDG_CUDA(cudaMalloc(&d, 5 * (size_t)n * sizeof(double)));
    cudaMemcpy(d, rho, n * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(d + n, sigma, n * sizeof(double), cudaMemcpyHostToDevice);
    { xc_eval_kernel<<<(n + 127) / 128, 128>>>(kind, n, d, d + n, d + 2 * n, d + 3 * n, d + 4 * n); pdg_count_launch(); }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(f, d + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(vrho, d + 3 * n, n * sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(vsigma, d + 4 * n, n * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) { pdg_set_error("pdg_xc_evaluate: %s", cudaGetErrorString(e)); return PDG_ERR_CUDA; }
    return PDG_OK;
}

// Radius beyond which every primitive combination of a shell stays below tol (value bound).
// ---- device grid construction ----------------------------------------------------------------
// Candidates in the reference order (atom, radial shell, Lebedev point) are generated and weighted
// on the device from a small table of radial shells; the kept points (|w| > 1e-30) are compacted
// in order, so each atom's points stay contiguous; each 128-point block then screens the split
// shells by distance and its functions by their largest value on the block's points.

// One candidate per thread: its shell by binary search over the shell offsets, the point from
// the shell's Lebedev rule and its Becke-style partition weight (DFTGridWeights_Weight,
// DFTGridWeights.c:220-258: size-adjusted cell functions of all atoms, normalised).
__global__ void grid_candidates_kernel(long long ncand, int nrs, const long long *__restrict__ rs_off,
                                       const int *__restrict__ rs_atom, const int *__restrict__ rs_leb,
                                       const double *__restrict__ rs_r, const double *__restrict__ rs_w,
                                       const double *__restrict__ leb, const int *__restrict__ leb_off, int natom,
                                       const double *__restrict__ xyz, const double *__restrict__ rinv,
                                       const double *__restrict__ aij, double *__restrict__ cand, int *__restrict__ flag) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= ncand) return;
    int lo = 0, hi = nrs;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (rs_off[mid] <= t) lo = mid; else hi = mid;
    }
    const int s = lo, g = rs_atom[s];
    const double *L = leb + 4 * ((long long)leb_off[rs_leb[s]] + (t - rs_off[s]));
    const double r = rs_r[s];
    const double px = L[0] * r + xyz[3 * g], py = L[1] * r + xyz[3 * g + 1], pz = L[2] * r + xyz[3 * g + 2];
    const double wraw = rs_w[s] * L[3];
    extern __shared__ double cR[];  // distances, one column per thread ([atom][thread])
    const int rs = blockDim.x;
    double *R = cR + threadIdx.x;
    for (int i = 0; i < natom; ++i) {
        const double dx = xyz[3 * i] - px, dy = xyz[3 * i + 1] - py, dz = xyz[3 * i + 2] - pz;
        R[i * rs] = sqrt(dx * dx + dy * dy + dz * dz);
    }
    // the grid atom's cell function first; another atom's is only formed down to 1e-30 of it, which
    // changes the partition sum by less than 1e-28 of the weight's numerator
    const double pg = cell_factor(g, natom, R, rs, rinv, aij);
    double sum = pg;
    for (int k = 0; k < natom; ++k)
        if (k != g) sum += cell_factor(k, natom, R, rs, rinv, aij, CELL_REL * pg);
    const double w = wraw * (pg / sum);
    cand[4 * t] = px; cand[4 * t + 1] = py; cand[4 * t + 2] = pz; cand[4 * t + 3] = w;
    flag[t] = fabs(w) > 1.0e-30 ? 1 : 0;
}

// Exclusive prefix sums of the keep flags, three passes: per-1024 block sums, their scan in one
// block, then the in-block scan plus the block's offset.
constexpr int SCAN_B = 1024;
__global__ void scan_block_sums_kernel(long long n, const int *__restrict__ flag, int *__restrict__ bsum) {
    __shared__ int sh[32];
    const long long i = blockIdx.x * (long long)SCAN_B + threadIdx.x;
    int v = i < n ? flag[i] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int w = 0; w < SCAN_B / 32; ++w) s += sh[w];
        bsum[blockIdx.x] = s;
    }
}
__global__ void scan_offsets_kernel(int nb, int *__restrict__ bsum) {  // one thread: nb is small
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int s = 0;
    for (int b = 0; b < nb; ++b) { const int v = bsum[b]; bsum[b] = s; s += v; }
    bsum[nb] = s;
}
__global__ void scan_final_kernel(long long n, const int *__restrict__ flag, const int *__restrict__ boff, int *__restrict__ pos) {
    __shared__ int warp_tot[SCAN_B / 32];
    const long long i = blockIdx.x * (long long)SCAN_B + threadIdx.x;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int f = i < n ? flag[i] : 0;
    int v = f;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) warp_tot[w] = v;
    __syncthreads();
    if (w == 0) {
        int x = lane < SCAN_B / 32 ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += u;
        }
        if (lane < SCAN_B / 32) warp_tot[lane] = x;
    }
    __syncthreads();
    if (i < n) pos[i] = boff[blockIdx.x] + (w ? warp_tot[w - 1] : 0) + v - f;
}

__global__ void grid_compact_kernel(long long ncand, const double *__restrict__ cand, const int *__restrict__ flag,
                                    const int *__restrict__ pos, double *__restrict__ pts) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= ncand || !flag[t]) return;
    const long long q = pos[t];
    pts[4 * q] = cand[4 * t]; pts[4 * q + 1] = cand[4 * t + 1];
    pts[4 * q + 2] = cand[4 * t + 2]; pts[4 * q + 3] = cand[4 * t + 3];
}

// Kept-point index at each atom's first candidate (and the total at the end).
__global__ void gather_atom_pos_kernel(int natom, const long long *__restrict__ aoff, long long ncand,
                                       const int *__restrict__ pos, const int *__restrict__ flag, int *__restrict__ out) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a > natom) return;
    const int total = ncand > 0 ? pos[ncand - 1] + flag[ncand - 1] : 0;
    out[a] = (a < natom && aoff[a] < ncand) ? pos[aoff[a]] : total;
}

// Per block: centroid and radius of its points, distance screen of every split shell, and for the
// surviving shells the largest |phi| of each function over the points; mask[b][f] = 1 above the
// reference's value tolerance (GridFunctionDataBlock_FilterValues, GridFunctionDataBlock.c:130).
__global__ void __launch_bounds__(BLK) block_screen_kernel(int nblk, const int *__restrict__ bstart,
                                                           const int *__restrict__ bcount, const double *__restrict__ pts,
                                                           const double *__restrict__ shell_rad, DeviceBasis bs,
                                                           double bf_tol, unsigned char *__restrict__ mask) {
    const int b = blockIdx.x, p = threadIdx.x, lane = p & 31, w = p >> 5;
    const int np = bcount[b];
    __shared__ double red[4][BLK / 32];
    __shared__ double cen[4];
    double px = 0, py = 0, pz = 0;
    if (p < np) {
        const long long q = (long long)bstart[b] + p;
        px = pts[4 * q]; py = pts[4 * q + 1]; pz = pts[4 * q + 2];
    }
    double sx = px, sy = py, sz = pz;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
        sz += __shfl_xor_sync(0xffffffffu, sz, o);
    }
    if (lane == 0) { red[0][w] = sx; red[1][w] = sy; red[2][w] = sz; }
    __syncthreads();
    if (p == 0) {
        double a = 0, c = 0, d = 0;
        for (int k = 0; k < BLK / 32; ++k) { a += red[0][k]; c += red[1][k]; d += red[2][k]; }
        cen[0] = a / np; cen[1] = c / np; cen[2] = d / np;
    }
    __syncthreads();
    double rr = 0.0;
    if (p < np) {
        const double dx = px - cen[0], dy = py - cen[1], dz = pz - cen[2];
        rr = sqrt(dx * dx + dy * dy + dz * dz);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) rr = fmax(rr, __shfl_xor_sync(0xffffffffu, rr, o));
    if (lane == 0) red[3][w] = rr;
    __syncthreads();
    double rad = red[3][0];
    for (int k = 1; k < BLK / 32; ++k) rad = fmax(rad, red[3][k]);
    unsigned char *mb = mask + (long long)b * bs.nbf;
    for (int s = 0; s < bs.nshell; ++s) {
        const int at = bs.sh_atom[s], nf = ncart(bs.sh_l[s]), f0 = bs.sh_bf[s];
        const double dx = bs.atom_xyz[3 * at] - cen[0], dy = bs.atom_xyz[3 * at + 1] - cen[1], dz = bs.atom_xyz[3 * at + 2] - cen[2];
        if (sqrt(dx * dx + dy * dy + dz * dz) - rad >= shell_rad[s]) {
            if (p < nf) mb[f0 + p] = 0;
            continue;
        }
        for (int i = 0; i < nf; ++i) {
            const int f = f0 + i;
            double v = 0.0;
            if (p < np) {
                double o[1];
                basis_eval<0>(bs, f, px, py, pz, o);
                v = fabs(o[0] * bs.bf_norm[f]);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
            __syncthreads();  // red[0] reuse
            if (lane == 0) red[0][w] = v;
            __syncthreads();
            if (p == 0) {
                double m = red[0][0];
                for (int k = 1; k < BLK / 32; ++k) m = fmax(m, red[0][k]);
                mb[f] = m > bf_tol ? 1 : 0;
            }
        }
    }
}

// Number of kept functions per block.
__global__ void mask_count_kernel(int nblk, int nbf, const unsigned char *__restrict__ mask, int *__restrict__ cnt) {
    const int b = blockIdx.x;
    int c = 0;
    for (int f = threadIdx.x; f < nbf; f += 32) c += mask[(long long)b * nbf + f];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (threadIdx.x == 0) cnt[b] = c;
}

// Kept functions of each block in increasing order (one warp per block).
__global__ void mask_compact_kernel(int nblk, int nbf, const unsigned char *__restrict__ mask,
                                    const long long *__restrict__ foff, int *__restrict__ fun) {
    const int b = blockIdx.x, lane = threadIdx.x;
    long long o = foff[b];
    for (int f0 = 0; f0 < nbf; f0 += 32) {
        const int f = f0 + lane;
        const bool keep = f < nbf && mask[(long long)b * nbf + f];
        const unsigned bal = __ballot_sync(0xffffffffu, keep);
        if (keep) fun[o + __popc(bal & ((1u << lane) - 1u))] = f;
        o += __popc(bal);
    }
}

static double shell_radius(const pdg_context *ctx, const HostShell &h, double tol) {
    auto bound = [&](double r) {
        double s = 0.0;
        for (int k = 0; k < h.np; ++k)
            s += std::fabs(ctx->prim_coef[h.poff + k]) * std::pow(r, h.l) * std::exp(-ctx->prim_exp[h.poff + k] * r * r);
        return s * 1.7320508075688772;
    };
    double r = 1.0;
    while (bound(r) > tol && r < 200.0) r *= 1.5;
    // the bound decreases beyond its maximum; refine downwards
    double lo = 0.0, hi = r;
    for (int it = 0; it < 60; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (bound(mid) > tol) lo = mid; else hi = mid;
    }
    return hi;
}

extern "C" int pdg_grid_build(pdg_context *ctx, int accuracy, int n_radial, int angular_l, long long *n_points) {
    if (!ctx || accuracy < 1 || accuracy > 5 || n_radial < 0 || angular_l < 0) {
        pdg_set_error("pdg_grid_build: invalid argument");
        return PDG_ERR_ARG;
    }
    if (ctx->nbf == 0 || !ctx->have_geometry) { pdg_set_error("pdg_grid_build: basis and geometry required"); return PDG_ERR_STATE; }
    if (ctx->natom > 256) { pdg_set_error("pdg_grid_build: more than 256 atoms"); return PDG_ERR_UNSUPPORTED; }
    cudaSetDevice(ctx->device);
    ProfScope prof(ctx, "grid_build");
    if (!ctx->xc) ctx->xc = new XCData();
    ctx->xc->accuracy = accuracy;
    ctx->xc->nr = n_radial;
    ctx->xc->lq = angular_l;
    delete ctx->grid;
    ctx->grid = new GridData();
    GridData &G = *ctx->grid;
    const int acc = accuracy - 1;
    G.bf_tol = kBfTol[acc];
    G.rho_tol = kRhoTol[acc];
    const int na = ctx->natom;
    // ---- radial shells in the reference order (atom, radial shell); points made on the device ----
    std::vector<long long> rs_off, aoff(na + 1, 0);
    std::vector<int> rs_atom, rs_leb;
    std::vector<double> rs_r, rs_w;
    long long ncand = 0;
    const int nAngMin = leb_count[leb_index_for_order(9)];
    for (int at = 0; at < na; ++at) {
        aoff[at] = ncand;
        const int z = ctx->atomic_numbers.empty() ? (int)std::lround(ctx->Z[at]) : ctx->atomic_numbers[at];
        int nR, lMax;
        double rmax;
        atom_parameters(acc, z, &nR, &lMax, &rmax);
        if (n_radial > 0) nR = n_radial;
        if (angular_l > 0) lMax = angular_l;
        const int kmax = leb_index_for_order(lMax);
        const int nAngMax = leb_count[kmax];
        const double range = bragg(z), rcut = 0.2 * range;
        const double dfac = 1.0 + nR;
        for (int ir = 0; ir < nR; ++ir) {
            const double xn = (ir + 1) / dfac;
            const double r = range * std::pow(xn / (1.0 - xn), 2.0);
            const double wr = 2.0 * std::pow(range, 3.0) * std::pow(xn, 5.0) / std::pow(1.0 - xn, 7.0) / dfac;
            if (r > rmax) break;
            int k;
            if (r > rcut) k = kmax;
            else {
                const int n = (int)std::ceil((double)nAngMax * r / rcut);
                k = (n < nAngMin) ? leb_index_for_order(9) : leb_index_for_count(n);
            }
            rs_off.push_back(ncand);
            rs_atom.push_back(at);
            rs_leb.push_back(k);
            rs_r.push_back(r);
            rs_w.push_back(4.0 * PI * wr);
            ncand += leb_count[k];
        }
    }
    aoff[na] = ncand;
    // ---- partition weights on the device ----
    std::vector<double> rinv((size_t)na * na, 0.0), aij((size_t)na * na, 0.0);
    for (int i = 0; i < na; ++i)
        for (int j = 0; j < na; ++j) {
            if (i == j) continue;
            const double dx = ctx->xyz[3 * i] - ctx->xyz[3 * j], dy = ctx->xyz[3 * i + 1] - ctx->xyz[3 * j + 1],
                         dz = ctx->xyz[3 * i + 2] - ctx->xyz[3 * j + 2];
            rinv[i * na + j] = 1.0 / std::sqrt(dx * dx + dy * dy + dz * dz);
            const int zi = ctx->atomic_numbers.empty() ? (int)std::lround(ctx->Z[i]) : ctx->atomic_numbers[i];
            const int zj = ctx->atomic_numbers.empty() ? (int)std::lround(ctx->Z[j]) : ctx->atomic_numbers[j];
            const double chi = bragg(zi) / bragg(zj);
            const double temp = (chi - 1.0) / (chi + 1.0);
            double a = temp / (temp * temp - 1.0);
            if (a > 0.5) a = 0.5;
            if (a < -0.5) a = -0.5;
            aij[i * na + j] = a;
        }
    PDG_CHECK(pupload(ctx, "grid.rinv", &G.rinv, rinv));
    PDG_CHECK(pupload(ctx, "grid.aij", &G.aij, aij));
    const int nrs = (int)rs_off.size();
    long long *d_rs_off = nullptr, *d_aoff = nullptr;
    int *d_rs_atom = nullptr, *d_rs_leb = nullptr, *d_leb_off = nullptr;
    double *d_rs_r = nullptr, *d_rs_w = nullptr, *d_leb = nullptr;
    PDG_CHECK(pupload(ctx, "grid.rs_off", &d_rs_off, rs_off));
    PDG_CHECK(pupload(ctx, "grid.rs_atom", &d_rs_atom, rs_atom));
    PDG_CHECK(pupload(ctx, "grid.rs_leb", &d_rs_leb, rs_leb));
    PDG_CHECK(pupload(ctx, "grid.rs_r", &d_rs_r, rs_r));
    PDG_CHECK(pupload(ctx, "grid.rs_w", &d_rs_w, rs_w));
    PDG_CHECK(pupload(ctx, "grid.aoff", &d_aoff, aoff));
    PDG_CHECK(pupload(ctx, "grid.leb", &d_leb, std::vector<double>(leb_data, leb_data + 4 * LEB_TOTAL)));
    PDG_CHECK(pupload(ctx, "grid.leb_off", &d_leb_off, std::vector<int>(leb_offset, leb_offset + LEB_NORDERS)));
    const long long nscan = (ncand + SCAN_B - 1) / SCAN_B;
    double *dcand = (double *)pdg_pool(ctx, "grid.cand", std::max<long long>(1, 4 * ncand) * sizeof(double));
    int *dflag = (int *)pdg_pool(ctx, "grid.flag", std::max<long long>(1, ncand) * sizeof(int));
    int *dpos = (int *)pdg_pool(ctx, "grid.pos", std::max<long long>(1, ncand) * sizeof(int));
    int *dbsum = (int *)pdg_pool(ctx, "grid.bsum", (nscan + 1) * sizeof(int));
    int *dapos = (int *)pdg_pool(ctx, "grid.apos", (na + 1) * sizeof(int));
    if (!dcand || !dflag || !dpos || !dbsum || !dapos) { pdg_set_error("pdg_grid_build: allocation failed"); return PDG_ERR_ALLOC; }
    if (ncand > 0) {
        const int ct = wg_threads(na);
        const size_t csm = (size_t)ct * na * sizeof(double);
        PDG_CUDA(pdg_allow_max_smem(grid_candidates_kernel));
        { grid_candidates_kernel<<<(unsigned)((ncand + ct - 1) / ct), ct, csm, ctx->stream>>>(
            ncand, nrs, d_rs_off, d_rs_atom, d_rs_leb, d_rs_r, d_rs_w, d_leb, d_leb_off, na, ctx->dbasis.atom_xyz, G.rinv,
            G.aij, dcand, dflag); pdg_count_launch(); }
        { scan_block_sums_kernel<<<(unsigned)nscan, SCAN_B, 0, ctx->stream>>>(ncand, dflag, dbsum); pdg_count_launch(); }
        { scan_offsets_kernel<<<1, 32, 0, ctx->stream>>>((int)nscan, dbsum); pdg_count_launch(); }
        { scan_final_kernel<<<(unsigned)nscan, SCAN_B, 0, ctx->stream>>>(ncand, dflag, dbsum, dpos); pdg_count_launch(); }
        { gather_atom_pos_kernel<<<(na + 1 + 127) / 128, 128, 0, ctx->stream>>>(na, d_aoff, ncand, dpos, dflag, dapos); pdg_count_launch(); }
        PDG_CUDA(cudaGetLastError());
    }
    std::vector<int> apos(na + 1, 0);
    if (ncand > 0) PDG_CUDA(cudaMemcpyAsync(apos.data(), dapos, (na + 1) * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    // ---- 128-point blocks per atom over the kept points ----
    std::vector<int> bstart, bcount, batom;
    for (int at = 0; at < na; ++at)
        for (long long s = apos[at]; s < apos[at + 1]; s += BLK) {
            bstart.push_back((int)s);
            bcount.push_back((int)std::min<long long>(BLK, apos[at + 1] - s));
            batom.push_back(at);
        }
    G.npts = apos[na];
    G.nblk = (int)bstart.size();
    G.pts = (double *)pdg_pool(ctx, "grid.pts", std::max<long long>(1, 4 * G.npts) * sizeof(double));
    if (!G.pts) { pdg_set_error("pdg_grid_build: allocation failed"); return PDG_ERR_ALLOC; }
    if (ncand > 0) { grid_compact_kernel<<<(unsigned)((ncand + 255) / 256), 256, 0, ctx->stream>>>(ncand, dcand, dflag, dpos, G.pts); pdg_count_launch(); }
    PDG_CHECK(pupload(ctx, "grid.bstart", &G.bstart, bstart));
    PDG_CHECK(pupload(ctx, "grid.bcount", &G.bcount, bcount));
    PDG_CHECK(pupload(ctx, "grid.batom", &G.batom, batom));
    // ---- functions per block: distance screen and value filter on the device ----
    const int nsh = (int)ctx->shells.size();
    std::vector<double> shr(nsh);
    for (int s = 0; s < nsh; ++s) shr[s] = shell_radius(ctx, ctx->shells[s], 0.01 * G.bf_tol);
    double *dshr = nullptr;
    PDG_CHECK(pupload(ctx, "grid.shell_rad", &dshr, shr));
    const int nbf = ctx->nbf;
    unsigned char *dmask = (unsigned char *)pdg_pool(ctx, "grid.mask", std::max<size_t>(1, (size_t)G.nblk * nbf));
    int *dcnt = (int *)pdg_pool(ctx, "grid.fcnt", std::max(1, G.nblk) * sizeof(int));
    if (!dmask || !dcnt) { pdg_set_error("pdg_grid_build: allocation failed"); return PDG_ERR_ALLOC; }
    std::vector<int> fcnt(G.nblk, 0);
    if (G.nblk > 0) {
        { block_screen_kernel<<<G.nblk, BLK, 0, ctx->stream>>>(G.nblk, G.bstart, G.bcount, G.pts, dshr, ctx->dbasis, G.bf_tol, dmask); pdg_count_launch(); }
        { mask_count_kernel<<<G.nblk, 32, 0, ctx->stream>>>(G.nblk, nbf, dmask, dcnt); pdg_count_launch(); }
        PDG_CUDA(cudaGetLastError());
        PDG_CUDA(cudaMemcpyAsync(fcnt.data(), dcnt, G.nblk * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    std::vector<long long> foff(G.nblk + 1, 0), voff(G.nblk, 0);
    G.max_nf = 0;
    for (int b = 0; b < G.nblk; ++b) {
        foff[b + 1] = foff[b] + fcnt[b];
        voff[b] = 4 * BLK * foff[b];
        G.max_nf = std::max<int>(G.max_nf, fcnt[b]);
    }
    G.nfun_total = foff[G.nblk];
    G.h_foff = foff;
    G.h_bcount = bcount;
    PDG_CHECK(pupload(ctx, "grid.foff", &G.foff, foff));
    PDG_CHECK(pupload(ctx, "grid.voff", &G.voff, voff));
    G.fun = (int *)pdg_pool(ctx, "grid.fun", std::max<long long>(1, G.nfun_total) * sizeof(int));
    if (!G.fun) { pdg_set_error("pdg_grid_build: allocation failed"); return PDG_ERR_ALLOC; }
    if (G.nblk > 0) { mask_compact_kernel<<<G.nblk, 32, 0, ctx->stream>>>(G.nblk, nbf, dmask, G.foff, G.fun); pdg_count_launch(); }
    PDG_CUDA(cudaGetLastError());
    G.skip = (int *)pdg_pool(ctx, "grid.skip", std::max(1, G.nblk) * sizeof(int));
    if (!G.skip) { pdg_set_error("pdg_grid_build: allocation failed"); return PDG_ERR_ALLOC; }
    PDG_CUDA(cudaMemsetAsync(G.skip, 0, std::max(1, G.nblk) * sizeof(int), ctx->stream));
    const size_t vbytes = (size_t)4 * BLK * std::max<long long>(1, G.nfun_total) * sizeof(double);
    G.bval = (double *)pdg_pool(ctx, "grid.bval", vbytes);
    if (!G.bval) {
        pdg_set_error("pdg_grid_build: %zu bytes for resident basis values", vbytes);
        return PDG_ERR_ALLOC;
    }
    if (G.nblk > 0)
        { basis_values_kernel<<<G.nblk, BLK, 0, ctx->stream>>>(G.nblk, G.bstart, G.bcount, G.foff, G.fun, G.voff, G.pts,
                                                             ctx->dbasis, G.bval); pdg_count_launch(); }
    PDG_CUDA(cudaGetLastError());
    // per-point buffers
    XCData &X = *ctx->xc;
    // pool buffers: sized for this molecule and grid, grown (never freed) when a later one is larger
    X.pcoef = (double *)pdg_pool(ctx, "xc.pcoef", 4 * std::max<long long>(1, G.npts) * sizeof(double));
    X.pF = (double *)pdg_pool(ctx, "xc.pF", std::max<long long>(1, G.npts) * sizeof(double));
    X.V = (double *)pdg_pool(ctx, "xc.V", (size_t)ctx->nbf * ctx->nbf * sizeof(double));
    X.red = (double *)pdg_pool(ctx, "xc.red", 8 * sizeof(double));
    if (!X.pcoef || !X.pF || !X.V || !X.red) { pdg_set_error("pdg_grid_build: allocation failed"); return PDG_ERR_ALLOC; }
    X.cap = G.npts;
    X.have_coef = false;
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    if (n_points) *n_points = G.npts;
    return PDG_OK;
}

// Algorithmic FLOPs and resident-value bytes of one call of the XC density or V_xc kernel.
double pdg_grid_work(const pdg_context *ctx, const char *region, double *bytes) {
    *bytes = 0.0;
    if (!ctx->grid) return 0.0;
    const GridData &G = *ctx->grid;
    const bool rho = std::strcmp(region, "xc_rho") == 0;
    double w = 0.0;
    for (int b = 0; b < G.nblk; ++b) {
        const double nb = (double)(G.h_foff[b + 1] - G.h_foff[b]), P = G.h_bcount[b];
        w += rho ? (2.0 * nb * nb * P + 8.0 * nb * P) : 4.0 * nb * nb * P;
        *bytes += 4.0 * nb * BLK * sizeof(double);
    }
    return w;
}

static int ensure_grid(pdg_context *ctx) {
    if (ctx->grid) return PDG_OK;
    long long n;
    return pdg_grid_build(ctx, ctx->xc ? ctx->xc->accuracy : 3, ctx->xc ? ctx->xc->nr : 0, ctx->xc ? ctx->xc->lq : 0, &n);
}

static int chunk_for(int nf) { return nf * 16 * 8 <= 200 * 1024 ? 16 : 8; }

// Quadrature Fock: adds N V_xc N into the normalised Cartesian matrix d_F from the scaled density
// in ctx->d_D; returns E_xc and the integrated density.
int pdg_dft_fock_device(pdg_context *ctx, double *d_F, double *exc, double *rho) {
    PDG_CHECK(ensure_grid(ctx));
    GridData &G = *ctx->grid;
    XCData &X = *ctx->xc;
    const int n = ctx->nbf;
    PDG_CUDA(cudaMemsetAsync(X.red, 0, 8 * sizeof(double), ctx->stream));
    PDG_CUDA(cudaMemsetAsync(X.V, 0, (size_t)n * n * sizeof(double), ctx->stream));
    if (G.nblk > 0) {
        RhoArgs a;
        a.nblk = G.nblk; a.bstart = G.bstart; a.bcount = G.bcount; a.foff = G.foff; a.voff = G.voff; a.fun = G.fun;
        a.pts = G.pts; a.bval = G.bval; a.D = ctx->d_D; a.n = n; a.kind = X.kind; a.chunk = chunk_for(G.max_nf);
        a.rho_tol = G.rho_tol; a.pcoef = X.pcoef; a.pF = X.pF; a.red = X.red; a.skip = G.skip;
        {
            ProfScope prof(ctx, "xc_rho");
            const size_t sm = rho_smem(G.max_nf);
            PDG_CUDA(pdg_allow_max_smem(rho_xc_dmma_kernel));
            rho_xc_dmma_kernel<<<G.nblk, XT, sm, ctx->stream>>>(a);
            pdg_count_launch();
        }
        PDG_CUDA(cudaGetLastError());
        VxcArgs v;
        v.bcount = G.bcount; v.bstart = G.bstart; v.foff = G.foff; v.voff = G.voff; v.fun = G.fun; v.bval = G.bval;
        v.pcoef = X.pcoef; v.skip = G.skip; v.n = n; v.V = X.V; v.c0scale = 0.5;
        v.Z = (double *)pdg_pool(ctx, "xc.zval", (size_t)BLK * std::max<long long>(1, G.nfun_total) * sizeof(double));
        if (!v.Z) { pdg_set_error("device allocation failed (xc.zval)"); return PDG_ERR_ALLOC; }
        {
            ProfScope prof(ctx, "xc_vxc");
            PDG_CUDA(pdg_allow_max_smem(vxc_dmma_kernel));
            xc_z_kernel<<<G.nblk, XT, 0, ctx->stream>>>(v);
            pdg_count_launch();
            vxc_dmma_kernel<<<G.nblk, XT, sizeof(VxcSmem), ctx->stream>>>(v);
            pdg_count_launch();
        }
        PDG_CUDA(cudaGetLastError());
    }
    { vxc_finish_kernel<<<dim3((n + 255) / 256 < 4 ? (n + 255) / 256 : 4, n), 256, 0, ctx->stream>>>(
        n, X.V, ctx->dbasis.bf_norm, ctx->d_D, d_F, X.red + 2); pdg_count_launch(); }
    PDG_CUDA(cudaGetLastError());
    double h[3];
    PDG_CUDA(cudaMemcpyAsync(h, X.red, 3 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    *exc = h[0];
    *rho = h[1];
    X.last_vxc_trace = h[2];
    X.have_coef = true;
    return PDG_OK;
}

// XC gradient (basis + weight terms) of the density whose Fock build ran last, added to d_grad.
int pdg_dft_grad_device(pdg_context *ctx, double *d_grad) {
    PDG_CHECK(ensure_grid(ctx));
    GridData &G = *ctx->grid;
    XCData &X = *ctx->xc;
    if (!X.have_coef) { pdg_set_error("XC gradient needs a quadrature Fock build of the same density first"); return PDG_ERR_STATE; }
    if (G.nblk == 0) return PDG_OK;
    GradArgs a;
    a.bstart = G.bstart; a.bcount = G.bcount; a.batom = G.batom; a.foff = G.foff; a.voff = G.voff; a.fun = G.fun;
    a.pts = G.pts; a.bval = G.bval; a.pcoef = X.pcoef; a.D = ctx->d_D; a.skip = G.skip; a.bs = ctx->dbasis;
    a.n = ctx->nbf; a.chunk = 0; a.grad = d_grad;
    VxcArgs v;  // Zg = c . grad B rows for the W product
    v.bcount = G.bcount; v.bstart = G.bstart; v.foff = G.foff; v.voff = G.voff; v.fun = G.fun; v.bval = G.bval;
    v.pcoef = X.pcoef; v.skip = G.skip; v.n = ctx->nbf; v.V = nullptr; v.c0scale = 0.0;
    v.Z = (double *)pdg_pool(ctx, "xc.zval", (size_t)BLK * std::max<long long>(1, G.nfun_total) * sizeof(double));
    if (!v.Z) { pdg_set_error("device allocation failed (xc.zval)"); return PDG_ERR_ALLOC; }
    a.Z = v.Z;
    const size_t smem = xcgrad_smem(G.max_nf);
    PDG_CUDA(pdg_allow_max_smem(xc_grad_dmma_kernel));
    {
        ProfScope prof(ctx, "xc_grad");
        xc_z_kernel<<<G.nblk, XT, 0, ctx->stream>>>(v);
        pdg_count_launch();
        xc_grad_dmma_kernel<<<G.nblk, XT, smem, ctx->stream>>>(a);
        pdg_count_launch();
    }
    ProfScope profw(ctx, "xc_weight_grad");
    PDG_CUDA(cudaGetLastError());
    const size_t wsm = wg_smem(ctx->natom);
    PDG_CUDA(pdg_allow_max_smem(weight_grad_kernel));
    { weight_grad_kernel<<<G.nblk, wg_threads(ctx->natom), wsm, ctx->stream>>>(
        G.bstart, G.bcount, G.batom, G.skip, G.pts, X.pF, ctx->natom, ctx->dbasis.atom_xyz, G.rinv, G.aij, d_grad); pdg_count_launch(); }
    PDG_CUDA(cudaGetLastError());
    return PDG_OK;
}

int pdg_load_density(pdg_context *ctx, const double *packed_host);
int pdg_store_packed(pdg_context *ctx, const double *d_full_out, double *packed_host);
int pdg_cart_to_out(pdg_context *ctx, const double *Mc, double *Mo);

extern "C" int pdg_fock_quadrature(pdg_context *ctx, const double *density, double *fock, double *e_xc, double *rho_integral) {
    if (!ctx || !density || !fock) { pdg_set_error("pdg_fock_quadrature: invalid argument"); return PDG_ERR_ARG; }
    if (!pdg_dft_active(ctx)) { pdg_set_error("pdg_fock_quadrature: no density functional set"); return PDG_ERR_STATE; }
    if (ctx->nbf == 0 || !ctx->have_geometry) { pdg_set_error("pdg_fock_quadrature: basis and geometry required"); return PDG_ERR_STATE; }
    cudaSetDevice(ctx->device);
    PDG_CHECK(pdg_load_density(ctx, density));
    PDG_CUDA(cudaMemsetAsync(ctx->d_F, 0, (size_t)ctx->nbf * ctx->nbf * sizeof(double), ctx->stream));
    double exc = 0, rho = 0;
    PDG_CHECK(pdg_dft_fock_device(ctx, ctx->d_F, &exc, &rho));
    PDG_CHECK(pdg_cart_to_out(ctx, ctx->d_F, ctx->d_Fout));
    const int m = ctx->nbf_out;
    const size_t np = (size_t)m * (m + 1) / 2;
    std::vector<double> add(np);
    PDG_CHECK(pdg_store_packed(ctx, ctx->d_Fout, add.data()));
    for (size_t k = 0; k < np; ++k) fock[k] += add[k];
    if (e_xc) *e_xc = exc;
    if (rho_integral) *rho_integral = rho;
    return PDG_OK;
}

extern "C" int pdg_gradients_quadrature(pdg_context *ctx, const double *density, double *gradients3) {
    if (!ctx || !density || !gradients3) { pdg_set_error("pdg_gradients_quadrature: invalid argument"); return PDG_ERR_ARG; }
    if (!pdg_dft_active(ctx)) { pdg_set_error("pdg_gradients_quadrature: no density functional set"); return PDG_ERR_STATE; }
    cudaSetDevice(ctx->device);
    PDG_CHECK(pdg_load_density(ctx, density));
    double exc, rho;
    PDG_CUDA(cudaMemsetAsync(ctx->d_F, 0, (size_t)ctx->nbf * ctx->nbf * sizeof(double), ctx->stream));
    PDG_CHECK(pdg_dft_fock_device(ctx, ctx->d_F, &exc, &rho));  // per-point coefficients of this density
    PDG_CUDA(cudaMemsetAsync(ctx->d_grad, 0, 3 * ctx->natom * sizeof(double), ctx->stream));
    PDG_CHECK(pdg_dft_grad_device(ctx, ctx->d_grad));
    std::vector<double> h(3 * ctx->natom);
    PDG_CUDA(cudaMemcpyAsync(h.data(), ctx->d_grad, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    for (size_t k = 0; k < h.size(); ++k) gradients3[k] += h[k];
    return PDG_OK;
}
