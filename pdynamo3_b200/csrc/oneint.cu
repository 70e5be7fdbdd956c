// One-electron integrals (overlap, kinetic, electron-nuclear) and their gradients.
//
// Replaces GaussianBasisContainerIntegrals_f1KOf1i / _f1KOf1R1
// (GaussianBases/__extensions__/csource/GaussianBasisContainerIntegrals_f1Xg1.c:233,298) and
// _f2Cm1V / _f2Cm1R1 (GaussianBasisContainerIntegrals_f2Cp1.c:104,30).  One thread per shell
// pair; overlap and kinetic by the Obara-Saika recursion, electron-nuclear attraction by
// Rys quadrature with the nucleus as a narrow Gaussian charge, as the reference models it.
// Raw Cartesian integrals; the
// per-component normalisation is applied by the caller (N S N).
#include "context.h"
#include "rys.cuh"

namespace {

constexpr double PI = 3.141592653589793;
// Nuclei are normalised Gaussian charges of width 1e-4 bohr, exponent 4/(w^2 pi)
// (GaussianBases/__extensions__/cinclude/GaussianNucleus.h:13-15).  NUC_PREF =
// 2 pi^(5/2) (zeta/pi)^(3/2) / zeta, so that V = -Z NUC_PREF/(p sqrt(p+zeta)) K sum w Ix Iy Iz.
constexpr double NUC_ZETA = 4.0 / (1.0e-4 * 1.0e-4 * PI);
#define NUC_PREF (34.986836655249725 * sqrt(NUC_ZETA / PI) / PI)

// 1D overlap table S[i][j], i <= IM, j <= JM, without the exponential prefactor.
template <int IM, int JM>
__device__ __forceinline__ void os_overlap(double (&S)[IM + 1][JM + 1], double PA, double PB, double r2p) {
    S[0][0] = 1.0;
#pragma unroll
    for (int i = 0; i < IM; ++i) S[i + 1][0] = PA * S[i][0] + (i > 0 ? i * r2p * S[i > 0 ? i - 1 : 0][0] : 0.0);
#pragma unroll
    for (int j = 0; j < JM; ++j)
#pragma unroll
        for (int i = 0; i <= IM; ++i)
            S[i][j + 1] = PB * S[i][j] + (i > 0 ? i * r2p * S[i > 0 ? i - 1 : 0][j] : 0.0) +
                          (j > 0 ? j * r2p * S[i][j > 0 ? j - 1 : 0] : 0.0);
}

// 1D kinetic piece: -1/2 d^2/dx^2 acting on the second function, x^j exp(-b x^2).
template <int IM, int JM>
__device__ __forceinline__ double kin1d(const double (&S)[IM + 1][JM + 1], int i, int j, double b) {
    double t = -2.0 * b * (2 * j + 1) * S[i][j] + 4.0 * b * b * S[i][j + 2 <= JM ? j + 2 : JM];
    if (j >= 2) t += j * (j - 1) * S[i][j >= 2 ? j - 2 : 0];
    return -0.5 * t;
}

__device__ __forceinline__ void sh_xyz(const DeviceBasis &bs, int sh, double *r) {
    const int at = bs.sh_atom[sh];
    r[0] = bs.atom_xyz[3 * at]; r[1] = bs.atom_xyz[3 * at + 1]; r[2] = bs.atom_xyz[3 * at + 2];
}

// Electron-nuclear 1D integrals for one Rys node: I[a][b], a<=IA, b<=IB.
template <int IA, int IB>
__device__ __forceinline__ void nuc1d(double (&I)[IA + 1][IB + 1], double g0, double c00, double b10, double AB) {
    constexpr int L = IA + IB;
    double G[L + 1];
    G[0] = g0;
    if constexpr (L > 0) {
        G[1] = c00 * g0;
#pragma unroll
        for (int e = 1; e < L; ++e) G[e + 1] = c00 * G[e] + e * b10 * G[e - 1];
    }
    double T[L + 1][IB + 1];
#pragma unroll
    for (int e = 0; e <= L; ++e) T[e][0] = G[e];
#pragma unroll
    for (int b = 1; b <= IB; ++b)
#pragma unroll
        for (int a = 0; a <= L - b; ++a) T[a][b] = T[a + 1][b - 1] + AB * T[a][b - 1];
#pragma unroll
    for (int a = 0; a <= IA; ++a)
#pragma unroll
        for (int b = 0; b <= IB; ++b) I[a][b] = T[a][b];
}

template <int LA, int LB>
__global__ void __launch_bounds__(64) oneint_kernel(PairList pl, PrimPairs pp, DeviceBasis bs, int n,
                                                    double *__restrict__ Sm, double *__restrict__ Tm,
                                                    double *__restrict__ Vm) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= pl.n) return;
    constexpr int NA = ncart(LA), NB = ncart(LB);
    constexpr int NR = (LA + LB) / 2 + 1;
    const int A = pl.shA[t], B = pl.shB[t];
    double rA[3], rB[3];
    sh_xyz(bs, A, rA);
    sh_xyz(bs, B, rB);
    double s[NA * NB], k[NA * NB], v[NA * NB];
#pragma unroll
    for (int i = 0; i < NA * NB; ++i) { s[i] = 0.0; k[i] = 0.0; v[i] = 0.0; }
    const double AB[3] = {rA[0] - rB[0], rA[1] - rB[1], rA[2] - rB[2]};
    for (int ip = pl.poff[t]; ip < pl.poff[t] + pl.np[t]; ++ip) {
        const double a = pp.a[ip], b = pp.b[ip], p = a + b, r2p = 0.5 / p;
        const double P[3] = {pp.Px[ip], pp.Py[ip], pp.Pz[ip]};
        const double K = pp.K[ip];
        double Sx[LA + 1][LB + 3], Sy[LA + 1][LB + 3], Sz[LA + 1][LB + 3];
        os_overlap<LA, LB + 2>(Sx, P[0] - rA[0], P[0] - rB[0], r2p);
        os_overlap<LA, LB + 2>(Sy, P[1] - rA[1], P[1] - rB[1], r2p);
        os_overlap<LA, LB + 2>(Sz, P[2] - rA[2], P[2] - rB[2], r2p);
        const double sp = PI / p;
        const double pref = sp * sqrt(sp) * K;
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int jb = 0; jb < NB; ++jb) {
                const int ax = cart_x(LA, ia), ay = cart_y(LA, ia), az = cart_z(LA, ia);
                const int bx = cart_x(LB, jb), by = cart_y(LB, jb), bz = cart_z(LB, jb);
                const double ox = Sx[ax][bx], oy = Sy[ay][by], oz = Sz[az][bz];
                s[ia * NB + jb] += pref * ox * oy * oz;
                k[ia * NB + jb] += pref * (kin1d<LA, LB + 2>(Sx, ax, bx, b) * oy * oz + ox * kin1d<LA, LB + 2>(Sy, ay, by, b) * oz +
                                           ox * oy * kin1d<LA, LB + 2>(Sz, az, bz, b));
            }
        // electron-nuclear attraction with Gaussian nuclei: -sum_C Z_C (ab|C) with the nucleus a
        // normalised Gaussian of exponent NUC_ZETA, i.e. a (ab|ss) integral with q = NUC_ZETA.
        const double rhoN = p * NUC_ZETA / (p + NUC_ZETA), fz = NUC_ZETA / (p + NUC_ZETA);
        const double vpref = NUC_PREF / (p * sqrt(p + NUC_ZETA)) * K;
        for (int c = 0; c < bs.natom; ++c) {
            const double Z = bs.atom_Z[c];
            if (Z == 0.0) continue;
            const double PC[3] = {P[0] - bs.atom_xyz[3 * c], P[1] - bs.atom_xyz[3 * c + 1], P[2] - bs.atom_xyz[3 * c + 2]};
            const double x = rhoN * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
            double u[NR], w[NR];
            rys_roots<NR>(x, u, w);
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const double ur = u[r] * fz;
                const double b10 = r2p * (1.0 - ur);
                double Ix[LA + 1][LB + 1], Iy[LA + 1][LB + 1], Iz[LA + 1][LB + 1];
                nuc1d<LA, LB>(Ix, 1.0, P[0] - rA[0] - ur * PC[0], b10, AB[0]);
                nuc1d<LA, LB>(Iy, 1.0, P[1] - rA[1] - ur * PC[1], b10, AB[1]);
                nuc1d<LA, LB>(Iz, -Z * vpref * w[r], P[2] - rA[2] - ur * PC[2], b10, AB[2]);
#pragma unroll
                for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                    for (int jb = 0; jb < NB; ++jb)
                        v[ia * NB + jb] += Ix[cart_x(LA, ia)][cart_x(LB, jb)] * Iy[cart_y(LA, ia)][cart_y(LB, jb)] *
                                           Iz[cart_z(LA, ia)][cart_z(LB, jb)];
            }
        }
    }
    const int oa = bs.sh_bf[A], ob = bs.sh_bf[B];
#pragma unroll
    for (int ia = 0; ia < NA; ++ia)
#pragma unroll
        for (int jb = 0; jb < NB; ++jb) {
            const int f = ia * NB + jb;
            Sm[(oa + ia) * n + ob + jb] = s[f]; Sm[(ob + jb) * n + oa + ia] = s[f];
            Tm[(oa + ia) * n + ob + jb] = k[f]; Tm[(ob + jb) * n + oa + ia] = k[f];
            Vm[(oa + ia) * n + ob + jb] = v[f]; Vm[(ob + jb) * n + oa + ia] = v[f];
        }
}

// Gradient of sum_uv [P_uv (T+V)_uv - Ws_uv S_uv] with respect to nuclear positions, where
// P and Ws carry the component normalisation (N P N).  Ws is the energy-weighted density
// sum_i n_i e_i C C^T.
template <int LA, int LB>
__global__ void __launch_bounds__(64) oneint_grad_kernel(PairList pl, PrimPairs pp, DeviceBasis bs, int n,
                                                         const double *__restrict__ Pm, const double *__restrict__ Wm,
                                                         double *__restrict__ grad) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= pl.n) return;
    constexpr int NA = ncart(LA), NB = ncart(LB);
    constexpr int NR = (LA + LB + 1) / 2 + 1;
    const int A = pl.shA[t], B = pl.shB[t];
    const int atA = bs.sh_atom[A], atB = bs.sh_atom[B];
    double rA[3], rB[3];
    sh_xyz(bs, A, rA);
    sh_xyz(bs, B, rB);
    const int oa = bs.sh_bf[A], ob = bs.sh_bf[B];
    const double fac = (A == B) ? 1.0 : 2.0;
    double Pab[NA * NB], Wab[NA * NB];
#pragma unroll
    for (int ia = 0; ia < NA; ++ia)
#pragma unroll
        for (int jb = 0; jb < NB; ++jb) {
            Pab[ia * NB + jb] = fac * Pm[(oa + ia) * n + ob + jb];
            Wab[ia * NB + jb] = fac * Wm[(oa + ia) * n + ob + jb];
        }
    const double AB[3] = {rA[0] - rB[0], rA[1] - rB[1], rA[2] - rB[2]};
    double gA[3] = {0.0, 0.0, 0.0};  // overlap + kinetic, dB = -dA
    double gAv[3] = {0.0, 0.0, 0.0}, gBv[3] = {0.0, 0.0, 0.0};
    for (int ip = pl.poff[t]; ip < pl.poff[t] + pl.np[t]; ++ip) {
        const double a = pp.a[ip], b = pp.b[ip], p = a + b, r2p = 0.5 / p;
        const double P[3] = {pp.Px[ip], pp.Py[ip], pp.Pz[ip]};
        const double K = pp.K[ip];
        if (atA != atB) {
            double Sx[LA + 2][LB + 3], Sy[LA + 2][LB + 3], Sz[LA + 2][LB + 3];
            os_overlap<LA + 1, LB + 2>(Sx, P[0] - rA[0], P[0] - rB[0], r2p);
            os_overlap<LA + 1, LB + 2>(Sy, P[1] - rA[1], P[1] - rB[1], r2p);
            os_overlap<LA + 1, LB + 2>(Sz, P[2] - rA[2], P[2] - rB[2], r2p);
            const double sp = PI / p;
            const double pref = sp * sqrt(sp) * K;
#pragma unroll
            for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                for (int jb = 0; jb < NB; ++jb) {
                    const int ax = cart_x(LA, ia), ay = cart_y(LA, ia), az = cart_z(LA, ia);
                    const int bx = cart_x(LB, jb), by = cart_y(LB, jb), bz = cart_z(LB, jb);
                    const double ox = Sx[ax][bx], oy = Sy[ay][by], oz = Sz[az][bz];
                    const double tx = kin1d<LA + 1, LB + 2>(Sx, ax, bx, b);
                    const double ty = kin1d<LA + 1, LB + 2>(Sy, ay, by, b);
                    const double tz = kin1d<LA + 1, LB + 2>(Sz, az, bz, b);
                    // derivative of the first function along x: 2a S(ax+1) - ax S(ax-1)
                    const double dox = 2.0 * a * Sx[ax + 1][bx] - (ax > 0 ? ax * Sx[ax > 0 ? ax - 1 : 0][bx] : 0.0);
                    const double doy = 2.0 * a * Sy[ay + 1][by] - (ay > 0 ? ay * Sy[ay > 0 ? ay - 1 : 0][by] : 0.0);
                    const double doz = 2.0 * a * Sz[az + 1][bz] - (az > 0 ? az * Sz[az > 0 ? az - 1 : 0][bz] : 0.0);
                    const double dtx = 2.0 * a * kin1d<LA + 1, LB + 2>(Sx, ax + 1, bx, b) -
                                       (ax > 0 ? ax * kin1d<LA + 1, LB + 2>(Sx, ax > 0 ? ax - 1 : 0, bx, b) : 0.0);
                    const double dty = 2.0 * a * kin1d<LA + 1, LB + 2>(Sy, ay + 1, by, b) -
                                       (ay > 0 ? ay * kin1d<LA + 1, LB + 2>(Sy, ay > 0 ? ay - 1 : 0, by, b) : 0.0);
                    const double dtz = 2.0 * a * kin1d<LA + 1, LB + 2>(Sz, az + 1, bz, b) -
                                       (az > 0 ? az * kin1d<LA + 1, LB + 2>(Sz, az > 0 ? az - 1 : 0, bz, b) : 0.0);
                    const double dSx = dox * oy * oz, dSy = ox * doy * oz, dSz = ox * oy * doz;
                    const double dTx = dtx * oy * oz + dox * ty * oz + dox * oy * tz;
                    const double dTy = tx * doy * oz + ox * dty * oz + ox * doy * tz;
                    const double dTz = tx * oy * doz + ox * ty * doz + ox * oy * dtz;
                    const double pw = Pab[ia * NB + jb], ww = Wab[ia * NB + jb];
                    gA[0] += pref * (pw * dTx - ww * dSx);
                    gA[1] += pref * (pw * dTy - ww * dSy);
                    gA[2] += pref * (pw * dTz - ww * dSz);
                }
        }
        const double rhoN = p * NUC_ZETA / (p + NUC_ZETA), fz = NUC_ZETA / (p + NUC_ZETA);
        const double vpref = NUC_PREF / (p * sqrt(p + NUC_ZETA)) * K;
        for (int c = 0; c < bs.natom; ++c) {
            const double Z = bs.atom_Z[c];
            if (Z == 0.0) continue;
            const double PC[3] = {P[0] - bs.atom_xyz[3 * c], P[1] - bs.atom_xyz[3 * c + 1], P[2] - bs.atom_xyz[3 * c + 2]};
            const double x = rhoN * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
            double u[NR], w[NR];
            rys_roots<NR>(x, u, w);
            double cA[3] = {0.0, 0.0, 0.0}, cB[3] = {0.0, 0.0, 0.0};
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const double ur = u[r] * fz;
                const double b10 = r2p * (1.0 - ur);
                double Ix[LA + 2][LB + 2], Iy[LA + 2][LB + 2], Iz[LA + 2][LB + 2];
                nuc1d<LA + 1, LB + 1>(Ix, 1.0, P[0] - rA[0] - ur * PC[0], b10, AB[0]);
                nuc1d<LA + 1, LB + 1>(Iy, 1.0, P[1] - rA[1] - ur * PC[1], b10, AB[1]);
                nuc1d<LA + 1, LB + 1>(Iz, -Z * vpref * w[r], P[2] - rA[2] - ur * PC[2], b10, AB[2]);
#pragma unroll
                for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                    for (int jb = 0; jb < NB; ++jb) {
                        const int ax = cart_x(LA, ia), ay = cart_y(LA, ia), az = cart_z(LA, ia);
                        const int bx = cart_x(LB, jb), by = cart_y(LB, jb), bz = cart_z(LB, jb);
                        const double x0 = Ix[ax][bx], y0 = Iy[ay][by], z0 = Iz[az][bz];
                        const double dax = 2.0 * a * Ix[ax + 1][bx] - (ax > 0 ? ax * Ix[ax > 0 ? ax - 1 : 0][bx] : 0.0);
                        const double day = 2.0 * a * Iy[ay + 1][by] - (ay > 0 ? ay * Iy[ay > 0 ? ay - 1 : 0][by] : 0.0);
                        const double daz = 2.0 * a * Iz[az + 1][bz] - (az > 0 ? az * Iz[az > 0 ? az - 1 : 0][bz] : 0.0);
                        const double dbx = 2.0 * b * Ix[ax][bx + 1] - (bx > 0 ? bx * Ix[ax][bx > 0 ? bx - 1 : 0] : 0.0);
                        const double dby = 2.0 * b * Iy[ay][by + 1] - (by > 0 ? by * Iy[ay][by > 0 ? by - 1 : 0] : 0.0);
                        const double dbz = 2.0 * b * Iz[az][bz + 1] - (bz > 0 ? bz * Iz[az][bz > 0 ? bz - 1 : 0] : 0.0);
                        const double pw = Pab[ia * NB + jb];
                        cA[0] += pw * dax * y0 * z0; cA[1] += pw * x0 * day * z0; cA[2] += pw * x0 * y0 * daz;
                        cB[0] += pw * dbx * y0 * z0; cB[1] += pw * x0 * dby * z0; cB[2] += pw * x0 * y0 * dbz;
                    }
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                gAv[d] += cA[d];
                gBv[d] += cB[d];
            }
            // translational invariance of each nuclear term: dC = -(dA + dB)
            atomicAdd(&grad[3 * c + 0], -(cA[0] + cB[0]));
            atomicAdd(&grad[3 * c + 1], -(cA[1] + cB[1]));
            atomicAdd(&grad[3 * c + 2], -(cA[2] + cB[2]));
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        atomicAdd(&grad[3 * atA + d], gA[d] + gAv[d]);
        atomicAdd(&grad[3 * atB + d], -gA[d] + gBv[d]);
    }
}

constexpr int PLA[PDG_NPAIRCLASS] = {0, 1, 1, 2, 2, 2};
constexpr int PLB[PDG_NPAIRCLASS] = {0, 0, 1, 0, 1, 2};

template <int C>
void launch_oneint(const pdg_context *ctx, double *S, double *T, double *V) {
    const PairList &pl = ctx->pairs[C];
    if (pl.n == 0) return;
    { oneint_kernel<PLA[C], PLB[C]><<<(pl.n + 63) / 64, 64, 0, ctx->stream>>>(pl, ctx->pp, ctx->dbasis, ctx->nbf, S, T, V); pdg_count_launch(); }
}
template <int C>
void launch_oneint_grad(const pdg_context *ctx, const double *P, const double *W, double *g) {
    const PairList &pl = ctx->pairs[C];
    if (pl.n == 0) return;
    { oneint_grad_kernel<PLA[C], PLB[C]><<<(pl.n + 63) / 64, 64, 0, ctx->stream>>>(pl, ctx->pp, ctx->dbasis, ctx->nbf, P, W, g); pdg_count_launch(); }
}

}  // namespace

int pdg_oneint(pdg_context *ctx, double *d_S, double *d_T, double *d_V) {
    PDG_CHECK(pdg_ensure_pairs(ctx));
    ProfScope prof(ctx, "oneint");
    const size_t nn = (size_t)ctx->nbf * ctx->nbf * sizeof(double);
    PDG_CUDA(cudaMemsetAsync(d_S, 0, nn, ctx->stream));
    PDG_CUDA(cudaMemsetAsync(d_T, 0, nn, ctx->stream));
    PDG_CUDA(cudaMemsetAsync(d_V, 0, nn, ctx->stream));
    launch_oneint<0>(ctx, d_S, d_T, d_V);
    launch_oneint<1>(ctx, d_S, d_T, d_V);
    launch_oneint<2>(ctx, d_S, d_T, d_V);
    launch_oneint<3>(ctx, d_S, d_T, d_V);
    launch_oneint<4>(ctx, d_S, d_T, d_V);
    launch_oneint<5>(ctx, d_S, d_T, d_V);
    PDG_CUDA(cudaGetLastError());
    return PDG_OK;
}

int pdg_oneint_grad(pdg_context *ctx, const double *d_P, const double *d_W, double *d_grad) {
    PDG_CHECK(pdg_ensure_pairs(ctx));
    ProfScope prof(ctx, "oneint_grad");
    launch_oneint_grad<0>(ctx, d_P, d_W, d_grad);
    launch_oneint_grad<1>(ctx, d_P, d_W, d_grad);
    launch_oneint_grad<2>(ctx, d_P, d_W, d_grad);
    launch_oneint_grad<3>(ctx, d_P, d_W, d_grad);
    launch_oneint_grad<4>(ctx, d_P, d_W, d_grad);
    launch_oneint_grad<5>(ctx, d_P, d_W, d_grad);
    PDG_CUDA(cudaGetLastError());
    return PDG_OK;
}
