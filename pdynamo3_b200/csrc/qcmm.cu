// QC/MM electrostatics with MM point charges on the device.
//
// Replaces what NBModel/QCMMElectrostaticModelDensityFullGaussianBasis.py:131-185 asks of the
// Gaussian-basis evaluator: the electron-charge potentials f2Cm1V and their gradients f2Cm1R1
// (GaussianBases/__extensions__/csource/GaussianBasisContainerIntegrals_f2Cp1.c:104,30) with the
// MM charges, and the nucleus-charge term m1Cn1ER1 (GaussianBasisContainerIntegrals_p1Cq1.c:20-90).
// Without widths the reference treats the MM charges like the nuclei, as normalised Gaussian charges
// of width 1e-4 bohr (GaussianNucleus.h:13-19), so the integrals are the electron-nuclear ones with
// (q_c, R_c) in place of (Z_C, R_C).
//
// Layout: charges as (x, y, z, q) per charge, resident in the context's pool.  Potentials: one CTA
// per shell pair, its threads striding over the charges, block reduction of the component block
// (each matrix element has one writer).  Gradients: a 2D grid of (128-charge tiles) x (64-pair
// chunks); a thread owns one charge and keeps its gradient in registers over the chunk, the shell
// pair's two centre derivatives are reduced over the warp into per-CTA shared atom accumulators.
#include "context.h"
#include "rys.cuh"

int pdg_ensure_pairs(pdg_context *ctx);
int pdg_load_density(pdg_context *ctx, const double *packed_host);
int pdg_cart_to_out(pdg_context *ctx, const double *Mc, double *Mo);
int pdg_store_packed(pdg_context *ctx, const double *d_full_out, double *packed_host);
int pdg_out_to_cart(pdg_context *ctx, const double *Mo, double *Mc);
void pdg_launch_scale_full(pdg_context *ctx, int n, double *M, const double *norm);
const double *pdg_scf_resident_density(const pdg_context *ctx);

namespace {

constexpr double PI = 3.141592653589793;
constexpr double NUC_ZETA = 4.0 / (1.0e-4 * 1.0e-4 * PI);
#define NUC_PREF (34.986836655249725 * sqrt(NUC_ZETA / PI) / PI)
constexpr int QT = 128;   // threads per CTA
constexpr int PCH = 64;   // shell pairs per gradient CTA

// Electron-charge 1D integrals for one Rys node: I[a][b], a <= IA, b <= IB (vertical recursion on
// the combined index, then the horizontal transfer to the second centre).
template <int IA, int IB>
__device__ __forceinline__ void chg1d(double (&I)[IA + 1][IB + 1], double g0, double c00, double b10, double AB) {
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

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// V[a][b] += -sum_c q_c (ab|c) for one shell pair (raw Cartesian, both triangles).
template <int LA, int LB>
__global__ void __launch_bounds__(QT) qcmm_potential_kernel(PairList pl, PrimPairs pp, DeviceBasis bs, int n, int nmm,
                                                            const double4 *__restrict__ mm, double *__restrict__ Vm) {
    constexpr int NA = ncart(LA), NB = ncart(LB), NR = (LA + LB) / 2 + 1;
    __shared__ double red[QT / 32][NA * NB];
    const int t = blockIdx.x;
    const int A = pl.shA[t], B = pl.shB[t];
    const int atA = bs.sh_atom[A], atB = bs.sh_atom[B];
    const double rA[3] = {bs.atom_xyz[3 * atA], bs.atom_xyz[3 * atA + 1], bs.atom_xyz[3 * atA + 2]};
    const double rB[3] = {bs.atom_xyz[3 * atB], bs.atom_xyz[3 * atB + 1], bs.atom_xyz[3 * atB + 2]};
    const double AB[3] = {rA[0] - rB[0], rA[1] - rB[1], rA[2] - rB[2]};
    double v[NA * NB];
#pragma unroll
    for (int i = 0; i < NA * NB; ++i) v[i] = 0.0;
    for (int ip = pl.poff[t]; ip < pl.poff[t] + pl.np[t]; ++ip) {
        const double p = pp.a[ip] + pp.b[ip], r2p = 0.5 / p;
        const double P[3] = {pp.Px[ip], pp.Py[ip], pp.Pz[ip]};
        const double rhoN = p * NUC_ZETA / (p + NUC_ZETA), fz = NUC_ZETA / (p + NUC_ZETA);
        const double vpref = NUC_PREF / (p * sqrt(p + NUC_ZETA)) * pp.K[ip];
        for (int c = threadIdx.x; c < nmm; c += QT) {
            const double4 ch = mm[c];
            if (ch.w == 0.0) continue;
            const double PC[3] = {P[0] - ch.x, P[1] - ch.y, P[2] - ch.z};
            const double x = rhoN * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
            double u[NR], w[NR];
            rys_roots<NR>(x, u, w);
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const double ur = u[r] * fz;
                const double b10 = r2p * (1.0 - ur);
                double Ix[LA + 1][LB + 1], Iy[LA + 1][LB + 1], Iz[LA + 1][LB + 1];
                chg1d<LA, LB>(Ix, 1.0, P[0] - rA[0] - ur * PC[0], b10, AB[0]);
                chg1d<LA, LB>(Iy, 1.0, P[1] - rA[1] - ur * PC[1], b10, AB[1]);
                chg1d<LA, LB>(Iz, -ch.w * vpref * w[r], P[2] - rA[2] - ur * PC[2], b10, AB[2]);
#pragma unroll
                for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                    for (int jb = 0; jb < NB; ++jb)
                        v[ia * NB + jb] += Ix[cart_x(LA, ia)][cart_x(LB, jb)] * Iy[cart_y(LA, ia)][cart_y(LB, jb)] *
                                           Iz[cart_z(LA, ia)][cart_z(LB, jb)];
            }
        }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < NA * NB; ++i) {
        const double s = warp_sum(v[i]);
        if (lane == 0) red[warp][i] = s;
    }
    __syncthreads();
    const int oa = bs.sh_bf[A], ob = bs.sh_bf[B];
    for (int i = threadIdx.x; i < NA * NB; i += QT) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < QT / 32; ++w) s += red[w][i];
        const int ia = i / NB, jb = i - ia * NB;
        Vm[(long long)(oa + ia) * n + ob + jb] += s;
        if (A != B) Vm[(long long)(ob + jb) * n + oa + ia] += s;
    }
}

// Gradient of sum_ab P'_ab V_ab (P' the scaled Cartesian density, off-diagonal shell blocks
// doubled) over the pairs [p0, p1) of one class: the charge's gradient in registers, the centre
// derivatives of A and B reduced over the warp into shared per-atom sums.
template <int LA, int LB>
__global__ void __launch_bounds__(QT) qcmm_grad_kernel(PairList pl, PrimPairs pp, DeviceBasis bs, int n, int nmm,
                                                       const double4 *__restrict__ mm, const double *__restrict__ Pm,
                                                       double *__restrict__ gqc, double *__restrict__ gmm) {
    constexpr int NA = ncart(LA), NB = ncart(LB), NR = (LA + LB + 1) / 2 + 1;
    extern __shared__ double gsh[];  // 3 * natom
    for (int e = threadIdx.x; e < 3 * bs.natom; e += QT) gsh[e] = 0.0;
    __syncthreads();
    const int c = blockIdx.x * QT + threadIdx.x;
    const bool have = c < nmm;
    const double4 ch = have ? mm[c] : make_double4(0.0, 0.0, 0.0, 0.0);
    const bool live = have && ch.w != 0.0;
    const int lane = threadIdx.x & 31;
    double gC[3] = {0.0, 0.0, 0.0};
    const int p0 = blockIdx.y * PCH, p1 = min(pl.n, p0 + PCH);
    for (int t = p0; t < p1; ++t) {
        const int A = pl.shA[t], B = pl.shB[t];
        const int atA = bs.sh_atom[A], atB = bs.sh_atom[B];
        const double rA[3] = {bs.atom_xyz[3 * atA], bs.atom_xyz[3 * atA + 1], bs.atom_xyz[3 * atA + 2]};
        const double rB[3] = {bs.atom_xyz[3 * atB], bs.atom_xyz[3 * atB + 1], bs.atom_xyz[3 * atB + 2]};
        const double AB[3] = {rA[0] - rB[0], rA[1] - rB[1], rA[2] - rB[2]};
        const int oa = bs.sh_bf[A], ob = bs.sh_bf[B];
        const double fac = (A == B) ? 1.0 : 2.0;
        double Pab[NA * NB];
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int jb = 0; jb < NB; ++jb) Pab[ia * NB + jb] = fac * Pm[(long long)(oa + ia) * n + ob + jb];
        double cA[3] = {0.0, 0.0, 0.0}, cB[3] = {0.0, 0.0, 0.0};
        if (live) {
            for (int ip = pl.poff[t]; ip < pl.poff[t] + pl.np[t]; ++ip) {
                const double a = pp.a[ip], b = pp.b[ip], p = a + b, r2p = 0.5 / p;
                const double P[3] = {pp.Px[ip], pp.Py[ip], pp.Pz[ip]};
                const double rhoN = p * NUC_ZETA / (p + NUC_ZETA), fz = NUC_ZETA / (p + NUC_ZETA);
                const double vpref = NUC_PREF / (p * sqrt(p + NUC_ZETA)) * pp.K[ip];
                const double PC[3] = {P[0] - ch.x, P[1] - ch.y, P[2] - ch.z};
                const double x = rhoN * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
                double u[NR], w[NR];
                rys_roots<NR>(x, u, w);
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    const double ur = u[r] * fz;
                    const double b10 = r2p * (1.0 - ur);
                    double Ix[LA + 2][LB + 2], Iy[LA + 2][LB + 2], Iz[LA + 2][LB + 2];
                    chg1d<LA + 1, LB + 1>(Ix, 1.0, P[0] - rA[0] - ur * PC[0], b10, AB[0]);
                    chg1d<LA + 1, LB + 1>(Iy, 1.0, P[1] - rA[1] - ur * PC[1], b10, AB[1]);
                    chg1d<LA + 1, LB + 1>(Iz, -ch.w * vpref * w[r], P[2] - rA[2] - ur * PC[2], b10, AB[2]);
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
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            gC[d] -= cA[d] + cB[d];  // translational invariance of each charge term
            const double sa = warp_sum(cA[d]), sb = warp_sum(cB[d]);
            if (lane == 0) {
                if (sa != 0.0) atomicAdd(&gsh[3 * atA + d], sa);
                if (sb != 0.0) atomicAdd(&gsh[3 * atB + d], sb);
            }
        }
    }
    if (have) {
#pragma unroll
        for (int d = 0; d < 3; ++d)
            if (gC[d] != 0.0) atomicAdd(&gmm[3 * c + d], gC[d]);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 3 * bs.natom; e += QT)
        if (gsh[e] != 0.0) atomicAdd(&gqc[e], gsh[e]);
}

// Nucleus-charge energy and gradients, one thread per charge: both are Gaussian charges of the
// nuclear width, E = q_c Z_C 2 sqrt(rho/pi) F0(rho r^2) with rho = zeta/2 (p1Cq1.c:69-74), and
// dE/dr = -4 rho sqrt(rho/pi) q Z F0 u r with u the one-node Rys node F1/F0.
__global__ void __launch_bounds__(QT) qcmm_core_kernel(DeviceBasis bs, int nmm, const double4 *__restrict__ mm,
                                                       double *__restrict__ energy, double *__restrict__ gqc,
                                                       double *__restrict__ gmm) {
    extern __shared__ double csh[];  // 3 * natom gradient sums, then the per-warp energies
    double *wen = csh + 3 * bs.natom;
    for (int e = threadIdx.x; e < 3 * bs.natom; e += QT) csh[e] = 0.0;
    __syncthreads();
    const int c = blockIdx.x * QT + threadIdx.x;
    const double rho = 0.5 * NUC_ZETA, f0 = 2.0 * sqrt(rho / PI);
    double e = 0.0, g[3] = {0.0, 0.0, 0.0};
    if (c < nmm) {
        const double4 ch = mm[c];
        for (int i = 0; i < bs.natom; ++i) {
            const double Z = bs.atom_Z[i];
            if (Z == 0.0 || ch.w == 0.0) continue;
            const double d[3] = {bs.atom_xyz[3 * i] - ch.x, bs.atom_xyz[3 * i + 1] - ch.y, bs.atom_xyz[3 * i + 2] - ch.z};
            const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
            double u[1], w[1];
            rys_roots<1>(rho * r2, u, w);
            const double term = f0 * Z * ch.w * w[0];
            e += term;
            if (gqc) {
                const double dF = -2.0 * rho * u[0] * term;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    atomicAdd(&csh[3 * i + k], dF * d[k]);
                    g[k] -= dF * d[k];
                }
            }
        }
    }
    const double ws = warp_sum(e);
    if ((threadIdx.x & 31) == 0) wen[threadIdx.x >> 5] = ws;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < QT / 32; ++k) s += wen[k];
        atomicAdd(energy, s);
    }
    if (gqc) {
        if (c < nmm)
#pragma unroll
            for (int k = 0; k < 3; ++k) gmm[3 * c + k] += g[k];
        for (int i = threadIdx.x; i < 3 * bs.natom; i += QT)
            if (csh[i] != 0.0) atomicAdd(&gqc[i], csh[i]);
    }
}

constexpr int PLA[PDG_NPAIRCLASS] = {0, 1, 1, 2, 2, 2};
constexpr int PLB[PDG_NPAIRCLASS] = {0, 0, 1, 0, 1, 2};

template <int C>
void launch_potential(const pdg_context *ctx, double *V) {
    const PairList &pl = ctx->pairs[C];
    if (pl.n == 0) return;
    { qcmm_potential_kernel<PLA[C], PLB[C]><<<pl.n, QT, 0, ctx->stream>>>(pl, ctx->pp, ctx->dbasis, ctx->nbf, ctx->nmm,
        reinterpret_cast<const double4 *>(ctx->d_mm), V); pdg_count_launch(); }
}
template <int C>
void launch_grad(const pdg_context *ctx, const double *P, double *gq, double *gm) {
    const PairList &pl = ctx->pairs[C];
    if (pl.n == 0) return;
    const dim3 grid((ctx->nmm + QT - 1) / QT, (pl.n + PCH - 1) / PCH);
    { qcmm_grad_kernel<PLA[C], PLB[C]><<<grid, QT, 3 * ctx->natom * sizeof(double), ctx->stream>>>(
        pl, ctx->pp, ctx->dbasis, ctx->nbf, ctx->nmm, reinterpret_cast<const double4 *>(ctx->d_mm), P, gq, gm); pdg_count_launch(); }
}

}  // namespace

// V_mm added into the raw Cartesian electron-nuclear matrix Vc (n x n) when charges are set.
int pdg_qcmm_add_potentials(pdg_context *ctx, double *Vc) {
    if (ctx->nmm == 0) return PDG_OK;
    PDG_CHECK(pdg_ensure_pairs(ctx));
    ProfScope prof(ctx, "qcmm_potentials");
    launch_potential<0>(ctx, Vc);
    launch_potential<1>(ctx, Vc);
    launch_potential<2>(ctx, Vc);
    launch_potential<3>(ctx, Vc);
    launch_potential<4>(ctx, Vc);
    launch_potential<5>(ctx, Vc);
    PDG_CUDA(cudaGetLastError());
    return PDG_OK;
}

extern "C" int pdg_set_point_charges(pdg_context *ctx, int n, const double *charges, const double *xyz) {
    if (!ctx || n < 0 || (n > 0 && (!charges || !xyz))) { pdg_set_error("pdg_set_point_charges: invalid argument"); return PDG_ERR_ARG; }
    cudaSetDevice(ctx->device);
    ctx->nmm = 0;
    ctx->inc_count = -1;  // the core Hamiltonian changes: no difference build across it
    if (n == 0) return PDG_OK;
    std::vector<double> h(4 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        h[4 * i] = xyz[3 * i]; h[4 * i + 1] = xyz[3 * i + 1]; h[4 * i + 2] = xyz[3 * i + 2]; h[4 * i + 3] = charges[i];
    }
    ctx->d_mm = (double *)pdg_pool(ctx, "qcmm.charges", h.size() * sizeof(double));
    if (!ctx->d_mm) { pdg_set_error("pdg_set_point_charges: device allocation failed"); return PDG_ERR_ALLOC; }
    PDG_CUDA(cudaMemcpyAsync(ctx->d_mm, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->nmm = n;
    return PDG_OK;
}

extern "C" int pdg_qcmm_potentials(pdg_context *ctx, double *potentials) {
    if (!ctx || !potentials) { pdg_set_error("pdg_qcmm_potentials: invalid argument"); return PDG_ERR_ARG; }
    if (ctx->nbf == 0 || !ctx->have_geometry) { pdg_set_error("pdg_qcmm_potentials: basis and geometry required"); return PDG_ERR_STATE; }
    cudaSetDevice(ctx->device);
    const int n = ctx->nbf;
    double *Vc = (double *)pdg_pool(ctx, "qcmm.V", (size_t)n * n * sizeof(double));
    if (!Vc) { pdg_set_error("pdg_qcmm_potentials: device allocation failed"); return PDG_ERR_ALLOC; }
    PDG_CUDA(cudaMemsetAsync(Vc, 0, (size_t)n * n * sizeof(double), ctx->stream));
    PDG_CHECK(pdg_qcmm_add_potentials(ctx, Vc));
    pdg_launch_scale_full(ctx, n, Vc, ctx->dbasis.bf_norm);
    PDG_CHECK(pdg_cart_to_out(ctx, Vc, ctx->d_Dout));
    return pdg_store_packed(ctx, ctx->d_Dout, potentials);
}

extern "C" int pdg_qcmm_gradients(pdg_context *ctx, const double *density, double *gradients_qc, double *gradients_mm) {
    if (!ctx || !gradients_qc || (ctx->nmm > 0 && !gradients_mm)) { pdg_set_error("pdg_qcmm_gradients: invalid argument"); return PDG_ERR_ARG; }
    if (ctx->nbf == 0 || !ctx->have_geometry) { pdg_set_error("pdg_qcmm_gradients: basis and geometry required"); return PDG_ERR_STATE; }
    if (ctx->nmm == 0) return PDG_OK;
    cudaSetDevice(ctx->device);
    PDG_CHECK(pdg_ensure_pairs(ctx));
    if (density) {
        PDG_CHECK(pdg_load_density(ctx, density));
    } else {
        const double *P = pdg_scf_resident_density(ctx);
        if (!P) { pdg_set_error("pdg_qcmm_gradients: no density given and no SCF result"); return PDG_ERR_STATE; }
        PDG_CHECK(pdg_out_to_cart(ctx, P, ctx->d_D));
        pdg_launch_scale_full(ctx, ctx->nbf, ctx->d_D, ctx->dbasis.bf_norm);
    }
    const int na = ctx->natom, nm = ctx->nmm;
    double *dg = (double *)pdg_pool(ctx, "qcmm.grad", 3 * (size_t)(na + nm) * sizeof(double));
    if (!dg) { pdg_set_error("pdg_qcmm_gradients: device allocation failed"); return PDG_ERR_ALLOC; }
    PDG_CUDA(cudaMemsetAsync(dg, 0, 3 * (size_t)(na + nm) * sizeof(double), ctx->stream));
    {
        ProfScope prof(ctx, "qcmm_grad");
        launch_grad<0>(ctx, ctx->d_D, dg, dg + 3 * na);
        launch_grad<1>(ctx, ctx->d_D, dg, dg + 3 * na);
        launch_grad<2>(ctx, ctx->d_D, dg, dg + 3 * na);
        launch_grad<3>(ctx, ctx->d_D, dg, dg + 3 * na);
        launch_grad<4>(ctx, ctx->d_D, dg, dg + 3 * na);
        launch_grad<5>(ctx, ctx->d_D, dg, dg + 3 * na);
    }
    PDG_CUDA(cudaGetLastError());
    std::vector<double> h(3 * (size_t)(na + nm));
    PDG_CUDA(cudaMemcpyAsync(h.data(), dg, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int k = 0; k < 3 * na; ++k) gradients_qc[k] += h[k];
    for (int k = 0; k < 3 * nm; ++k) gradients_mm[k] += h[3 * na + k];
    return PDG_OK;
}

extern "C" int pdg_qcmm_core(pdg_context *ctx, double *energy, double *gradients_qc, double *gradients_mm) {
    if (!ctx || !energy || ((gradients_qc == nullptr) != (gradients_mm == nullptr))) {
        pdg_set_error("pdg_qcmm_core: invalid argument"); return PDG_ERR_ARG;
    }
    if (ctx->nbf == 0 || !ctx->have_geometry) { pdg_set_error("pdg_qcmm_core: basis and geometry required"); return PDG_ERR_STATE; }
    *energy = 0.0;
    if (ctx->nmm == 0) return PDG_OK;
    cudaSetDevice(ctx->device);
    const int na = ctx->natom, nm = ctx->nmm;
    const bool grad = gradients_qc != nullptr;
    double *dg = (double *)pdg_pool(ctx, "qcmm.core", (1 + 3 * (size_t)(na + nm)) * sizeof(double));
    if (!dg) { pdg_set_error("pdg_qcmm_core: device allocation failed"); return PDG_ERR_ALLOC; }
    PDG_CUDA(cudaMemsetAsync(dg, 0, (1 + 3 * (size_t)(na + nm)) * sizeof(double), ctx->stream));
    { qcmm_core_kernel<<<(nm + QT - 1) / QT, QT, (3 * na + QT / 32) * sizeof(double), ctx->stream>>>(
        ctx->dbasis, nm, reinterpret_cast<const double4 *>(ctx->d_mm), dg, grad ? dg + 1 : nullptr,
        grad ? dg + 1 + 3 * na : nullptr); pdg_count_launch(); }
    PDG_CUDA(cudaGetLastError());
    std::vector<double> h(1 + 3 * (size_t)(na + nm));
    PDG_CUDA(cudaMemcpyAsync(h.data(), dg, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    *energy = h[0];
    if (grad) {
        for (int k = 0; k < 3 * na; ++k) gradients_qc[k] += h[1 + k];
        for (int k = 0; k < 3 * nm; ++k) gradients_mm[k] += h[1 + 3 * na + k];
    }
    return PDG_OK;
}
