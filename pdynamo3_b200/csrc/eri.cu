// Integral-direct two-electron Coulomb/exchange build: Rys shell-quartet kernels grouped
// by angular-momentum class, Schwarz-screened, digested straight into J and K.
//
// Replaces the reference's stored-integral path: GaussianBasisContainerIntegrals_f2Cf2i
// (GaussianBases/__extensions__/csource/GaussianBasisContainerIntegrals_f2Xf2.c:74-139),
// GaussianBasisIntegrals_f2Cf2i (GaussianBasisIntegrals_f2Xf2.c:496-891) and the digest
// Fock_MakeFromTEIs / _Coulomb / _Exchange (QCModel/__extensions__/csource/FockConstruction.c:209-377).
//
// Conventions (all on raw Cartesian integrals; the per-component normalisation n_a is
// folded into D' = N D N on input and F = N F' N on output):
//   for each unique shell quartet (AB|CD), A>=B, C>=D, (AB)>=(CD), degeneracy factor
//   s = 1/2^(#coincidences), full component block V[a][b][c][d]:
//     Jt[a][b] += 2 s sum_cd V D'cd,  Jt[c][d] += 2 s sum_ab V D'ab
//     Kt[a][c] += s sum V D'bd, Kt[a][d] += s sum V D'bc, Kt[b][c] += s sum V D'ad, Kt[b][d] += s sum V D'ac
//   J = Jt + Jt^T, K = Kt + Kt^T, F2 = J - (c_x/2) K, E2 = 1/2 tr(P F2)
// which equals the reference digest, including its 1e-12 storage underflow when
// tei_underflow = 1e-12 (BlockStorage.c:160-181).
#include <algorithm>
#include <cmath>
#include <numeric>

#include "context.h"
#include "rys.cuh"
#include "rys2d.cuh"

namespace {

constexpr double TWO_PI_POW_2P5 = 34.986836655249725;  // 2 pi^(5/2)

__host__ __device__ constexpr double comp_norm(int l, int i) {
    // sqrt((2l-1)!! / ((2x-1)!! (2y-1)!! (2z-1)!!)) for l <= 2: only xy, xz, yz differ from 1.
    return (l == 2 && (i == 1 || i == 3 || i == 4)) ? 1.7320508075688772 : 1.0;
}

struct QuartetGeom {
    double A[3], B[3], C[3], D[3];
};

// Contracted raw Cartesian block V[(a*NB+b)*NC*ND + c*ND + d] of one shell quartet.  CUT applies
// the reference's primitive-quartet cut; the Schwarz diagonal is computed without it, because a
// primitive pair cut in (ab|ab) can still contribute to (ab|cd) against a compact ket pair.
template <int LA, int LB, int LC, int LD, bool CUT = true>
__device__ __forceinline__ void eri_block(const PrimPairs &pp, int pb0, int npb, int pk0, int npk,
                                          const QuartetGeom &g,
                                          double (&V)[ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD)]) {
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    constexpr int LAB = LA + LB, LCD = LC + LD, NR = (LAB + LCD) / 2 + 1;
#pragma unroll
    for (int i = 0; i < NA * NB * NC * ND; ++i) V[i] = 0.0;
    const double ABx = g.A[0] - g.B[0], ABy = g.A[1] - g.B[1], ABz = g.A[2] - g.B[2];
    const double CDx = g.C[0] - g.D[0], CDy = g.C[1] - g.D[1], CDz = g.C[2] - g.D[2];
    for (int ib = pb0; ib < pb0 + npb; ++ib) {
        const double p = pp.a[ib] + pp.b[ib];
        const double Px = pp.Px[ib], Py = pp.Py[ib], Pz = pp.Pz[ib];
        const double Kb = pp.K[ib], argb = pp.arg[ib];
        const double PAx = Px - g.A[0], PAy = Py - g.A[1], PAz = Pz - g.A[2];
        for (int ik = pk0; ik < pk0 + npk; ++ik) {
            const double argk = pp.arg[ik];
            if (CUT && argb + argk > PDG_PRIMITIVE_CUT) continue;
            const double q = pp.a[ik] + pp.b[ik];
            const double Qx = pp.Px[ik], Qy = pp.Py[ik], Qz = pp.Pz[ik];
            const double pq = p * q, ppq = p + q, rppq = 1.0 / ppq;
            const double PQx = Px - Qx, PQy = Py - Qy, PQz = Pz - Qz;
            const double x = pq * rppq * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pref = TWO_PI_POW_2P5 / (pq * sqrt(ppq)) * Kb * pp.K[ik];
            double u[NR], w[NR];
            rys_roots<NR>(x, u, w);
            const double QCx = Qx - g.C[0], QCy = Qy - g.C[1], QCz = Qz - g.C[2];
            const double r2p = 0.5 / p, r2q = 0.5 / q;
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const double ur = u[r] * rppq;
                const double b00 = 0.5 * ur;
                const double b10 = r2p * (1.0 - q * ur);
                const double b01 = r2q * (1.0 - p * ur);
                const double fq = q * ur, fp = p * ur;
                double Gx[LAB + 1][LCD + 1], Gy[LAB + 1][LCD + 1], Gz[LAB + 1][LCD + 1];
                rys_vrr<LAB, LCD>(Gx, 1.0, PAx - fq * PQx, QCx + fp * PQx, b10, b01, b00);
                rys_vrr<LAB, LCD>(Gy, 1.0, PAy - fq * PQy, QCy + fp * PQy, b10, b01, b00);
                rys_vrr<LAB, LCD>(Gz, w[r] * pref, PAz - fq * PQz, QCz + fp * PQz, b10, b01, b00);
                double Ix[LA + 1][LB + 1][LC + 1][LD + 1], Iy[LA + 1][LB + 1][LC + 1][LD + 1],
                    Iz[LA + 1][LB + 1][LC + 1][LD + 1];
                rys_hrr<LA, LB, LC, LD>(Gx, ABx, CDx, Ix);
                rys_hrr<LA, LB, LC, LD>(Gy, ABy, CDy, Iy);
                rys_hrr<LA, LB, LC, LD>(Gz, ABz, CDz, Iz);
#pragma unroll
                for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                    for (int jb = 0; jb < NB; ++jb)
#pragma unroll
                        for (int kc = 0; kc < NC; ++kc)
#pragma unroll
                            for (int ld = 0; ld < ND; ++ld) {
                                const double vx = Ix[cart_x(LA, ia)][cart_x(LB, jb)][cart_x(LC, kc)][cart_x(LD, ld)];
                                const double vy = Iy[cart_y(LA, ia)][cart_y(LB, jb)][cart_y(LC, kc)][cart_y(LD, ld)];
                                const double vz = Iz[cart_z(LA, ia)][cart_z(LB, jb)][cart_z(LC, kc)][cart_z(LD, ld)];
                                V[((ia * NB + jb) * NC + kc) * ND + ld] += vx * vy * vz;
                            }
            }
        }
    }
}

__device__ __forceinline__ void load_xyz(const DeviceBasis &bs, int sh, double *r) {
    const int at = bs.sh_atom[sh];
    r[0] = bs.atom_xyz[3 * at];
    r[1] = bs.atom_xyz[3 * at + 1];
    r[2] = bs.atom_xyz[3 * at + 2];
}

// Schwarz bound per shell pair: Q = sqrt(max_ab |(ab|ab)|) with the true normalisation.
template <int LA, int LB>
__global__ void __launch_bounds__(64) schwarz_kernel(const int n, const int *__restrict__ shA,
                                                     const int *__restrict__ shB, const int *__restrict__ poff,
                                                     const int *__restrict__ np, PrimPairs pp, DeviceBasis bs,
                                                     double *__restrict__ Q) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    constexpr int NA = ncart(LA), NB = ncart(LB);
    QuartetGeom g;
    load_xyz(bs, shA[t], g.A);
    load_xyz(bs, shB[t], g.B);
#pragma unroll
    for (int c = 0; c < 3; ++c) { g.C[c] = g.A[c]; g.D[c] = g.B[c]; }
    double V[NA * NB * NA * NB];
    eri_block<LA, LB, LA, LB, false>(pp, poff[t], np[t], poff[t], np[t], g, V);
    double m = 0.0;
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const double nn = comp_norm(LA, a) * comp_norm(LB, b);
            m = fmax(m, fabs(V[((a * NB + b) * NA + a) * NB + b]) * nn * nn);
        }
    Q[t] = sqrt(m);
}

struct JKArgs {
    PairList bra, ket;
    const long long *offs;
    long long total;
    int same;
    PrimPairs pp;
    DeviceBasis bs;
    const double *D;
    double *J, *K;
    int n;
    double underflow;
    const double *dmax;  // optional: max |D'| per shell-pair block (nshell x nshell) for density screening
    int nshell;
    double dcut;         // skip a quartet when Q_AB Q_CD max(relevant dmax) < dcut
};

template <int LA, int LB, int LC, int LD, bool DOJ, bool DOK>
__global__ void __launch_bounds__(128) eri_jk_kernel(JKArgs args) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= args.total) return;
    int lo = 0, hi = args.bra.n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (args.offs[mid] <= t) lo = mid; else hi = mid;
    }
    const int ib = lo;
    const int ik = (int)(t - args.offs[ib]);
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    const int A = args.bra.shA[ib], B = args.bra.shB[ib], C = args.ket.shA[ik], D = args.ket.shB[ik];
    if (args.dmax) {
        // density screening: the quartet changes J (K) by at most Q_AB Q_CD times the largest
        // density element it is contracted with
        const int ns = args.nshell;
        double dm = 0.0;
        if (DOJ) dm = fmax(args.dmax[A * ns + B], args.dmax[C * ns + D]);
        if (DOK)
            dm = fmax(dm, fmax(fmax(args.dmax[B * ns + D], args.dmax[B * ns + C]),
                               fmax(args.dmax[A * ns + D], args.dmax[A * ns + C])));
        if (args.bra.Q[ib] * args.ket.Q[ik] * dm < args.dcut) return;
    }
    QuartetGeom g;
    load_xyz(args.bs, A, g.A);
    load_xyz(args.bs, B, g.B);
    load_xyz(args.bs, C, g.C);
    load_xyz(args.bs, D, g.D);
    double V[NA * NB * NC * ND];
    eri_block<LA, LB, LC, LD>(args.pp, args.bra.poff[ib], args.bra.np[ib], args.ket.poff[ik], args.ket.np[ik], g, V);
    double s = 1.0;
    if (A == B) s *= 0.5;
    if (C == D) s *= 0.5;
    if (args.same && ib == ik) s *= 0.5;
    const double uf = args.underflow;
    if (uf > 0.0) {
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int jb = 0; jb < NB; ++jb)
#pragma unroll
                for (int kc = 0; kc < NC; ++kc)
#pragma unroll
                    for (int ld = 0; ld < ND; ++ld) {
                        const int f = ((ia * NB + jb) * NC + kc) * ND + ld;
                        const double nn = comp_norm(LA, ia) * comp_norm(LB, jb) * comp_norm(LC, kc) * comp_norm(LD, ld);
                        if (fabs(V[f] * nn) <= uf) V[f] = 0.0;
                    }
    }
    const int n = args.n;
    const int oa = args.bs.sh_bf[A], ob = args.bs.sh_bf[B], oc = args.bs.sh_bf[C], od = args.bs.sh_bf[D];
    const double *__restrict__ Dm = args.D;
    if (DOJ) {
        const double s2 = 2.0 * s;
        double dcd[NC * ND];
#pragma unroll
        for (int kc = 0; kc < NC; ++kc)
#pragma unroll
            for (int ld = 0; ld < ND; ++ld) dcd[kc * ND + ld] = Dm[(oc + kc) * n + od + ld];
        double jcd[NC * ND];
#pragma unroll
        for (int i = 0; i < NC * ND; ++i) jcd[i] = 0.0;
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int jb = 0; jb < NB; ++jb) {
                const double dab = Dm[(oa + ia) * n + ob + jb];
                double jab = 0.0;
#pragma unroll
                for (int kl = 0; kl < NC * ND; ++kl) {
                    const double v = V[(ia * NB + jb) * NC * ND + kl];
                    jab += v * dcd[kl];
                    jcd[kl] += v * dab;
                }
                atomicAdd(&args.J[(oa + ia) * n + ob + jb], s2 * jab);
            }
#pragma unroll
        for (int kc = 0; kc < NC; ++kc)
#pragma unroll
            for (int ld = 0; ld < ND; ++ld) atomicAdd(&args.J[(oc + kc) * n + od + ld], s2 * jcd[kc * ND + ld]);
    }
    if (DOK) {
        // Kt[a][c] += s V Dbd ; Kt[a][d] += s V Dbc ; Kt[b][c] += s V Dad ; Kt[b][d] += s V Dac
#pragma unroll
        for (int ia = 0; ia < NA; ++ia) {
            double kac[NC], kad[ND];
#pragma unroll
            for (int i = 0; i < NC; ++i) kac[i] = 0.0;
#pragma unroll
            for (int i = 0; i < ND; ++i) kad[i] = 0.0;
#pragma unroll
            for (int jb = 0; jb < NB; ++jb) {
                double kbc[NC], kbd[ND];
#pragma unroll
                for (int i = 0; i < NC; ++i) kbc[i] = 0.0;
#pragma unroll
                for (int i = 0; i < ND; ++i) kbd[i] = 0.0;
#pragma unroll
                for (int kc = 0; kc < NC; ++kc) {
                    const double dbc = Dm[(ob + jb) * n + oc + kc];
                    const double dac = Dm[(oa + ia) * n + oc + kc];
#pragma unroll
                    for (int ld = 0; ld < ND; ++ld) {
                        const double v = V[((ia * NB + jb) * NC + kc) * ND + ld];
                        const double dbd = Dm[(ob + jb) * n + od + ld];
                        const double dad = Dm[(oa + ia) * n + od + ld];
                        kac[kc] += v * dbd;
                        kad[ld] += v * dbc;
                        kbc[kc] += v * dad;
                        kbd[ld] += v * dac;
                    }
                }
#pragma unroll
                for (int kc = 0; kc < NC; ++kc) atomicAdd(&args.K[(ob + jb) * n + oc + kc], s * kbc[kc]);
#pragma unroll
                for (int ld = 0; ld < ND; ++ld) atomicAdd(&args.K[(ob + jb) * n + od + ld], s * kbd[ld]);
            }
#pragma unroll
            for (int kc = 0; kc < NC; ++kc) atomicAdd(&args.K[(oa + ia) * n + oc + kc], s * kac[kc]);
#pragma unroll
            for (int ld = 0; ld < ND; ++ld) atomicAdd(&args.K[(oa + ia) * n + od + ld], s * kad[ld]);
        }
    }
}

constexpr int PLA[PDG_NPAIRCLASS] = {0, 1, 1, 2, 2, 2};
constexpr int PLB[PDG_NPAIRCLASS] = {0, 0, 1, 0, 1, 2};

template <int CB, int CK>
void launch_jk_t(const JKArgs &a, bool doJ, bool doK, cudaStream_t st) {
    constexpr int LA = PLA[CB], LB = PLB[CB], LC = PLA[CK], LD = PLB[CK];
    const int threads = 128;
    const long long blocks = (a.total + threads - 1) / threads;
    if (doJ && doK) { eri_jk_kernel<LA, LB, LC, LD, true, true><<<(unsigned)blocks, threads, 0, st>>>(a); pdg_count_launch(); }
    else if (doJ) { eri_jk_kernel<LA, LB, LC, LD, true, false><<<(unsigned)blocks, threads, 0, st>>>(a); pdg_count_launch(); }
    else { eri_jk_kernel<LA, LB, LC, LD, false, true><<<(unsigned)blocks, threads, 0, st>>>(a); pdg_count_launch(); }
}

typedef void (*jk_launcher)(const JKArgs &, bool, bool, cudaStream_t);

#define JKL(cb, ck) launch_jk_t<cb, ck>
const jk_launcher jk_table[PDG_NPAIRCLASS][PDG_NPAIRCLASS] = {
    {JKL(0, 0), nullptr, nullptr, nullptr, nullptr, nullptr},
    {JKL(1, 0), JKL(1, 1), nullptr, nullptr, nullptr, nullptr},
    {JKL(2, 0), JKL(2, 1), JKL(2, 2), nullptr, nullptr, nullptr},
    {JKL(3, 0), JKL(3, 1), JKL(3, 2), JKL(3, 3), nullptr, nullptr},
    {JKL(4, 0), JKL(4, 1), JKL(4, 2), JKL(4, 3), JKL(4, 4), nullptr},
    {JKL(5, 0), JKL(5, 1), JKL(5, 2), JKL(5, 3), JKL(5, 4), JKL(5, 5)},
};
#undef JKL

template <int C>
void launch_schwarz_t(int n, const int *shA, const int *shB, const int *poff, const int *np, const PrimPairs &pp,
                      const DeviceBasis &bs, double *Q, cudaStream_t st) {
    if (n == 0) return;
    { schwarz_kernel<PLA[C], PLB[C]><<<(n + 63) / 64, 64, 0, st>>>(n, shA, shB, poff, np, pp, bs, Q); pdg_count_launch(); }
}
typedef void (*schwarz_launcher)(int, const int *, const int *, const int *, const int *, const PrimPairs &,
                                 const DeviceBasis &, double *, cudaStream_t);
const schwarz_launcher schwarz_table[PDG_NPAIRCLASS] = {launch_schwarz_t<0>, launch_schwarz_t<1>, launch_schwarz_t<2>,
                                                        launch_schwarz_t<3>, launch_schwarz_t<4>, launch_schwarz_t<5>};

template <typename T>
int upload(T **dst, const std::vector<T> &src) {
    if (*dst) cudaFree(*dst);
    *dst = nullptr;
    if (src.empty()) return PDG_OK;
    PDG_CUDA(cudaMalloc(dst, src.size() * sizeof(T)));
    PDG_CUDA(cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice));
    return PDG_OK;
}

}  // namespace

void pdg_free_pairs(pdg_context *ctx) {
    for (int c = 0; c < PDG_NPAIRCLASS; ++c) {
        PairList &pl = ctx->pairs[c];
        cudaFree(pl.shA); cudaFree(pl.shB); cudaFree(pl.poff); cudaFree(pl.np); cudaFree(pl.Q);
        pl = PairList{};
    }
    PrimPairs &pp = ctx->pp;
    cudaFree(pp.a); cudaFree(pp.b); cudaFree(pp.Px); cudaFree(pp.Py); cudaFree(pp.Pz); cudaFree(pp.K); cudaFree(pp.arg);
    pp = PrimPairs{};
    for (auto &b : ctx->blocks) cudaFree(b.offs);
    ctx->blocks.clear();
    ctx->blocks_thr = -1.0;
}

// Build primitive-pair data and Schwarz-sorted shell-pair lists for the current geometry.
int pdg_ensure_pairs(pdg_context *ctx) {
    if (ctx->pairs[0].shA || ctx->pp.a) return PDG_OK;
    ProfScope prof(ctx, "pairs");
    const auto &sh = ctx->shells;
    const int ns = (int)sh.size();
    std::vector<int> cshA[PDG_NPAIRCLASS], cshB[PDG_NPAIRCLASS], cpoff[PDG_NPAIRCLASS], cnp[PDG_NPAIRCLASS];
    std::vector<double> va, vb, vPx, vPy, vPz, vK, varg;
    for (int i = 0; i < ns; ++i) {
        for (int j = 0; j <= i; ++j) {
            int A = i, B = j;
            if (sh[A].l < sh[B].l) std::swap(A, B);
            const double *rA = &ctx->xyz[3 * sh[A].atom], *rB = &ctx->xyz[3 * sh[B].atom];
            const double dx = rA[0] - rB[0], dy = rA[1] - rB[1], dz = rA[2] - rB[2];
            const double r2 = dx * dx + dy * dy + dz * dz;
            const int off = (int)va.size();
            for (int pa = 0; pa < sh[A].np; ++pa) {
                const double ea = ctx->prim_exp[sh[A].poff + pa], ca = ctx->prim_coef[sh[A].poff + pa];
                for (int pb = 0; pb < sh[B].np; ++pb) {
                    const double eb = ctx->prim_exp[sh[B].poff + pb], cb = ctx->prim_coef[sh[B].poff + pb];
                    const double p = ea + eb;
                    const double arg = ea * eb / p * r2;
                    if (arg > PDG_PRIMITIVE_CUT) continue;
                    va.push_back(ea);
                    vb.push_back(eb);
                    vPx.push_back((ea * rA[0] + eb * rB[0]) / p);
                    vPy.push_back((ea * rA[1] + eb * rB[1]) / p);
                    vPz.push_back((ea * rA[2] + eb * rB[2]) / p);
                    vK.push_back(std::exp(-arg) * ca * cb);
                    varg.push_back(arg);
                }
            }
            const int cnt = (int)va.size() - off;
            if (cnt == 0) continue;
            const int c = pair_class(sh[A].l, sh[B].l);
            cshA[c].push_back(A);
            cshB[c].push_back(B);
            cpoff[c].push_back(off);
            cnp[c].push_back(cnt);
        }
    }
    ctx->npp = (int)va.size();
    PDG_CHECK(upload(&ctx->pp.a, va));
    PDG_CHECK(upload(&ctx->pp.b, vb));
    PDG_CHECK(upload(&ctx->pp.Px, vPx));
    PDG_CHECK(upload(&ctx->pp.Py, vPy));
    PDG_CHECK(upload(&ctx->pp.Pz, vPz));
    PDG_CHECK(upload(&ctx->pp.K, vK));
    PDG_CHECK(upload(&ctx->pp.arg, varg));
    ctx->hostArg = varg;
    // Schwarz bounds on the unsorted lists, then sort each class by Q descending.
    for (int c = 0; c < PDG_NPAIRCLASS; ++c) {
        const int n = (int)cshA[c].size();
        ctx->hostQ[c].clear();
        ctx->qmax[c] = 0.0;
        if (n == 0) continue;
        int *dA = nullptr, *dB = nullptr, *dO = nullptr, *dN = nullptr;
        double *dQ = nullptr;
        PDG_CHECK(upload(&dA, cshA[c]));
        PDG_CHECK(upload(&dB, cshB[c]));
        PDG_CHECK(upload(&dO, cpoff[c]));
        PDG_CHECK(upload(&dN, cnp[c]));
        PDG_CUDA(cudaMalloc(&dQ, n * sizeof(double)));
        schwarz_table[c](n, dA, dB, dO, dN, ctx->pp, ctx->dbasis, dQ, ctx->stream);
        PDG_CUDA(cudaGetLastError());
        std::vector<double> Q(n);
        PDG_CUDA(cudaMemcpyAsync(Q.data(), dQ, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        PDG_CUDA(cudaStreamSynchronize(ctx->stream));
        cudaFree(dA); cudaFree(dB); cudaFree(dO); cudaFree(dN); cudaFree(dQ);
        std::vector<int> order(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return Q[x] > Q[y]; });
        std::vector<int> sA(n), sB(n), sO(n), sN(n);
        std::vector<double> sQ(n);
        for (int k = 0; k < n; ++k) {
            sA[k] = cshA[c][order[k]]; sB[k] = cshB[c][order[k]];
            sO[k] = cpoff[c][order[k]]; sN[k] = cnp[c][order[k]];
            sQ[k] = Q[order[k]];
        }
        PairList &pl = ctx->pairs[c];
        pl.n = n;
        PDG_CHECK(upload(&pl.shA, sA));
        PDG_CHECK(upload(&pl.shB, sB));
        PDG_CHECK(upload(&pl.poff, sO));
        PDG_CHECK(upload(&pl.np, sN));
        PDG_CHECK(upload(&pl.Q, sQ));
        ctx->hostQ[c] = sQ;
        ctx->hostPoff[c] = sO;
        ctx->hostNp[c] = sN;
        ctx->qmax[c] = sQ[0];
    }
    return PDG_OK;
}

// Screened work list: for each (bra class >= ket class) block, prefix sums over bra pairs of
// the number of ket pairs with Q_bra * Q_ket >= thr (and ket <= bra inside one class).
int pdg_build_blocks(pdg_context *ctx, double thr) {
    if (ctx->blocks_thr == thr && !ctx->blocks.empty()) return PDG_OK;
    for (auto &b : ctx->blocks) cudaFree(b.offs);
    ctx->blocks.clear();
    for (int cb = 0; cb < PDG_NPAIRCLASS; ++cb) {
        const auto &Qb = ctx->hostQ[cb];
        if (Qb.empty()) continue;
        for (int ck = 0; ck <= cb; ++ck) {
            const auto &Qk = ctx->hostQ[ck];
            if (Qk.empty()) continue;
            std::vector<long long> offs(Qb.size() + 1, 0);
            for (size_t i = 0; i < Qb.size(); ++i) {
                long long cnt = 0;
                if (Qb[i] > 0.0) {
                    const double need = thr / Qb[i];
                    // Qk sorted descending: count entries >= need
                    cnt = std::upper_bound(Qk.begin(), Qk.end(), need, [](double v, double e) { return v > e; }) - Qk.begin();
                    // entries with Qk[k] >= need: upper_bound with comparator (v > e) finds first e < need
                }
                if (cb == ck) cnt = std::min<long long>(cnt, (long long)i + 1);
                offs[i + 1] = offs[i] + cnt;
            }
            QuartetBlock qb{cb, ck, offs.back(), nullptr};
            if (qb.total == 0) continue;
            PDG_CHECK(upload(&qb.offs, offs));
            ctx->blocks.push_back(qb);
        }
    }
    ctx->blocks_thr = thr;
    return PDG_OK;
}

// Largest |D'| over each shell-pair block (nshell x nshell, symmetric), for density screening.
__global__ void shell_pair_dmax_kernel(int ns, int n, const int *__restrict__ sh_bf, const int *__restrict__ sh_l,
                                       const double *__restrict__ D, double *__restrict__ dmax) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ns * ns) return;
    const int a = t / ns, b = t - a * ns;
    const int oa = sh_bf[a], ob = sh_bf[b], na = ncart(sh_l[a]), nb = ncart(sh_l[b]);
    double m = 0.0;
    for (int i = 0; i < na; ++i)
        for (int j = 0; j < nb; ++j) m = fmax(m, fabs(D[(long long)(oa + i) * n + ob + j]));
    dmax[t] = m;
}

int pdg_shell_pair_dmax(pdg_context *ctx, const double *d_D, double *d_dmax) {
    const int ns = (int)ctx->shells.size();
    { shell_pair_dmax_kernel<<<(ns * ns + 127) / 128, 128, 0, ctx->stream>>>(ns, ctx->nbf, ctx->dbasis.sh_bf, ctx->dbasis.sh_l, d_D, d_dmax); pdg_count_launch(); }
    PDG_CUDA(cudaGetLastError());
    return PDG_OK;
}

int pdg_eri_jk(pdg_context *ctx, const double *d_D, double *d_J, double *d_K, bool doJ, bool doK) {
    return pdg_eri_jk_screened(ctx, d_D, d_J, d_K, doJ, doK, nullptr, 0.0);
}

int pdg_eri_jk_screened(pdg_context *ctx, const double *d_D, double *d_J, double *d_K, bool doJ, bool doK,
                        const double *d_dmax, double dcut) {
    PDG_CHECK(pdg_ensure_pairs(ctx));
    PDG_CHECK(pdg_build_blocks(ctx, ctx->schwarz_cut));
    long long nq = 0;
    ProfScope prof(ctx, "eri_jk");
    for (const auto &b : ctx->blocks) {
        JKArgs a;
        a.bra = ctx->pairs[b.cb];
        a.ket = ctx->pairs[b.ck];
        a.offs = b.offs;
        a.total = b.total;
        a.same = (b.cb == b.ck);
        a.pp = ctx->pp;
        a.bs = ctx->dbasis;
        a.D = d_D;
        a.J = d_J;
        a.K = d_K;
        a.n = ctx->nbf;
        a.underflow = ctx->tei_underflow;
        a.dmax = d_dmax;
        a.nshell = (int)ctx->shells.size();
        a.dcut = dcut;
        jk_table[b.cb][b.ck](a, doJ, doK, ctx->stream);
        PDG_CUDA(cudaGetLastError());
        nq += b.total;
    }
    ctx->last_quartets = nq;
    return PDG_OK;
}
