// Two-electron gradient: derivative Rys shell-quartet kernels contracted on the fly with
//   Gamma_abcd = 4 s [ D'ab D'cd - (c_x/4)(D'ac D'bd + D'ad D'bc) ]
// and reduced to atom gradients (centre D by translational invariance).
//
// Replaces GaussianBasisContainerIntegrals_f2Cf2R1 + ProcessTEIsD
// (GaussianBases/__extensions__/csource/GaussianBasisContainerIntegrals_f2Xf2.c:146-209,337-421)
// and GaussianBasisIntegrals_f2Cf2r1 (GaussianBasisIntegrals_f2Xf2.c:905-1364), whose density
// factor 4 s D D - s c_x (D D + D D) is the same Gamma.
#include "context.h"
#include "rys.cuh"
#include "rys2d.cuh"

namespace {

constexpr double TWO_PI_POW_2P5 = 34.986836655249725;

struct GradArgs {
    PairList bra, ket;
    const long long *offs;
    long long total;
    int same;
    PrimPairs pp;
    DeviceBasis bs;
    const double *D;
    double cx;
    int doJ;
    double *grad;
    int n;
};

// Transfers for derivatives: I[a][b][c][d] valid for a+b <= LA+LB+1 and c+d <= LC+LD+1,
// b <= LB+1, d <= LD.
template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ void grad_hrr(const double (&G)[LA + LB + 2][LC + LD + 2], double AB, double CD,
                                         double (&I)[LA + 2][LB + 2][LC + 2][LD + 1]) {
    constexpr int LAB = LA + LB + 1, LCD = LC + LD + 1;
    double T[LAB + 1][LB + 2][LCD + 1];
#pragma unroll
    for (int a = 0; a <= LAB; ++a)
#pragma unroll
        for (int f = 0; f <= LCD; ++f) T[a][0][f] = G[a][f];
#pragma unroll
    for (int b = 1; b <= LB + 1; ++b)
#pragma unroll
        for (int a = 0; a <= LAB - b; ++a)
#pragma unroll
            for (int f = 0; f <= LCD; ++f) T[a][b][f] = T[a + 1][b - 1][f] + AB * T[a][b - 1][f];
    double U[LA + 2][LB + 2][LCD + 1][LD + 1];
#pragma unroll
    for (int a = 0; a <= LA + 1; ++a)
#pragma unroll
        for (int b = 0; b <= LB + 1; ++b) {
            if (a + b > LAB) continue;
#pragma unroll
            for (int c = 0; c <= LCD; ++c) U[a][b][c][0] = T[a][b][c];
        }
#pragma unroll
    for (int d = 1; d <= LD; ++d)
#pragma unroll
        for (int a = 0; a <= LA + 1; ++a)
#pragma unroll
            for (int b = 0; b <= LB + 1; ++b) {
                if (a + b > LAB) continue;
#pragma unroll
                for (int c = 0; c <= LCD - d; ++c) U[a][b][c][d] = U[a][b][c + 1][d - 1] + CD * U[a][b][c][d - 1];
            }
#pragma unroll
    for (int a = 0; a <= LA + 1; ++a)
#pragma unroll
        for (int b = 0; b <= LB + 1; ++b) {
            if (a + b > LAB) continue;
#pragma unroll
            for (int c = 0; c <= LC + 1; ++c)
#pragma unroll
                for (int d = 0; d <= LD; ++d) {
                    if (c + d > LCD) continue;
                    I[a][b][c][d] = U[a][b][c][d];
                }
        }
}

template <int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(128) eri_grad_kernel(GradArgs args) {
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
    constexpr int LAB = LA + LB + 1, LCD = LC + LD + 1, NR = (LAB + LCD) / 2 + 1;
    const int A = args.bra.shA[ib], B = args.bra.shB[ib], C = args.ket.shA[ik], D = args.ket.shB[ik];
    const int atA = args.bs.sh_atom[A], atB = args.bs.sh_atom[B], atC = args.bs.sh_atom[C], atD = args.bs.sh_atom[D];
    if (atA == atB && atA == atC && atA == atD) return;  // one-centre quartets have no gradient
    double rA[3], rB[3], rC[3], rD[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        rA[k] = args.bs.atom_xyz[3 * atA + k]; rB[k] = args.bs.atom_xyz[3 * atB + k];
        rC[k] = args.bs.atom_xyz[3 * atC + k]; rD[k] = args.bs.atom_xyz[3 * atD + k];
    }
    double s = 1.0;
    if (A == B) s *= 0.5;
    if (C == D) s *= 0.5;
    if (args.same && ib == ik) s *= 0.5;
    const int n = args.n;
    const int oa = args.bs.sh_bf[A], ob = args.bs.sh_bf[B], oc = args.bs.sh_bf[C], od = args.bs.sh_bf[D];
    const double *__restrict__ Dm = args.D;
    const double cj = args.doJ ? 4.0 * s : 0.0, ck = -s * args.cx;
    double Gam[NA * NB * NC * ND];
#pragma unroll
    for (int ia = 0; ia < NA; ++ia)
#pragma unroll
        for (int jb = 0; jb < NB; ++jb) {
            const double dab = Dm[(oa + ia) * n + ob + jb];
#pragma unroll
            for (int kc = 0; kc < NC; ++kc) {
                const double dac = Dm[(oa + ia) * n + oc + kc], dbc = Dm[(ob + jb) * n + oc + kc];
#pragma unroll
                for (int ld = 0; ld < ND; ++ld) {
                    const double dcd = Dm[(oc + kc) * n + od + ld];
                    const double dbd = Dm[(ob + jb) * n + od + ld], dad = Dm[(oa + ia) * n + od + ld];
                    Gam[((ia * NB + jb) * NC + kc) * ND + ld] = cj * dab * dcd + ck * (dac * dbd + dad * dbc);
                }
            }
        }
    const double ABx = rA[0] - rB[0], ABy = rA[1] - rB[1], ABz = rA[2] - rB[2];
    const double CDx = rC[0] - rD[0], CDy = rC[1] - rD[1], CDz = rC[2] - rD[2];
    double g[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) g[k] = 0.0;
    const PrimPairs &pp = args.pp;
    const int pb0 = args.bra.poff[ib], npb = args.bra.np[ib], pk0 = args.ket.poff[ik], npk = args.ket.np[ik];
    for (int jb_ = pb0; jb_ < pb0 + npb; ++jb_) {
        const double ea = pp.a[jb_], eb = pp.b[jb_], p = ea + eb;
        const double Px = pp.Px[jb_], Py = pp.Py[jb_], Pz = pp.Pz[jb_];
        const double Kb = pp.K[jb_], argb = pp.arg[jb_];
        const double PAx = Px - rA[0], PAy = Py - rA[1], PAz = Pz - rA[2];
        for (int jk = pk0; jk < pk0 + npk; ++jk) {
            const double argk = pp.arg[jk];
            if (argb + argk > PDG_PRIMITIVE_CUT) continue;
            const double ec = pp.a[jk], ed = pp.b[jk], q = ec + ed;
            const double Qx = pp.Px[jk], Qy = pp.Py[jk], Qz = pp.Pz[jk];
            const double pq = p * q, ppq = p + q, rppq = 1.0 / ppq;
            const double PQx = Px - Qx, PQy = Py - Qy, PQz = Pz - Qz;
            const double x = pq * rppq * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pref = TWO_PI_POW_2P5 / (pq * sqrt(ppq)) * Kb * pp.K[jk];
            double u[NR], w[NR];
            rys_roots<NR>(x, u, w);
            const double QCx = Qx - rC[0], QCy = Qy - rC[1], QCz = Qz - rC[2];
            const double r2p = 0.5 / p, r2q = 0.5 / q;
            const double a2 = 2.0 * ea, b2 = 2.0 * eb, c2 = 2.0 * ec;
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const double ur = u[r] * rppq;
                const double b00 = 0.5 * ur, b10 = r2p * (1.0 - q * ur), b01 = r2q * (1.0 - p * ur);
                const double fq = q * ur, fp = p * ur;
                double Gx[LAB + 1][LCD + 1], Gy[LAB + 1][LCD + 1], Gz[LAB + 1][LCD + 1];
                rys_vrr<LAB, LCD>(Gx, 1.0, PAx - fq * PQx, QCx + fp * PQx, b10, b01, b00);
                rys_vrr<LAB, LCD>(Gy, 1.0, PAy - fq * PQy, QCy + fp * PQy, b10, b01, b00);
                rys_vrr<LAB, LCD>(Gz, w[r] * pref, PAz - fq * PQz, QCz + fp * PQz, b10, b01, b00);
                double Ix[LA + 2][LB + 2][LC + 2][LD + 1], Iy[LA + 2][LB + 2][LC + 2][LD + 1], Iz[LA + 2][LB + 2][LC + 2][LD + 1];
                grad_hrr<LA, LB, LC, LD>(Gx, ABx, CDx, Ix);
                grad_hrr<LA, LB, LC, LD>(Gy, ABy, CDy, Iy);
                grad_hrr<LA, LB, LC, LD>(Gz, ABz, CDz, Iz);
#pragma unroll
                for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                    for (int jb = 0; jb < NB; ++jb)
#pragma unroll
                        for (int kc = 0; kc < NC; ++kc)
#pragma unroll
                            for (int ld = 0; ld < ND; ++ld) {
                                const double gm = Gam[((ia * NB + jb) * NC + kc) * ND + ld];
                                const int ax = cart_x(LA, ia), ay = cart_y(LA, ia), az = cart_z(LA, ia);
                                const int bx = cart_x(LB, jb), by = cart_y(LB, jb), bz = cart_z(LB, jb);
                                const int cxx = cart_x(LC, kc), cy = cart_y(LC, kc), cz = cart_z(LC, kc);
                                const int dx = cart_x(LD, ld), dy = cart_y(LD, ld), dz = cart_z(LD, ld);
                                const double x0 = Ix[ax][bx][cxx][dx], y0 = Iy[ay][by][cy][dy], z0 = Iz[az][bz][cz][dz];
                                const double gy = gm * y0 * z0, gx = gm * x0 * z0, gz = gm * x0 * y0;
                                // centre A
                                g[0] += gy * (a2 * Ix[ax + 1][bx][cxx][dx] - (ax ? ax * Ix[ax ? ax - 1 : 0][bx][cxx][dx] : 0.0));
                                g[1] += gx * (a2 * Iy[ay + 1][by][cy][dy] - (ay ? ay * Iy[ay ? ay - 1 : 0][by][cy][dy] : 0.0));
                                g[2] += gz * (a2 * Iz[az + 1][bz][cz][dz] - (az ? az * Iz[az ? az - 1 : 0][bz][cz][dz] : 0.0));
                                // centre B
                                g[3] += gy * (b2 * Ix[ax][bx + 1][cxx][dx] - (bx ? bx * Ix[ax][bx ? bx - 1 : 0][cxx][dx] : 0.0));
                                g[4] += gx * (b2 * Iy[ay][by + 1][cy][dy] - (by ? by * Iy[ay][by ? by - 1 : 0][cy][dy] : 0.0));
                                g[5] += gz * (b2 * Iz[az][bz + 1][cz][dz] - (bz ? bz * Iz[az][bz ? bz - 1 : 0][cz][dz] : 0.0));
                                // centre C
                                g[6] += gy * (c2 * Ix[ax][bx][cxx + 1][dx] - (cxx ? cxx * Ix[ax][bx][cxx ? cxx - 1 : 0][dx] : 0.0));
                                g[7] += gx * (c2 * Iy[ay][by][cy + 1][dy] - (cy ? cy * Iy[ay][by][cy ? cy - 1 : 0][dy] : 0.0));
                                g[8] += gz * (c2 * Iz[az][bz][cz + 1][dz] - (cz ? cz * Iz[az][bz][cz ? cz - 1 : 0][dz] : 0.0));
                            }
            }
        }
    }
    double *gr = args.grad;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        atomicAdd(&gr[3 * atA + k], g[k]);
        atomicAdd(&gr[3 * atB + k], g[3 + k]);
        atomicAdd(&gr[3 * atC + k], g[6 + k]);
        atomicAdd(&gr[3 * atD + k], -(g[k] + g[3 + k] + g[6 + k]));
    }
}

constexpr int PLA[PDG_NPAIRCLASS] = {0, 1, 1, 2, 2, 2};
constexpr int PLB[PDG_NPAIRCLASS] = {0, 0, 1, 0, 1, 2};

template <int CB, int CK>
void launch_grad_t(const GradArgs &a, cudaStream_t st) {
    const int threads = 128;
    const long long blocks = (a.total + threads - 1) / threads;
    { eri_grad_kernel<PLA[CB], PLB[CB], PLA[CK], PLB[CK]><<<(unsigned)blocks, threads, 0, st>>>(a); pdg_count_launch(); }
}
typedef void (*grad_launcher)(const GradArgs &, cudaStream_t);
#define GL(cb, ck) launch_grad_t<cb, ck>
const grad_launcher grad_table[PDG_NPAIRCLASS][PDG_NPAIRCLASS] = {
    {GL(0, 0), nullptr, nullptr, nullptr, nullptr, nullptr},
    {GL(1, 0), GL(1, 1), nullptr, nullptr, nullptr, nullptr},
    {GL(2, 0), GL(2, 1), GL(2, 2), nullptr, nullptr, nullptr},
    {GL(3, 0), GL(3, 1), GL(3, 2), GL(3, 3), nullptr, nullptr},
    {GL(4, 0), GL(4, 1), GL(4, 2), GL(4, 3), GL(4, 4), nullptr},
    {GL(5, 0), GL(5, 1), GL(5, 2), GL(5, 3), GL(5, 4), GL(5, 5)},
};
#undef GL

}  // namespace

int pdg_eri_grad(pdg_context *ctx, const double *d_D, double cx, bool doJ, double *d_grad) {
    PDG_CHECK(pdg_ensure_pairs(ctx));
    PDG_CHECK(pdg_build_blocks(ctx, ctx->schwarz_cut));
    ProfScope prof(ctx, "eri_grad");
    for (const auto &b : ctx->blocks) {
        GradArgs a;
        a.bra = ctx->pairs[b.cb];
        a.ket = ctx->pairs[b.ck];
        a.offs = b.offs;
        a.total = b.total;
        a.same = (b.cb == b.ck);
        a.pp = ctx->pp;
        a.bs = ctx->dbasis;
        a.D = d_D;
        a.cx = cx;
        a.doJ = doJ ? 1 : 0;
        a.grad = d_grad;
        a.n = ctx->nbf;
        grad_table[b.cb][b.ck](a, ctx->stream);
        PDG_CUDA(cudaGetLastError());
    }
    return PDG_OK;
}
