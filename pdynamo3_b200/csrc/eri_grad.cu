// Two-electron gradient: derivative Rys shell-quartet kernels contracted on the fly with
//   Gamma_abcd = 4 s [ D'ab D'cd - (c_x/4)(D'ac D'bd + D'ad D'bc) ]
// and reduced to atom gradients (centre D by translational invariance).
//
// Replaces GaussianBasisContainerIntegrals_f2Cf2R1 + ProcessTEIsD
// (GaussianBases/__extensions__/csource/GaussianBasisContainerIntegrals_f2Xf2.c:146-209,337-421)
// and GaussianBasisIntegrals_f2Cf2r1 (GaussianBasisIntegrals_f2Xf2.c:905-1364), whose density
// factor 4 s D D - s c_x (D D + D D) is the same Gamma.
#include <type_traits>

#include "context.h"
#include "rys.cuh"
#include "rys2d.cuh"

namespace {

constexpr double TWO_PI_POW_2P5 = 34.986836655249725;

struct GradArgs {
    PairList bra, ket;
    WorkList work;       // the quartets: per ket bucket, prefix sums over bra pairs and the bra map
    int same;
    PrimPairs pp;
    DeviceBasis bs;
    const double *D;
    double cx;
    int doJ;
    double *grad;
    int n;
    const double *dmax;  // optional (mixed mode): max |D'| per shell-pair block, nshell x nshell
    int nshell;
    double gcut;         // skip a quartet when Q_AB Q_CD |Gamma|max < gcut
    int part;            // 0: every quartet; 1: bound >= mixed_cut (FP64); 2: bound < mixed_cut (FP32)
    double mixed_cut;
};

// Largest |Gamma| of a quartet from the shell-pair density maxima:
// |4 s [D_ab D_cd - (c_x/4)(D_ac D_bd + D_ad D_bc)]| <= 4 D_AB D_CD + |c_x| (D_AC D_BD + D_AD D_BC).
__device__ __forceinline__ bool grad_skip(const GradArgs &a, int ib, int ik, int A, int B, int C, int D) {
    if (!a.dmax) return false;
    const int ns = a.nshell;
    const double *m = a.dmax;
    const double gam = (a.doJ ? 4.0 * m[A * ns + B] * m[C * ns + D] : 0.0) +
                       fabs(a.cx) * (m[A * ns + C] * m[B * ns + D] + m[A * ns + D] * m[B * ns + C]);
    const double bound = a.bra.Q[ib] * a.ket.Q[ik] * gam;
    if (bound < a.gcut) return true;
    if (a.part == 1) return bound < a.mixed_cut;
    if (a.part == 2) return bound >= a.mixed_cut;
    return false;
}

// Transfers for derivatives: I[a][b][c][d] valid for a+b <= LA+LB+1 and c+d <= LC+LD+1,
// b <= LB+1, d <= LD.
template <int LA, int LB, int LC, int LD, typename R = double>
__device__ __forceinline__ void grad_hrr(const R (&G)[LA + LB + 2][LC + LD + 2], R AB, R CD,
                                         R (&I)[LA + 2][LB + 2][LC + 2][LD + 1]) {
    constexpr int LAB = LA + LB + 1, LCD = LC + LD + 1;
    R T[LAB + 1][LB + 2][LCD + 1];
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
    R U[LA + 2][LB + 2][LCD + 1][LD + 1];
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

// One shell quartet per P lanes (P = the ket bucket's lane count): the lanes split the primitive
// quartets and add their nine centre derivatives with shuffles before the first lane adds them to the
// atom gradients.  T is the arithmetic type of the primitive quartets (float for the quartets of the
// mixed mode whose Schwarz x |Gamma| bound is below the mixed cut): the centre differences and Gamma
// are formed in double and rounded once, the Boys argument, Rys rule, recursions, transfers and the
// accumulation run in T.
template <int LA, int LB, int LC, int LD, typename T = double>
__global__ void __launch_bounds__(128) eri_grad_kernel(GradArgs args) {
    const WorkSub ws = pick_sub(args.work);
    const int P = ws.lanes;
    const long long t = ((long long)blockIdx.x - ws.cta0) * blockDim.x / P + (long long)(threadIdx.x / P);
    const int lane = (int)(threadIdx.x & (P - 1));
    const int ib = bra_of(ws.offs, ws.cbra, min(t, ws.total - 1));
    if (t >= ws.total) return;
    const int ik = ws.k0 + (int)(t - ws.offs[ib]);
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    constexpr int LAB = LA + LB + 1, LCD = LC + LD + 1, NR = (LAB + LCD) / 2 + 1;
    const int A = args.bra.shA[ib], B = args.bra.shB[ib], C = args.ket.shA[ik], D = args.ket.shB[ik];
    const int atA = args.bs.sh_atom[A], atB = args.bs.sh_atom[B], atC = args.bs.sh_atom[C], atD = args.bs.sh_atom[D];
    if (atA == atB && atA == atC && atA == atD) return;  // one-centre quartets have no gradient
    if (grad_skip(args, ib, ik, A, B, C, D)) return;
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
    const T ABx = T(rA[0] - rB[0]), ABy = T(rA[1] - rB[1]), ABz = T(rA[2] - rB[2]);
    const T CDx = T(rC[0] - rD[0]), CDy = T(rC[1] - rD[1]), CDz = T(rC[2] - rD[2]);
    T g[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) g[k] = T(0);
    const PrimPairs &pp = args.pp;
    const int pb0 = args.bra.poff[ib], npb = args.bra.np[ib], pk0 = args.ket.poff[ik], npk = args.ket.np[ik];
    // primitive quartet idx = b npk + k, stepped by P without a division per step
    int sb = lane / npk, sk = lane - sb * npk;
    for (int idx = lane; idx < npb * npk; idx += P, sk += P) {
        while (sk >= npk) { sk -= npk; ++sb; }
        const int jb_ = pb0 + sb, jk = pk0 + sk;
        // the cut arguments and the first exponents of both pairs in two 16-byte loads
        const double2 xb = load_arg_a(pp.rec, jb_), xk = load_arg_a(pp.rec, jk);
        if (xb.x + xk.x > PDG_PRIMITIVE_CUT) continue;
        const PairRec Rb = load_rec(pp.rec, jb_), Rk = load_rec(pp.rec, jk);
        const T ea = T(xb.y), eb = T(Rb.p - xb.y), p = T(Rb.p);
        const T PAx = T(Rb.Px - rA[0]), PAy = T(Rb.Py - rA[1]), PAz = T(Rb.Pz - rA[2]);
        {
            const T ec = T(xk.y), q = T(Rk.p);
            T rs;
            if constexpr (std::is_same<T, float>::value) rs = rsqrtf(p + q);
            else rs = rsqrt(p + q);
            const T rppq = rs * rs;
            const T PQx = T(Rb.Px - Rk.Px), PQy = T(Rb.Py - Rk.Py), PQz = T(Rb.Pz - Rk.Pz);
            const T x = p * q * rppq * (PQx * PQx + PQy * PQy + PQz * PQz);
            const T pref = T(TWO_PI_POW_2P5) * rs * T(Rb.Kp) * T(Rk.Kp);
            T u[NR], w[NR];
            if constexpr (std::is_same<T, float>::value) rys_roots_f<NR>(x, u, w);
            else rys_roots<NR>(x, u, w);
            const T QCx = T(Rk.Px - rC[0]), QCy = T(Rk.Py - rC[1]), QCz = T(Rk.Pz - rC[2]);
            const T r2p = T(Rb.hp), r2q = T(Rk.hp);
            const T a2 = T(2) * ea, b2 = T(2) * eb, c2 = T(2) * ec;
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const T ur = u[r] * rppq;
                const T b00 = T(0.5) * ur, b10 = r2p * (T(1) - q * ur), b01 = r2q * (T(1) - p * ur);
                const T fq = q * ur, fp = p * ur;
                T Gx[LAB + 1][LCD + 1], Gy[LAB + 1][LCD + 1], Gz[LAB + 1][LCD + 1];
                rys_vrr<LAB, LCD, T>(Gx, T(1), PAx - fq * PQx, QCx + fp * PQx, b10, b01, b00);
                rys_vrr<LAB, LCD, T>(Gy, T(1), PAy - fq * PQy, QCy + fp * PQy, b10, b01, b00);
                rys_vrr<LAB, LCD, T>(Gz, w[r] * pref, PAz - fq * PQz, QCz + fp * PQz, b10, b01, b00);
                T Ix[LA + 2][LB + 2][LC + 2][LD + 1], Iy[LA + 2][LB + 2][LC + 2][LD + 1], Iz[LA + 2][LB + 2][LC + 2][LD + 1];
                grad_hrr<LA, LB, LC, LD, T>(Gx, ABx, CDx, Ix);
                grad_hrr<LA, LB, LC, LD, T>(Gy, ABy, CDy, Iy);
                grad_hrr<LA, LB, LC, LD, T>(Gz, ABz, CDz, Iz);
#pragma unroll
                for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                    for (int jb = 0; jb < NB; ++jb)
#pragma unroll
                        for (int kc = 0; kc < NC; ++kc)
#pragma unroll
                            for (int ld = 0; ld < ND; ++ld) {
                                const T gm = T(Gam[((ia * NB + jb) * NC + kc) * ND + ld]);
                                const int ax = cart_x(LA, ia), ay = cart_y(LA, ia), az = cart_z(LA, ia);
                                const int bx = cart_x(LB, jb), by = cart_y(LB, jb), bz = cart_z(LB, jb);
                                const int cxx = cart_x(LC, kc), cy = cart_y(LC, kc), cz = cart_z(LC, kc);
                                const int dx = cart_x(LD, ld), dy = cart_y(LD, ld), dz = cart_z(LD, ld);
                                const T x0 = Ix[ax][bx][cxx][dx], y0 = Iy[ay][by][cy][dy], z0 = Iz[az][bz][cz][dz];
                                const T gy = gm * y0 * z0, gx = gm * x0 * z0, gz = gm * x0 * y0;
                                // centre A
                                g[0] += gy * (a2 * Ix[ax + 1][bx][cxx][dx] - (ax ? ax * Ix[ax ? ax - 1 : 0][bx][cxx][dx] : T(0)));
                                g[1] += gx * (a2 * Iy[ay + 1][by][cy][dy] - (ay ? ay * Iy[ay ? ay - 1 : 0][by][cy][dy] : T(0)));
                                g[2] += gz * (a2 * Iz[az + 1][bz][cz][dz] - (az ? az * Iz[az ? az - 1 : 0][bz][cz][dz] : T(0)));
                                // centre B
                                g[3] += gy * (b2 * Ix[ax][bx + 1][cxx][dx] - (bx ? bx * Ix[ax][bx ? bx - 1 : 0][cxx][dx] : T(0)));
                                g[4] += gx * (b2 * Iy[ay][by + 1][cy][dy] - (by ? by * Iy[ay][by ? by - 1 : 0][cy][dy] : T(0)));
                                g[5] += gz * (b2 * Iz[az][bz + 1][cz][dz] - (bz ? bz * Iz[az][bz ? bz - 1 : 0][cz][dz] : T(0)));
                                // centre C
                                g[6] += gy * (c2 * Ix[ax][bx][cxx + 1][dx] - (cxx ? cxx * Ix[ax][bx][cxx ? cxx - 1 : 0][dx] : T(0)));
                                g[7] += gx * (c2 * Iy[ay][by][cy + 1][dy] - (cy ? cy * Iy[ay][by][cy ? cy - 1 : 0][dy] : T(0)));
                                g[8] += gz * (c2 * Iz[az][bz][cz + 1][dz] - (cz ? cz * Iz[az][bz][cz ? cz - 1 : 0][dz] : T(0)));
                            }
            }
        }
    }
    double gd[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) gd[k] = (double)g[k];
    if (P > 1) {
        const unsigned mask = lane_group_mask(P);
        for (int o = P >> 1; o > 0; o >>= 1) {
#pragma unroll
            for (int k = 0; k < 9; ++k) gd[k] += __shfl_xor_sync(mask, gd[k], o);
        }
        if (lane != 0) return;
    }
    double *gr = args.grad;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        atomicAdd(&gr[3 * atA + k], gd[k]);
        atomicAdd(&gr[3 * atB + k], gd[3 + k]);
        atomicAdd(&gr[3 * atC + k], gd[6 + k]);
        atomicAdd(&gr[3 * atD + k], -(gd[k] + gd[3 + k] + gd[6 + k]));
    }
}

// ---------------------------------------------------------------------------------------------
// Cooperative form for the d-shell classes (the one-thread form spills 5-116 KB per thread):
// G lanes share one shell quartet.  Lanes split the (root, direction) tasks of each primitive
// quartet (one Rys node, the 2D recursion to L+1 and the closed-form transfers into shared
// memory, indices a <= la+1, b <= lb+1, c <= lc+1, d <= ld); each lane owns bra rows (a,b) with
// all (c,d) and their Gamma values in registers, and accumulates the nine centre derivatives;
// the group reduces them with shuffles and one lane adds them to the atom gradients.
// ---------------------------------------------------------------------------------------------
__host__ __device__ constexpr int binom_small(int n, int k) { return (k == 0 || k == n) ? 1 : (n == 2 ? 2 : n); }

template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ void grad_hrr_store(const double (&Gm)[LA + LB + 2][LC + LD + 2], double AB, double CD,
                                               double *__restrict__ out) {
    constexpr int LAB = LA + LB + 1, LCD = LC + LD + 1;
    double abp[LB + 2], cdp[LD + 1];
    abp[0] = 1.0;
#pragma unroll
    for (int k = 1; k <= LB + 1; ++k) abp[k] = abp[k - 1] * AB;
    cdp[0] = 1.0;
#pragma unroll
    for (int k = 1; k <= LD; ++k) cdp[k] = cdp[k - 1] * CD;
#pragma unroll
    for (int a = 0; a <= LA + 1; ++a)
#pragma unroll
        for (int b = 0; b <= LB + 1; ++b) {
            if (a + b > LAB) continue;
            double row[LCD + 1];
#pragma unroll
            for (int f = 0; f <= LCD; ++f) {
                double s = Gm[a + b][f];
#pragma unroll
                for (int k = 0; k < b; ++k) s += binom_small(b, k) * abp[b - k] * Gm[a + k][f];
                row[f] = s;
            }
#pragma unroll
            for (int c = 0; c <= LC + 1; ++c)
#pragma unroll
                for (int d = 0; d <= LD; ++d) {
                    if (c + d > LCD) continue;
                    double s = row[c + d];
#pragma unroll
                    for (int m = 0; m < d; ++m) s += binom_small(d, m) * cdp[d - m] * row[c + m];
                    out[((a * (LB + 2) + b) * (LC + 2) + c) * (LD + 1) + d] = s;
                }
        }
}

template <int LA, int LB, int LC, int LD, int G>
struct GradShape {
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    static constexpr int NCD = NC * ND;
    static constexpr int NR = (LA + LB + LC + LD + 2) / 2 + 1;
    static constexpr int SC = LD + 1, SB = (LC + 2) * SC, SA = (LB + 2) * SB;
    static constexpr int NI = (LA + 2) * SA;
    static constexpr int R = NA * NB;
    static constexpr int FR = R / G;
    static constexpr int LR = R - FR * G;
    static constexpr int NUNIT = LR * NC;
    static constexpr int NU = (NUNIT + G - 1) / G;
    static constexpr int NIP = NI | 1;        // odd stride between the task arrays: distinct banks
    static constexpr int SMEM = 3 * NR * NIP; // doubles per group
    static constexpr int GPB = 128 / G;
};

// Nine centre-derivative contributions of one component (a,b,c,d) for one root; X, Y, Z point at
// the (a,b) row of the three direction arrays, off* at the (c,d) element.
template <int LA, int LB, int LC, int LD, int G>
__device__ __forceinline__ void grad_component(const double *__restrict__ X, const double *__restrict__ Y,
                                               const double *__restrict__ Z, int offx, int offy, int offz, int ax,
                                               int ay, int az, int bx, int by, int bz, int cxx, int cy, int cz, double gm,
                                               double a2, double b2, double c2, double (&g)[9]) {
    using S = GradShape<LA, LB, LC, LD, G>;
    const double x0 = X[offx], y0 = Y[offy], z0 = Z[offz];
    const double tyz = gm * y0 * z0, txz = gm * x0 * z0, txy = gm * x0 * y0;
    g[0] += tyz * (a2 * X[offx + S::SA] - ax * X[ax ? offx - S::SA : offx]);
    g[1] += txz * (a2 * Y[offy + S::SA] - ay * Y[ay ? offy - S::SA : offy]);
    g[2] += txy * (a2 * Z[offz + S::SA] - az * Z[az ? offz - S::SA : offz]);
    g[3] += tyz * (b2 * X[offx + S::SB] - bx * X[bx ? offx - S::SB : offx]);
    g[4] += txz * (b2 * Y[offy + S::SB] - by * Y[by ? offy - S::SB : offy]);
    g[5] += txy * (b2 * Z[offz + S::SB] - bz * Z[bz ? offz - S::SB : offz]);
    g[6] += tyz * (c2 * X[offx + S::SC] - cxx * X[cxx ? offx - S::SC : offx]);
    g[7] += txz * (c2 * Y[offy + S::SC] - cy * Y[cy ? offy - S::SC : offy]);
    g[8] += txy * (c2 * Z[offz + S::SC] - cz * Z[cz ? offz - S::SC : offz]);
}

template <int LA, int LB, int LC, int LD, int G>
__global__ void __launch_bounds__(128) eri_grad_group_kernel(GradArgs args) {
    using S = GradShape<LA, LB, LC, LD, G>;
    constexpr int NB = S::NB, NC = S::NC, ND = S::ND, NCD = S::NCD, NR = S::NR, NI = S::NIP;
    constexpr int LAB = LA + LB + 1, LCD = LC + LD + 1;
    extern __shared__ double gsm[];
    const int gq = threadIdx.x / G, lane = threadIdx.x % G;
    double *__restrict__ sm = gsm + gq * S::SMEM;
    const unsigned mask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) / G * G));
    const WorkSub ws = pick_sub(args.work);
    const long long t = ((long long)blockIdx.x - ws.cta0) * S::GPB + gq;
    const int ib = bra_of(ws.offs, ws.cbra, min(t, ws.total - 1));
    if (t >= ws.total) return;
    const int ik = ws.k0 + (int)(t - ws.offs[ib]);
    const int A = args.bra.shA[ib], B = args.bra.shB[ib], C = args.ket.shA[ik], D = args.ket.shB[ik];
    const int atA = args.bs.sh_atom[A], atB = args.bs.sh_atom[B], atC = args.bs.sh_atom[C], atD = args.bs.sh_atom[D];
    if (atA == atB && atA == atC && atA == atD) return;  // one-centre quartets have no gradient
    if (grad_skip(args, ib, ik, A, B, C, D)) return;
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

    // this lane's rows (a,b) and units (a,b,c): Cartesian powers, row offsets and Gamma values
    int rax[S::FR > 0 ? S::FR : 1], ray[S::FR > 0 ? S::FR : 1], raz[S::FR > 0 ? S::FR : 1];
    int rbx[S::FR > 0 ? S::FR : 1], rby[S::FR > 0 ? S::FR : 1], rbz[S::FR > 0 ? S::FR : 1];
    double gamR[S::FR > 0 ? S::FR : 1][NCD];
#pragma unroll
    for (int k = 0; k < S::FR; ++k) {
        const int row = lane + G * k, a = row / NB, b = row - (row / NB) * NB;
        rax[k] = cart_x(LA, a); ray[k] = cart_y(LA, a); raz[k] = cart_z(LA, a);
        rbx[k] = cart_x(LB, b); rby[k] = cart_y(LB, b); rbz[k] = cart_z(LB, b);
        const double dab = Dm[(oa + a) * n + ob + b];
#pragma unroll
        for (int kc = 0; kc < NC; ++kc) {
            const double dac = Dm[(oa + a) * n + oc + kc], dbc = Dm[(ob + b) * n + oc + kc];
#pragma unroll
            for (int ld = 0; ld < ND; ++ld) {
                const double dcd = Dm[(oc + kc) * n + od + ld];
                const double dbd = Dm[(ob + b) * n + od + ld], dad = Dm[(oa + a) * n + od + ld];
                gamR[k][kc * ND + ld] = cj * dab * dcd + ck * (dac * dbd + dad * dbc);
            }
        }
    }
    int uax[S::NU > 0 ? S::NU : 1], uay[S::NU > 0 ? S::NU : 1], uaz[S::NU > 0 ? S::NU : 1];
    int ubx[S::NU > 0 ? S::NU : 1], uby[S::NU > 0 ? S::NU : 1], ubz[S::NU > 0 ? S::NU : 1];
    int ucx[S::NU > 0 ? S::NU : 1], ucy[S::NU > 0 ? S::NU : 1], ucz[S::NU > 0 ? S::NU : 1];
    double gamU[S::NU > 0 ? S::NU : 1][ND];
#pragma unroll
    for (int j = 0; j < S::NU; ++j) {
        const bool valid = lane + G * j < S::NUNIT;
        const int u = valid ? lane + G * j : 0;
        const int row = S::FR * G + u / NC, c = u % NC, a = row / NB, b = row % NB;
        uax[j] = cart_x(LA, a); uay[j] = cart_y(LA, a); uaz[j] = cart_z(LA, a);
        ubx[j] = cart_x(LB, b); uby[j] = cart_y(LB, b); ubz[j] = cart_z(LB, b);
        ucx[j] = cart_x(LC, c); ucy[j] = cart_y(LC, c); ucz[j] = cart_z(LC, c);
        const double dab = Dm[(oa + a) * n + ob + b];
        const double dac = Dm[(oa + a) * n + oc + c], dbc = Dm[(ob + b) * n + oc + c];
#pragma unroll
        for (int ld = 0; ld < ND; ++ld) {
            const double dcd = Dm[(oc + c) * n + od + ld];
            const double dbd = Dm[(ob + b) * n + od + ld], dad = Dm[(oa + a) * n + od + ld];
            gamU[j][ld] = valid ? cj * dab * dcd + ck * (dac * dbd + dad * dbc) : 0.0;
        }
    }
    double g[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) g[k] = 0.0;
    const PrimPairs &pp = args.pp;
    const int pb0 = args.bra.poff[ib], npb = args.bra.np[ib], pk0 = args.ket.poff[ik], npk = args.ket.np[ik];
    for (int xb = pb0; xb < pb0 + npb; ++xb) {
        const double ea = pp.a[xb], eb = pp.b[xb], p = ea + eb;
        const double Px = pp.Px[xb], Py = pp.Py[xb], Pz = pp.Pz[xb];
        const double Kb = pp.Kp[xb], argb = pp.arg[xb], hpb = pp.hp[xb];
        for (int xk = pk0; xk < pk0 + npk; ++xk) {
            if (argb + pp.arg[xk] > PDG_PRIMITIVE_CUT) continue;
            const double ec = pp.a[xk], q = ec + pp.b[xk], hpk = pp.hp[xk];
            const double Qx = pp.Px[xk], Qy = pp.Py[xk], Qz = pp.Pz[xk];
            const double rs = rsqrt(p + q), rppq = rs * rs;
            const double PQx = Px - Qx, PQy = Py - Qy, PQz = Pz - Qz;
            const double x = p * q * rppq * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pref = TWO_PI_POW_2P5 * rs * Kb * pp.Kp[xk];
            __syncwarp(mask);
            for (int task = lane; task < 3 * NR; task += G) {
                const int r = task / 3, dir = task - 3 * (task / 3);
                double ur, wr;
                rys_root_single<NR>(x, r, ur, wr);
                ur *= rppq;
                const double b00 = 0.5 * ur, b10 = hpb * (1.0 - q * ur), b01 = hpk * (1.0 - p * ur);
                const double fq = q * ur, fp = p * ur;
                const double PA = dir == 0 ? Px - rA[0] : dir == 1 ? Py - rA[1] : Pz - rA[2];
                const double QC = dir == 0 ? Qx - rC[0] : dir == 1 ? Qy - rC[1] : Qz - rC[2];
                const double PQ = dir == 0 ? PQx : dir == 1 ? PQy : PQz;
                const double AB = dir == 0 ? rA[0] - rB[0] : dir == 1 ? rA[1] - rB[1] : rA[2] - rB[2];
                const double CD = dir == 0 ? rC[0] - rD[0] : dir == 1 ? rC[1] - rD[1] : rC[2] - rD[2];
                double Gm[LAB + 1][LCD + 1];
                rys_vrr<LAB, LCD>(Gm, dir == 2 ? wr * pref : 1.0, PA - fq * PQ, QC + fp * PQ, b10, b01, b00);
                grad_hrr_store<LA, LB, LC, LD>(Gm, AB, CD, sm + task * NI);
            }
            __syncwarp(mask);
            const double a2 = 2.0 * ea, b2 = 2.0 * eb, c2 = 2.0 * ec;
#pragma unroll 1
            for (int r = 0; r < NR; ++r) {
                const double *__restrict__ Ix = sm + (3 * r) * NI;
                const double *__restrict__ Iy = Ix + NI;
                const double *__restrict__ Iz = Iy + NI;
#pragma unroll
                for (int k = 0; k < S::FR; ++k) {
                    const double *X = Ix + rax[k] * S::SA + rbx[k] * S::SB;
                    const double *Y = Iy + ray[k] * S::SA + rby[k] * S::SB;
                    const double *Z = Iz + raz[k] * S::SA + rbz[k] * S::SB;
#pragma unroll
                    for (int kc = 0; kc < NC; ++kc)
#pragma unroll
                        for (int ld = 0; ld < ND; ++ld) {
                            const int cxx = cart_x(LC, kc), cy = cart_y(LC, kc), cz = cart_z(LC, kc);
                            grad_component<LA, LB, LC, LD, G>(
                                X, Y, Z, cxx * S::SC + cart_x(LD, ld), cy * S::SC + cart_y(LD, ld), cz * S::SC + cart_z(LD, ld),
                                rax[k], ray[k], raz[k], rbx[k], rby[k], rbz[k], cxx, cy, cz, gamR[k][kc * ND + ld], a2, b2, c2, g);
                        }
                }
#pragma unroll
                for (int j = 0; j < S::NU; ++j) {
                    const double *X = Ix + uax[j] * S::SA + ubx[j] * S::SB + ucx[j] * S::SC;
                    const double *Y = Iy + uay[j] * S::SA + uby[j] * S::SB + ucy[j] * S::SC;
                    const double *Z = Iz + uaz[j] * S::SA + ubz[j] * S::SB + ucz[j] * S::SC;
#pragma unroll
                    for (int ld = 0; ld < ND; ++ld)
                        grad_component<LA, LB, LC, LD, G>(X, Y, Z, cart_x(LD, ld), cart_y(LD, ld), cart_z(LD, ld), uax[j],
                                                          uay[j], uaz[j], ubx[j], uby[j], ubz[j], ucx[j], ucy[j], ucz[j],
                                                          gamU[j][ld], a2, b2, c2, g);
                }
            }
        }
    }
    // reduce over the group's lanes, one lane adds to the atom gradients
#pragma unroll
    for (int k = 0; k < 9; ++k)
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) g[k] += __shfl_xor_sync(mask, g[k], o);
    if (lane == 0) {
        double *gr = args.grad;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            atomicAdd(&gr[3 * atA + k], g[k]);
            atomicAdd(&gr[3 * atB + k], g[3 + k]);
            atomicAdd(&gr[3 * atC + k], g[6 + k]);
            atomicAdd(&gr[3 * atD + k], -(g[k] + g[3 + k] + g[6 + k]));
        }
    }
}

__host__ __device__ constexpr int grad_group(int la, int lb, int lc, int ld) {
    return (la == 2 && lb == 2 && lc == 2) ? 32
         : (la == 2 && lb == 2 && lc == 1 && ld == 1) ? 16
         : (la == 2 && lb == 1 && lc == 2 && ld == 1) ? 16
         : (la == 2 && lb == 1 && lc == 1 && ld == 1) ? 8
         : (la == 2 && lb == 2 && lc == 1 && ld == 0) ? 8
         : (la == 2 && lb == 1 && lc == 2 && ld == 0) ? 8
         : 0;
}

constexpr int PLA[PDG_NPAIRCLASS] = {0, 1, 1, 2, 2, 2};
constexpr int PLB[PDG_NPAIRCLASS] = {0, 0, 1, 0, 1, 2};

// Lanes per quartet of the one-thread gradient form by ket bucket: the buckets with many primitive
// pairs split their primitive quartets.
constexpr int kGradLanes[PDG_NBUCKET] = {1, 1, 2, 4, 4};

template <int CB, int CK>
void launch_grad_t(const GradArgs &a0, const QuartetBlock &b, cudaStream_t st) {
    GradArgs a = a0;
    constexpr int LA = PLA[CB], LB = PLB[CB], LC = PLA[CK], LD = PLB[CK];
    constexpr int G = grad_group(LA, LB, LC, LD);
    if constexpr (G > 0) {
        using S = GradShape<LA, LB, LC, LD, G>;
        const size_t smem = (size_t)S::SMEM * S::GPB * sizeof(double);
        auto kern = eri_grad_group_kernel<LA, LB, LC, LD, G>;
        if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        const int lanes[PDG_NBUCKET] = {G, G, G, G, G};
        const long long blocks = pdg_fill_work(a.work, b, lanes);
        a.part = 0;  // the cooperative d-class form evaluates every quartet in FP64
        { kern<<<(unsigned)blocks, 128, smem, st>>>(a); pdg_count_launch(); }
    } else {
        const long long blocks = pdg_fill_work(a.work, b, kGradLanes);
        if (a.part == 0) {
            { eri_grad_kernel<LA, LB, LC, LD, double><<<(unsigned)blocks, 128, 0, st>>>(a); pdg_count_launch(); }
        } else {
            // mixed mode: the quartets above the mixed cut in FP64, the rest in FP32
            a.part = 1;
            { eri_grad_kernel<LA, LB, LC, LD, double><<<(unsigned)blocks, 128, 0, st>>>(a); pdg_count_launch(); }
            a.part = 2;
            { eri_grad_kernel<LA, LB, LC, LD, float><<<(unsigned)blocks, 128, 0, st>>>(a); pdg_count_launch(); }
        }
    }
}
typedef void (*grad_launcher)(const GradArgs &, const QuartetBlock &, cudaStream_t);
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
    const int ns = (int)ctx->shells.size();
    // quartets whose Schwarz x |Gamma| bound is below the SCF's density-screening bound (FP64) or
    // below mixed_drop (mixed mode) are skipped
    double *dmax = (double *)pdg_pool(ctx, "grad_dmax", (size_t)ns * ns * sizeof(double));
    if (!dmax) { pdg_set_error("pdg_eri_grad: device buffer allocation failed"); return PDG_ERR_ALLOC; }
    PDG_CHECK(pdg_shell_pair_dmax(ctx, d_D, dmax));
    const double gcut = ctx->precision_mode == 1 ? ctx->mixed_drop : ctx->inc_cut;
    ctx->grad_valid = true;
    ctx->grad_doJ = doJ ? 1 : 0;
    ctx->grad_cx = cx;
    ctx->grad_gcut = gcut;
    ProfScope prof(ctx, "eri_grad");
    for (const auto &b : ctx->blocks) {
        GradArgs a;
        a.bra = ctx->pairs[b.cb];
        a.ket = ctx->pairs[b.ck];
        a.same = (b.cb == b.ck);
        a.pp = ctx->pp;
        a.bs = ctx->dbasis;
        a.D = d_D;
        a.cx = cx;
        a.doJ = doJ ? 1 : 0;
        a.grad = d_grad;
        a.n = ctx->nbf;
        a.dmax = dmax;
        a.nshell = ns;
        a.gcut = gcut;
        a.part = ctx->precision_mode == 1 ? 1 : 0;
        a.mixed_cut = ctx->mixed_cut;
        grad_table[b.cb][b.ck](a, b, ctx->stream);
        PDG_CUDA(cudaGetLastError());
    }
    return PDG_OK;
}
