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
#include <string>
#include <atomic>
#include <type_traits>

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

// One primitive quartet (bra primitive pair B, ket primitive pair K) added to the raw Cartesian
// block V[(a*NB+b)*NC*ND + c*ND + d].  T is the arithmetic type of the recursions and the
// accumulation (float for the quartets of the mixed-precision mode); the Boys argument, the Rys
// rule and the prefactors stay in double.
template <int LA, int LB, int LC, int LD, typename T = double>
__device__ __forceinline__ void eri_prim(const PairRec &B, const PairRec &K, const QuartetGeom &g,
                                         T (&V)[ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD)]) {
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    constexpr int LAB = LA + LB, LCD = LC + LD, NR = (LAB + LCD) / 2 + 1;
    const double p = B.p, Px = B.Px, Py = B.Py, Pz = B.Pz;
    const double q = K.p, Qx = K.Px, Qy = K.Py, Qz = K.Pz;
    const double rs = rsqrt(p + q), rppq = rs * rs;
    const double PQx = Px - Qx, PQy = Py - Qy, PQz = Pz - Qz;
    const double x = p * q * rppq * (PQx * PQx + PQy * PQy + PQz * PQz);
    const double pref = TWO_PI_POW_2P5 * rs * B.Kp * K.Kp;
    double u[NR], w[NR];
    rys_roots<NR>(x, u, w);
    const double PAx = Px - g.A[0], PAy = Py - g.A[1], PAz = Pz - g.A[2];
    const double QCx = Qx - g.C[0], QCy = Qy - g.C[1], QCz = Qz - g.C[2];
    const T ABx = T(g.A[0] - g.B[0]), ABy = T(g.A[1] - g.B[1]), ABz = T(g.A[2] - g.B[2]);
    const T CDx = T(g.C[0] - g.D[0]), CDy = T(g.C[1] - g.D[1]), CDz = T(g.C[2] - g.D[2]);
    const double r2p = B.hp, r2q = K.hp;
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const double ur = u[r] * rppq;
        const T b00 = T(0.5 * ur);
        const T b10 = T(r2p * (1.0 - q * ur));
        const T b01 = T(r2q * (1.0 - p * ur));
        const double fq = q * ur, fp = p * ur;
        T Gx[LAB + 1][LCD + 1], Gy[LAB + 1][LCD + 1], Gz[LAB + 1][LCD + 1];
        rys_vrr<LAB, LCD, T>(Gx, T(1), T(PAx - fq * PQx), T(QCx + fp * PQx), b10, b01, b00);
        rys_vrr<LAB, LCD, T>(Gy, T(1), T(PAy - fq * PQy), T(QCy + fp * PQy), b10, b01, b00);
        rys_vrr<LAB, LCD, T>(Gz, T(w[r] * pref), T(PAz - fq * PQz), T(QCz + fp * PQz), b10, b01, b00);
        T Ix[LA + 1][LB + 1][LC + 1][LD + 1], Iy[LA + 1][LB + 1][LC + 1][LD + 1], Iz[LA + 1][LB + 1][LC + 1][LD + 1];
        rys_hrr<LA, LB, LC, LD, T>(Gx, ABx, CDx, Ix);
        rys_hrr<LA, LB, LC, LD, T>(Gy, ABy, CDy, Iy);
        rys_hrr<LA, LB, LC, LD, T>(Gz, ABz, CDz, Iz);
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int jb = 0; jb < NB; ++jb)
#pragma unroll
                for (int kc = 0; kc < NC; ++kc)
#pragma unroll
                    for (int ld = 0; ld < ND; ++ld) {
                        const T vx = Ix[cart_x(LA, ia)][cart_x(LB, jb)][cart_x(LC, kc)][cart_x(LD, ld)];
                        const T vy = Iy[cart_y(LA, ia)][cart_y(LB, jb)][cart_y(LC, kc)][cart_y(LD, ld)];
                        const T vz = Iz[cart_z(LA, ia)][cart_z(LB, jb)][cart_z(LC, kc)][cart_z(LD, ld)];
                        V[((ia * NB + jb) * NC + kc) * ND + ld] += vx * vy * vz;
                    }
    }
}

// Quartet geometry for the FP32 quartets: the centre differences, taken in double and rounded once.
struct QuartetGeom32 {
    float ABx, ABy, ABz, CDx, CDy, CDz, ACx, ACy, ACz;
};
__device__ __forceinline__ QuartetGeom32 geom32(const QuartetGeom &g) {
    return QuartetGeom32{(float)(g.A[0] - g.B[0]), (float)(g.A[1] - g.B[1]), (float)(g.A[2] - g.B[2]),
                         (float)(g.C[0] - g.D[0]), (float)(g.C[1] - g.D[1]), (float)(g.C[2] - g.D[2]),
                         (float)(g.A[0] - g.C[0]), (float)(g.A[1] - g.C[1]), (float)(g.A[2] - g.C[2])};
}

// eri_prim entirely in single precision, for the quartets of the mixed mode whose bound is below the
// mixed cut: Boys argument, Rys rule (rys_roots_f), prefactor, recursions and accumulation.  With
// P - A and Q - C from the records, P - Q = (P - A) - (Q - C) + (A - C).
template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ void eri_prim32(const PairRec32 &B, const PairRec32 &K, const QuartetGeom32 &g,
                                           float (&V)[ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD)]) {
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    constexpr int LAB = LA + LB, LCD = LC + LD, NR = (LAB + LCD) / 2 + 1;
    const float p = B.p, q = K.p;
    const float rs = rsqrtf(p + q), rppq = rs * rs;
    const float PQx = B.PAx - K.PAx + g.ACx, PQy = B.PAy - K.PAy + g.ACy, PQz = B.PAz - K.PAz + g.ACz;
    const float x = p * q * rppq * (PQx * PQx + PQy * PQy + PQz * PQz);
    const float pref = (float)TWO_PI_POW_2P5 * rs * B.Kp * K.Kp;
    float u[NR], w[NR];
    rys_roots_f<NR>(x, u, w);
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const float ur = u[r] * rppq;
        const float b00 = 0.5f * ur, b10 = B.hp * (1.0f - q * ur), b01 = K.hp * (1.0f - p * ur);
        const float fq = q * ur, fp = p * ur;
        float Gx[LAB + 1][LCD + 1], Gy[LAB + 1][LCD + 1], Gz[LAB + 1][LCD + 1];
        rys_vrr<LAB, LCD, float>(Gx, 1.0f, B.PAx - fq * PQx, K.PAx + fp * PQx, b10, b01, b00);
        rys_vrr<LAB, LCD, float>(Gy, 1.0f, B.PAy - fq * PQy, K.PAy + fp * PQy, b10, b01, b00);
        rys_vrr<LAB, LCD, float>(Gz, w[r] * pref, B.PAz - fq * PQz, K.PAz + fp * PQz, b10, b01, b00);
        float Ix[LA + 1][LB + 1][LC + 1][LD + 1], Iy[LA + 1][LB + 1][LC + 1][LD + 1], Iz[LA + 1][LB + 1][LC + 1][LD + 1];
        rys_hrr<LA, LB, LC, LD, float>(Gx, g.ABx, g.CDx, Ix);
        rys_hrr<LA, LB, LC, LD, float>(Gy, g.ABy, g.CDy, Iy);
        rys_hrr<LA, LB, LC, LD, float>(Gz, g.ABz, g.CDz, Iz);
#pragma unroll
        for (int ia = 0; ia < NA; ++ia)
#pragma unroll
            for (int jb = 0; jb < NB; ++jb)
#pragma unroll
                for (int kc = 0; kc < NC; ++kc)
#pragma unroll
                    for (int ld = 0; ld < ND; ++ld) {
                        const float vx = Ix[cart_x(LA, ia)][cart_x(LB, jb)][cart_x(LC, kc)][cart_x(LD, ld)];
                        const float vy = Iy[cart_y(LA, ia)][cart_y(LB, jb)][cart_y(LC, kc)][cart_y(LD, ld)];
                        const float vz = Iz[cart_z(LA, ia)][cart_z(LB, jb)][cart_z(LC, kc)][cart_z(LD, ld)];
                        V[((ia * NB + jb) * NC + kc) * ND + ld] += vx * vy * vz;
                    }
    }
}

// Contracted raw Cartesian block of one shell quartet.  CUT applies the reference's
// primitive-quartet cut; the Schwarz diagonal is computed without it, because a primitive pair
// cut in (ab|ab) can still contribute to (ab|cd) against a compact ket pair.
template <int LA, int LB, int LC, int LD, bool CUT = true, typename T = double>
__device__ __forceinline__ void eri_block(const PrimPairs &pp, int pb0, int npb, int pk0, int npk,
                                          const QuartetGeom &g,
                                          T (&V)[ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD)]) {
#pragma unroll
    for (int i = 0; i < ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD); ++i) V[i] = T(0);
    for (int ib = pb0; ib < pb0 + npb; ++ib) {
        if constexpr (std::is_same<T, float>::value) {
            const PairRec32 Bp = load_rec32(pp.rec32, ib);
            const QuartetGeom32 g32 = geom32(g);
            for (int ik = pk0; ik < pk0 + npk; ++ik) {
                const PairRec32 Kp = load_rec32(pp.rec32, ik);
                if (CUT && Bp.arg + Kp.arg > (float)PDG_PRIMITIVE_CUT) continue;
                eri_prim32<LA, LB, LC, LD>(Bp, Kp, g32, V);
            }
        } else {
            const double argb = load_arg(pp.rec, ib);
            const PairRec Bp = load_rec(pp.rec, ib);
            for (int ik = pk0; ik < pk0 + npk; ++ik) {
                if (CUT && argb + load_arg(pp.rec, ik) > PDG_PRIMITIVE_CUT) continue;
                eri_prim<LA, LB, LC, LD, T>(Bp, load_rec(pp.rec, ik), g, V);
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
    WorkList work;       // the quartets: per ket bucket, prefix sums over bra pairs and the bra map
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
    int part;            // 0: every quartet; 1: only bound >= mixed_cut (FP64); 2: only bound < mixed_cut (FP32)
    double mixed_cut;
    int variant;         // host side: lanes-per-bucket table of the launch (-1: the tuned table)
    unsigned long long *count32;  // optional: running count of quartets evaluated in FP32
};

// Adds the quartets of the calling lanes that lead a quartet (leader) to args.count32, one atomic
// per warp.
__device__ __forceinline__ void count_fp32(const JKArgs &args, bool leader) {
    if (!args.count32 || args.part != 2) return;
    const unsigned am = __activemask();
    const unsigned bm = __ballot_sync(am, leader);
    if (leader && (int)(threadIdx.x & 31) == __ffs(bm) - 1) atomicAdd(args.count32, (unsigned long long)__popc(bm));
}

// Density screening and the precision partition of the mixed mode.  The Coulomb and exchange
// parts are screened separately: a quartet changes J by at most Q_AB Q_CD max(|D_AB|, |D_CD|) and
// K by at most Q_AB Q_CD max(|D_AC|, |D_AD|, |D_BC|, |D_BD|); each part is digested only when its
// bound reaches dcut, and the quartet is skipped when neither does.  The mixed mode partitions on
// the larger of the two bounds.
struct JKScreen {
    bool any, j, k;
};
template <bool DOJ, bool DOK>
__device__ __forceinline__ JKScreen jk_screen(const JKArgs &args, int ib, int ik, int A, int B, int C, int D) {
    if (!args.dmax) return {true, DOJ, DOK};
    const int ns = args.nshell;
    const double q = args.bra.Q[ib] * args.ket.Q[ik];
    const double bj = DOJ ? q * fmax(args.dmax[A * ns + B], args.dmax[C * ns + D]) : 0.0;
    const double bk = DOK ? q * fmax(fmax(args.dmax[B * ns + D], args.dmax[B * ns + C]),
                                     fmax(args.dmax[A * ns + D], args.dmax[A * ns + C])) : 0.0;
    JKScreen r{false, DOJ && bj >= args.dcut, DOK && bk >= args.dcut};
    r.any = r.j || r.k;
    const double bound = fmax(bj, bk);
    if (args.part == 1) r.any = r.any && bound >= args.mixed_cut;
    if (args.part == 2) r.any = r.any && bound < args.mixed_cut;
    return r;
}

// One shell quartet per P lanes (SPLIT: P = the bucket's lane count, 1 to 8; else 1): the lanes split
// the primitive quartets and add their blocks with shuffles; the first lanes digest, one the J part
// and up to two the K parts (rows of a, rows of b), as independent streams of loads and atomics that
// the warp scheduler interleaves.  Splitting keeps more primitive loads in flight for the contracted
// s/p classes (up to 6 x 6 primitive pairs per shell pair), whose one-lane loops are bound by load
// latency; the ket buckets give the quartets of a warp the same primitive count.
template <int LA, int LB, int LC, int LD, bool DOJ, bool DOK, typename T = double, bool SPLIT = false>
__global__ void __launch_bounds__(128) eri_jk_kernel(JKArgs args) {
    const WorkSub ws = pick_sub(args.work);
    const int P = SPLIT ? ws.lanes : 1;
    const long long t = ((long long)blockIdx.x - ws.cta0) * blockDim.x / P + (long long)(threadIdx.x / P);
    const int lane = SPLIT ? (int)(threadIdx.x & (P - 1)) : 0;
    const int ib = bra_of(ws.offs, ws.cbra, min(t, ws.total - 1));
    if (t >= ws.total) return;
    const int ik = ws.k0 + (int)(t - ws.offs[ib]);
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    const int A = args.bra.shA[ib], B = args.bra.shB[ib], C = args.ket.shA[ik], D = args.ket.shB[ik];
    // density screening: the quartet changes J (K) by at most Q_AB Q_CD times the largest
    // density element it is contracted with
    const JKScreen scr = jk_screen<DOJ, DOK>(args, ib, ik, A, B, C, D);
    if (!scr.any) return;
    count_fp32(args, lane == 0);
    QuartetGeom g;
    load_xyz(args.bs, A, g.A);
    load_xyz(args.bs, B, g.B);
    load_xyz(args.bs, C, g.C);
    load_xyz(args.bs, D, g.D);
    T V[NA * NB * NC * ND];
    if constexpr (!SPLIT) {
        eri_block<LA, LB, LC, LD, true, T>(args.pp, args.bra.poff[ib], args.bra.np[ib], args.ket.poff[ik], args.ket.np[ik], g, V);
    } else {
#pragma unroll
        for (int i = 0; i < NA * NB * NC * ND; ++i) V[i] = T(0);
        const int pb0 = args.bra.poff[ib], pk0 = args.ket.poff[ik], npk = args.ket.np[ik];
        const int nprim = args.bra.np[ib] * npk;
        // primitive quartet idx = jb npk + jk, stepped by P without a division per step
        int jb = lane / npk, jk = lane - jb * npk;
        if constexpr (std::is_same<T, float>::value) {
            const QuartetGeom32 g32 = geom32(g);
            for (int idx = lane; idx < nprim; idx += P, jk += P) {
                while (jk >= npk) { jk -= npk; ++jb; }
                const PairRec32 Bp = load_rec32(args.pp.rec32, pb0 + jb), Kp = load_rec32(args.pp.rec32, pk0 + jk);
                if (Bp.arg + Kp.arg > (float)PDG_PRIMITIVE_CUT) continue;
                eri_prim32<LA, LB, LC, LD>(Bp, Kp, g32, V);
            }
        } else {
            for (int idx = lane; idx < nprim; idx += P, jk += P) {
                while (jk >= npk) { jk -= npk; ++jb; }
                const int xb = pb0 + jb, xk = pk0 + jk;
                if (load_arg(args.pp.rec, xb) + load_arg(args.pp.rec, xk) > PDG_PRIMITIVE_CUT) continue;
                eri_prim<LA, LB, LC, LD, T>(load_rec(args.pp.rec, xb), load_rec(args.pp.rec, xk), g, V);
            }
        }
        const unsigned mask = lane_group_mask(P);
        for (int o = P >> 1; o > 0; o >>= 1) {
#pragma unroll
            for (int i = 0; i < NA * NB * NC * ND; ++i) V[i] += __shfl_xor_sync(mask, V[i], o);
        }
        // every lane of the group now holds the contracted block; up to three of them share the
        // digest (J; K rows of a; K rows of b)
        if (lane >= (P < 3 ? P : 3)) return;
    }
    const int roles = SPLIT ? (P < 3 ? P : 3) : 1;
    const bool do_j = lane == 0;
    const bool do_ka = roles == 3 ? lane == 1 : lane == 0;
    const bool do_kb = lane == roles - 1;
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
                        if (fabs((double)V[f] * nn) <= uf) V[f] = T(0);
                    }
    }
    const int n = args.n;
    const int oa = args.bs.sh_bf[A], ob = args.bs.sh_bf[B], oc = args.bs.sh_bf[C], od = args.bs.sh_bf[D];
    const double *__restrict__ Dm = args.D;
    if (DOJ && scr.j && do_j) {
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
    if (DOK && scr.k && do_ka) {
        // Kt[a][c] += s V Dbd ; Kt[a][d] += s V Dbc
#pragma unroll
        for (int ia = 0; ia < NA; ++ia) {
            double kac[NC], kad[ND];
#pragma unroll
            for (int i = 0; i < NC; ++i) kac[i] = 0.0;
#pragma unroll
            for (int i = 0; i < ND; ++i) kad[i] = 0.0;
#pragma unroll
            for (int jb = 0; jb < NB; ++jb)
#pragma unroll
                for (int kc = 0; kc < NC; ++kc) {
                    const double dbc = Dm[(ob + jb) * n + oc + kc];
#pragma unroll
                    for (int ld = 0; ld < ND; ++ld) {
                        const double v = V[((ia * NB + jb) * NC + kc) * ND + ld];
                        kac[kc] += v * Dm[(ob + jb) * n + od + ld];
                        kad[ld] += v * dbc;
                    }
                }
#pragma unroll
            for (int kc = 0; kc < NC; ++kc) atomicAdd(&args.K[(oa + ia) * n + oc + kc], s * kac[kc]);
#pragma unroll
            for (int ld = 0; ld < ND; ++ld) atomicAdd(&args.K[(oa + ia) * n + od + ld], s * kad[ld]);
        }
    }
    if (DOK && scr.k && do_kb) {
        // Kt[b][c] += s V Dad ; Kt[b][d] += s V Dac
#pragma unroll
        for (int jb = 0; jb < NB; ++jb) {
            double kbc[NC], kbd[ND];
#pragma unroll
            for (int i = 0; i < NC; ++i) kbc[i] = 0.0;
#pragma unroll
            for (int i = 0; i < ND; ++i) kbd[i] = 0.0;
#pragma unroll
            for (int ia = 0; ia < NA; ++ia)
#pragma unroll
                for (int kc = 0; kc < NC; ++kc) {
                    const double dac = Dm[(oa + ia) * n + oc + kc];
#pragma unroll
                    for (int ld = 0; ld < ND; ++ld) {
                        const double v = V[((ia * NB + jb) * NC + kc) * ND + ld];
                        kbc[kc] += v * Dm[(oa + ia) * n + od + ld];
                        kbd[ld] += v * dac;
                    }
                }
#pragma unroll
            for (int kc = 0; kc < NC; ++kc) atomicAdd(&args.K[(ob + jb) * n + oc + kc], s * kbc[kc]);
#pragma unroll
            for (int ld = 0; ld < ND; ++ld) atomicAdd(&args.K[(ob + jb) * n + od + ld], s * kbd[ld]);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Cooperative form for the d-shell classes whose component block (up to 6^4 = 1296 values) does
// not fit one thread's registers: G lanes of a warp share one shell quartet.
//  - per primitive quartet, lanes take the 3 x n_R (root, direction) tasks: one Rys node each
//    (rys_root_single), the 2D recursion and the closed-form transfers
//    I(a,b,c,d) = sum_k sum_m C(b,k) (A-B)^(b-k) C(d,m) (C-D)^(d-m) G(a+k, c+m), written to
//    shared memory;
//  - each lane owns whole bra rows (a,b) of the block (all c,d) and accumulates them over roots
//    and primitives in registers; rows left over after the full rounds are split by c.  Lanes
//    of a row share the (a_x,b_x) slice of the 2D integrals, so a warp load touches at most 9
//    distinct words and is served in one wavefront;
//  - the contracted block is written to shared memory (after the storage underflow) and the
//    J/K digest is spread over the lanes with the needed density blocks staged beside it.
// ---------------------------------------------------------------------------------------------
__host__ __device__ constexpr int binom_small(int n, int k) { return (k == 0 || k == n) ? 1 : (n == 2 ? 2 : n); }

template <int LA, int LB, int LC, int LD, typename T = double>
__device__ __forceinline__ void hrr_store(const T (&Gm)[LA + LB + 1][LC + LD + 1], T AB, T CD, T *__restrict__ out) {
    constexpr int LCD = LC + LD;
    T abp[LB + 1], cdp[LD + 1];
    abp[0] = T(1);
#pragma unroll
    for (int k = 1; k <= LB; ++k) abp[k] = abp[k - 1] * AB;
    cdp[0] = T(1);
#pragma unroll
    for (int k = 1; k <= LD; ++k) cdp[k] = cdp[k - 1] * CD;
#pragma unroll
    for (int a = 0; a <= LA; ++a)
#pragma unroll
        for (int b = 0; b <= LB; ++b) {
            T row[LCD + 1];
#pragma unroll
            for (int f = 0; f <= LCD; ++f) {
                T s = Gm[a + b][f];
#pragma unroll
                for (int k = 0; k < b; ++k) s += T(binom_small(b, k)) * abp[b - k] * Gm[a + k][f];
                row[f] = s;
            }
#pragma unroll
            for (int c = 0; c <= LC; ++c)
#pragma unroll
                for (int d = 0; d <= LD; ++d) {
                    T s = row[c + d];
#pragma unroll
                    for (int m = 0; m < d; ++m) s += T(binom_small(d, m)) * cdp[d - m] * row[c + m];
                    out[((a * (LB + 1) + b) * (LC + 1) + c) * (LD + 1) + d] = s;
                }
        }
}

template <int LA, int LB, int LC, int LD, int G>
struct GroupShape {
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    static constexpr int NCD = NC * ND;
    static constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
    static constexpr int NI = (LA + 1) * (LB + 1) * (LC + 1) * (LD + 1);
    static constexpr int NCOMP = NA * NB * NC * ND;
    static constexpr int R = NA * NB;            // bra rows
    static constexpr int FR = R / G;             // full rounds of rows per lane
    static constexpr int LR = R - FR * G;        // rows left over, split by c into units
    static constexpr int NUNIT = LR * NC;
    static constexpr int NU = (NUNIT + G - 1) / G;
    static constexpr int NIP = NI | 1;           // odd strides keep the lanes' rows in distinct banks
    static constexpr int NCDP = NCD | 1;
    static constexpr int NDBLK = NA * NB + NC * ND + NA * NC + NA * ND + NB * NC + NB * ND;
    static constexpr int WORK = (3 * NR * NIP > R * NCDP) ? 3 * NR * NIP : R * NCDP;
    static constexpr int SMEM = WORK + NDBLK;    // doubles per group
    static constexpr int GPB = 128 / G;          // groups per 128-thread block
};

template <int LA, int LB, int LC, int LD, int G, bool DOJ, bool DOK, typename T = double>
__global__ void __launch_bounds__(128) eri_jk_group_kernel(JKArgs args) {
    using S = GroupShape<LA, LB, LC, LD, G>;
    constexpr int NA = S::NA, NB = S::NB, NC = S::NC, ND = S::ND, NCD = S::NCD, NR = S::NR, NI = S::NIP;
    constexpr int NCDP = S::NCDP;  // row stride of the contracted block in shared memory
    constexpr int LAB = LA + LB, LCD = LC + LD;
    extern __shared__ double gsm[];
    const int gq = threadIdx.x / G, lane = threadIdx.x % G;
    double *__restrict__ sm = gsm + gq * S::SMEM;
    double *__restrict__ sD = sm + S::WORK;
    T *__restrict__ sI = reinterpret_cast<T *>(sm);  // 2D integrals during the primitive loop
    const unsigned mask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) / G * G));
    const WorkSub ws = pick_sub(args.work);
    const long long t = ((long long)blockIdx.x - ws.cta0) * S::GPB + gq;
    const int ib = bra_of(ws.offs, ws.cbra, min(t, ws.total - 1));
    if (t >= ws.total) return;
    const int ik = ws.k0 + (int)(t - ws.offs[ib]);
    const int A = args.bra.shA[ib], B = args.bra.shB[ib], C = args.ket.shA[ik], D = args.ket.shB[ik];
    const JKScreen scr = jk_screen<DOJ, DOK>(args, ib, ik, A, B, C, D);
    if (!scr.any) return;
    count_fp32(args, lane == 0);
    QuartetGeom g;
    load_xyz(args.bs, A, g.A);
    load_xyz(args.bs, B, g.B);
    load_xyz(args.bs, C, g.C);
    load_xyz(args.bs, D, g.D);

    // this lane's rows and units: offsets of their (a,b[,c]) slices in the 2D-integral arrays
    int rx[S::FR > 0 ? S::FR : 1], ry[S::FR > 0 ? S::FR : 1], rz[S::FR > 0 ? S::FR : 1];
#pragma unroll
    for (int k = 0; k < S::FR; ++k) {
        const int row = lane + G * k, a = row / NB, b = row - (row / NB) * NB;
        rx[k] = (cart_x(LA, a) * (LB + 1) + cart_x(LB, b)) * (LC + 1) * (LD + 1);
        ry[k] = (cart_y(LA, a) * (LB + 1) + cart_y(LB, b)) * (LC + 1) * (LD + 1);
        rz[k] = (cart_z(LA, a) * (LB + 1) + cart_z(LB, b)) * (LC + 1) * (LD + 1);
    }
    int ux[S::NU > 0 ? S::NU : 1], uy[S::NU > 0 ? S::NU : 1], uz[S::NU > 0 ? S::NU : 1];
#pragma unroll
    for (int j = 0; j < S::NU; ++j) {
        const int u = min(lane + G * j, S::NUNIT - 1);
        const int row = S::FR * G + u / NC, c = u % NC, a = row / NB, b = row % NB;
        ux[j] = ((cart_x(LA, a) * (LB + 1) + cart_x(LB, b)) * (LC + 1) + cart_x(LC, c)) * (LD + 1);
        uy[j] = ((cart_y(LA, a) * (LB + 1) + cart_y(LB, b)) * (LC + 1) + cart_y(LC, c)) * (LD + 1);
        uz[j] = ((cart_z(LA, a) * (LB + 1) + cart_z(LB, b)) * (LC + 1) + cart_z(LC, c)) * (LD + 1);
    }
    T accR[S::FR > 0 ? S::FR : 1][NCD], accU[S::NU > 0 ? S::NU : 1][ND];
#pragma unroll
    for (int k = 0; k < S::FR; ++k)
#pragma unroll
        for (int i = 0; i < NCD; ++i) accR[k][i] = T(0);
#pragma unroll
    for (int j = 0; j < S::NU; ++j)
#pragma unroll
        for (int i = 0; i < ND; ++i) accU[j][i] = T(0);

    const PrimPairs &pp = args.pp;
    const int pb0 = args.bra.poff[ib], npb = args.bra.np[ib], pk0 = args.ket.poff[ik], npk = args.ket.np[ik];
    for (int xb = pb0; xb < pb0 + npb; ++xb) {
        const double p = pp.a[xb] + pp.b[xb];
        const double Px = pp.Px[xb], Py = pp.Py[xb], Pz = pp.Pz[xb];
        const double Kb = pp.Kp[xb], argb = pp.arg[xb], hpb = pp.hp[xb];
        for (int xk = pk0; xk < pk0 + npk; ++xk) {
            if (argb + pp.arg[xk] > PDG_PRIMITIVE_CUT) continue;
            const double q = pp.a[xk] + pp.b[xk], hpk = pp.hp[xk];
            const double Qx = pp.Px[xk], Qy = pp.Py[xk], Qz = pp.Pz[xk];
            const double rs = rsqrt(p + q), rppq = rs * rs;
            const double PQx = Px - Qx, PQy = Py - Qy, PQz = Pz - Qz;
            const double x = p * q * rppq * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pref = TWO_PI_POW_2P5 * rs * Kb * pp.Kp[xk];
            __syncwarp(mask);  // the previous primitive's assembly has read the shared arrays
            for (int task = lane; task < 3 * NR; task += G) {
                const int r = task / 3, dir = task - 3 * (task / 3);
                double ur, wr;
                rys_root_single<NR>(x, r, ur, wr);
                ur *= rppq;
                const T b00 = T(0.5 * ur), b10 = T(hpb * (1.0 - q * ur)), b01 = T(hpk * (1.0 - p * ur));
                const double fq = q * ur, fp = p * ur;
                const double PA = dir == 0 ? Px - g.A[0] : dir == 1 ? Py - g.A[1] : Pz - g.A[2];
                const double QC = dir == 0 ? Qx - g.C[0] : dir == 1 ? Qy - g.C[1] : Qz - g.C[2];
                const double PQ = dir == 0 ? PQx : dir == 1 ? PQy : PQz;
                const double AB = dir == 0 ? g.A[0] - g.B[0] : dir == 1 ? g.A[1] - g.B[1] : g.A[2] - g.B[2];
                const double CD = dir == 0 ? g.C[0] - g.D[0] : dir == 1 ? g.C[1] - g.D[1] : g.C[2] - g.D[2];
                T Gm[LAB + 1][LCD + 1];
                rys_vrr<LAB, LCD, T>(Gm, T(dir == 2 ? wr * pref : 1.0), T(PA - fq * PQ), T(QC + fp * PQ), b10, b01, b00);
                hrr_store<LA, LB, LC, LD, T>(Gm, T(AB), T(CD), sI + task * NI);
            }
            __syncwarp(mask);
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const T *__restrict__ Ix = sI + (3 * r) * NI;
                const T *__restrict__ Iy = Ix + NI;
                const T *__restrict__ Iz = Iy + NI;
#pragma unroll
                for (int k = 0; k < S::FR; ++k) {
                    T X[(LC + 1) * (LD + 1)], Y[(LC + 1) * (LD + 1)], Z[(LC + 1) * (LD + 1)];
#pragma unroll
                    for (int i = 0; i < (LC + 1) * (LD + 1); ++i) { X[i] = Ix[rx[k] + i]; Y[i] = Iy[ry[k] + i]; Z[i] = Iz[rz[k] + i]; }
#pragma unroll
                    for (int kc = 0; kc < NC; ++kc)
#pragma unroll
                        for (int ld = 0; ld < ND; ++ld)
                            accR[k][kc * ND + ld] += X[cart_x(LC, kc) * (LD + 1) + cart_x(LD, ld)] *
                                                     Y[cart_y(LC, kc) * (LD + 1) + cart_y(LD, ld)] *
                                                     Z[cart_z(LC, kc) * (LD + 1) + cart_z(LD, ld)];
                }
#pragma unroll
                for (int j = 0; j < S::NU; ++j) {
                    T X[LD + 1], Y[LD + 1], Z[LD + 1];
#pragma unroll
                    for (int i = 0; i <= LD; ++i) { X[i] = Ix[ux[j] + i]; Y[i] = Iy[uy[j] + i]; Z[i] = Iz[uz[j] + i]; }
#pragma unroll
                    for (int ld = 0; ld < ND; ++ld)
                        accU[j][ld] += X[cart_x(LD, ld)] * Y[cart_y(LD, ld)] * Z[cart_z(LD, ld)];
                }
            }
        }
    }
    __syncwarp(mask);
    // contracted block to shared memory, with the storage underflow
    const double uf = args.underflow;
#pragma unroll
    for (int k = 0; k < S::FR; ++k) {
        const int row = lane + G * k, a = row / NB, b = row - (row / NB) * NB;
        const double nab = comp_norm(LA, a) * comp_norm(LB, b);
#pragma unroll
        for (int kc = 0; kc < NC; ++kc)
#pragma unroll
            for (int ld = 0; ld < ND; ++ld) {
                double v = (double)accR[k][kc * ND + ld];
                if (uf > 0.0 && fabs(v * nab * comp_norm(LC, kc) * comp_norm(LD, ld)) <= uf) v = 0.0;
                sm[row * NCDP + kc * ND + ld] = v;
            }
    }
#pragma unroll
    for (int j = 0; j < S::NU; ++j) {
        const int u = lane + G * j;
        if (u < S::NUNIT) {
            const int row = S::FR * G + u / NC, c = u % NC, a = row / NB, b = row % NB;
            const double nabc = comp_norm(LA, a) * comp_norm(LB, b) * comp_norm(LC, c);
#pragma unroll
            for (int ld = 0; ld < ND; ++ld) {
                double v = (double)accU[j][ld];
                if (uf > 0.0 && fabs(v * nabc * comp_norm(LD, ld)) <= uf) v = 0.0;
                sm[row * NCDP + c * ND + ld] = v;
            }
        }
    }
    // density blocks beside it: D_ab, D_cd, D_ac, D_ad, D_bc, D_bd
    const int n = args.n;
    const int oa = args.bs.sh_bf[A], ob = args.bs.sh_bf[B], oc = args.bs.sh_bf[C], od = args.bs.sh_bf[D];
    const double *__restrict__ Dm = args.D;
    double *dAB = sD, *dCD = dAB + NA * NB, *dAC = dCD + NC * ND, *dAD = dAC + NA * NC, *dBC = dAD + NA * ND,
           *dBD = dBC + NB * NC;
    for (int e = lane; e < NA * NB; e += G) dAB[e] = Dm[(oa + e / NB) * n + ob + e % NB];
    for (int e = lane; e < NC * ND; e += G) dCD[e] = Dm[(oc + e / ND) * n + od + e % ND];
    if (DOK) {
        for (int e = lane; e < NA * NC; e += G) dAC[e] = Dm[(oa + e / NC) * n + oc + e % NC];
        for (int e = lane; e < NA * ND; e += G) dAD[e] = Dm[(oa + e / ND) * n + od + e % ND];
        for (int e = lane; e < NB * NC; e += G) dBC[e] = Dm[(ob + e / NC) * n + oc + e % NC];
        for (int e = lane; e < NB * ND; e += G) dBD[e] = Dm[(ob + e / ND) * n + od + e % ND];
    }
    __syncwarp(mask);
    double s = 1.0;
    if (A == B) s *= 0.5;
    if (C == D) s *= 0.5;
    if (args.same && ib == ik) s *= 0.5;
    if (DOJ && scr.j) {
        const double s2 = 2.0 * s;
        for (int e = lane; e < NA * NB + NCD; e += G) {
            double acc = 0.0;
            if (e < NA * NB) {
#pragma unroll
                for (int cd = 0; cd < NCD; ++cd) acc += sm[e * NCDP + cd] * dCD[cd];
                atomicAdd(&args.J[(oa + e / NB) * n + ob + e % NB], s2 * acc);
            } else {
                const int cd = e - NA * NB;
#pragma unroll
                for (int ab = 0; ab < NA * NB; ++ab) acc += sm[ab * NCDP + cd] * dAB[ab];
                atomicAdd(&args.J[(oc + cd / ND) * n + od + cd % ND], s2 * acc);
            }
        }
    }
    if (DOK && scr.k) {
        constexpr int E1 = NA * NC, E2 = E1 + NA * ND, E3 = E2 + NB * NC, E4 = E3 + NB * ND;
        for (int e = lane; e < E4; e += G) {
            double acc = 0.0;
            if (e < E1) {  // Kt[a][c] += s sum_bd V D_bd
                const int a = e / NC, c = e % NC;
#pragma unroll
                for (int b = 0; b < NB; ++b)
#pragma unroll
                    for (int d = 0; d < ND; ++d) acc += sm[(a * NB + b) * NCDP + c * ND + d] * dBD[b * ND + d];
                atomicAdd(&args.K[(oa + a) * n + oc + c], s * acc);
            } else if (e < E2) {  // Kt[a][d] += s sum_bc V D_bc
                const int a = (e - E1) / ND, d = (e - E1) % ND;
#pragma unroll
                for (int b = 0; b < NB; ++b)
#pragma unroll
                    for (int c = 0; c < NC; ++c) acc += sm[(a * NB + b) * NCDP + c * ND + d] * dBC[b * NC + c];
                atomicAdd(&args.K[(oa + a) * n + od + d], s * acc);
            } else if (e < E3) {  // Kt[b][c] += s sum_ad V D_ad
                const int b = (e - E2) / NC, c = (e - E2) % NC;
#pragma unroll
                for (int a = 0; a < NA; ++a)
#pragma unroll
                    for (int d = 0; d < ND; ++d) acc += sm[(a * NB + b) * NCDP + c * ND + d] * dAD[a * ND + d];
                atomicAdd(&args.K[(ob + b) * n + oc + c], s * acc);
            } else {  // Kt[b][d] += s sum_ac V D_ac
                const int b = (e - E3) / ND, d = (e - E3) % ND;
#pragma unroll
                for (int a = 0; a < NA; ++a)
#pragma unroll
                    for (int c = 0; c < NC; ++c) acc += sm[(a * NB + b) * NCDP + c * ND + d] * dAC[a * NC + c];
                atomicAdd(&args.K[(ob + b) * n + od + d], s * acc);
            }
        }
    }
}

// Lanes per quartet for the cooperative form (0: one thread per quartet).
__host__ __device__ constexpr int jk_group(int la, int lb, int lc, int ld) {
    return (la == 2 && lb == 2 && lc == 2 && ld >= 1) ? 32
         : (la == 2 && lb == 2 && lc == 1 && ld == 1) ? 16
         : (la == 2 && lb == 1 && lc == 2 && ld == 1) ? 16
         : (la == 2 && lb == 2 && lc == 2 && ld == 0) ? 16
         : (la == 2 && lb == 1 && lc == 1 && ld == 1) ? 8
         : (la == 2 && lb == 2 && lc == 1 && ld == 0) ? 8
         : (la == 2 && lb == 1 && lc == 2 && ld == 0) ? 8
         : 0;
}

// One-quartet-per-thread form: the small component blocks split their primitive quartets over lanes,
// more lanes for the ket buckets with more primitive pairs.
__host__ __device__ constexpr bool jk_split(int la, int lb, int lc, int ld) {
    return ncart(la) * ncart(lb) * ncart(lc) * ncart(ld) <= 36;
}
// Lanes per quartet by ket bucket for the small-block classes: five candidate tables, one chosen per
// (bra class, ket class) by pdg_autotune_eri.  The default per class pair (pair classes ss, ps, pp,
// ds, dp, dd) is the autotuner's choice on a 14-heavy-atom organic molecule in B3LYP/6-31G*
// (Cartesian): table 3 (2-16 lanes) for (ss|ss), table 0 for (dp|ss) and (dd|ss), table 1 for the
// rest.
constexpr int kNLanesV = 5;
constexpr int kSplitLanesV[kNLanesV][PDG_NBUCKET] = {
    {1, 1, 1, 2, 2}, {1, 1, 2, 4, 4}, {1, 2, 4, 8, 8}, {2, 4, 8, 16, 16}, {4, 8, 16, 32, 32}};
constexpr int kDefaultLanesV[PDG_NPAIRCLASS][PDG_NPAIRCLASS] = {
    {3, 1, 1, 1, 1, 1}, {1, 1, 1, 1, 1, 1}, {1, 1, 1, 1, 1, 1},
    {1, 1, 1, 1, 1, 1}, {0, 1, 1, 1, 1, 1}, {0, 1, 1, 1, 1, 1}};
std::atomic<int> g_jk_variant[PDG_NPAIRCLASS][PDG_NPAIRCLASS];
struct VariantInit {
    VariantInit() {
        for (int i = 0; i < PDG_NPAIRCLASS; ++i)
            for (int j = 0; j < PDG_NPAIRCLASS; ++j) g_jk_variant[i][j].store(kDefaultLanesV[i][j]);
    }
} g_variant_init;
constexpr int kOneLane[PDG_NBUCKET] = {1, 1, 1, 1, 1};

constexpr int PLA[PDG_NPAIRCLASS] = {0, 1, 1, 2, 2, 2};
constexpr int PLB[PDG_NPAIRCLASS] = {0, 0, 1, 0, 1, 2};

template <int LA, int LB, int LC, int LD, int G, bool DOJ, bool DOK, typename T>
void launch_jk_group(JKArgs a, const QuartetBlock &b, cudaStream_t st) {
    using S = GroupShape<LA, LB, LC, LD, G>;
    const size_t smem = (size_t)S::SMEM * S::GPB * sizeof(double);
    auto kern = eri_jk_group_kernel<LA, LB, LC, LD, G, DOJ, DOK, T>;
    if (smem > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int lanes[PDG_NBUCKET] = {G, G, G, G, G};
    const long long blocks = pdg_fill_work(a.work, b, lanes);
    { kern<<<(unsigned)blocks, 128, smem, st>>>(a); pdg_count_launch(); }
}

template <int CB, int CK, typename T>
void launch_jk_p(JKArgs a, const QuartetBlock &b, bool doJ, bool doK, cudaStream_t st) {
    constexpr int LA = PLA[CB], LB = PLB[CB], LC = PLA[CK], LD = PLB[CK];
    constexpr int G = jk_group(LA, LB, LC, LD);
    if constexpr (G > 0) {
        if (doJ && doK) launch_jk_group<LA, LB, LC, LD, G, true, true, T>(a, b, st);
        else if (doJ) launch_jk_group<LA, LB, LC, LD, G, true, false, T>(a, b, st);
        else launch_jk_group<LA, LB, LC, LD, G, false, true, T>(a, b, st);
    } else {
        constexpr bool SP = jk_split(LA, LB, LC, LD);
        const int v = a.variant >= 0 ? a.variant : g_jk_variant[CB][CK].load(std::memory_order_relaxed);
        const long long blocks = pdg_fill_work(a.work, b, SP ? kSplitLanesV[v] : kOneLane);
        if (doJ && doK) { eri_jk_kernel<LA, LB, LC, LD, true, true, T, SP><<<(unsigned)blocks, 128, 0, st>>>(a); pdg_count_launch(); }
        else if (doJ) { eri_jk_kernel<LA, LB, LC, LD, true, false, T, SP><<<(unsigned)blocks, 128, 0, st>>>(a); pdg_count_launch(); }
        else { eri_jk_kernel<LA, LB, LC, LD, false, true, T, SP><<<(unsigned)blocks, 128, 0, st>>>(a); pdg_count_launch(); }
    }
}

template <int CB, int CK>
void launch_jk_t(const JKArgs &a, const QuartetBlock &b, bool doJ, bool doK, bool fp32, cudaStream_t st) {
    if (fp32) launch_jk_p<CB, CK, float>(a, b, doJ, doK, st);
    else launch_jk_p<CB, CK, double>(a, b, doJ, doK, st);
}

typedef void (*jk_launcher)(const JKArgs &, const QuartetBlock &, bool, bool, bool, cudaStream_t);

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

// Upload into the context's named buffer pool (grown when needed, never freed before the context
// is destroyed), stream-ordered on the context's non-blocking stream and complete on return, so a
// new geometry reuses the device memory of the last one without allocating.
template <typename T>
int upload(pdg_context *ctx, const std::string &name, T **dst, const std::vector<T> &src) {
    *dst = (T *)pdg_pool(ctx, name.c_str(), std::max<size_t>(1, src.size()) * sizeof(T));
    if (!*dst) { pdg_set_error("device buffer allocation failed (%s)", name.c_str()); return PDG_ERR_ALLOC; }
    if (src.empty()) return PDG_OK;
    PDG_CUDA(cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
    PDG_CUDA(cudaStreamSynchronize(ctx->stream));
    return PDG_OK;
}

std::string cname(const char *base, int c) { return std::string(base) + "." + std::to_string(c); }

}  // namespace

// Forget the shell-pair data of the last geometry; the device buffers stay in the context's pool.
void pdg_free_pairs(pdg_context *ctx) {
    for (int c = 0; c < PDG_NPAIRCLASS; ++c) ctx->pairs[c] = PairList{};
    ctx->pp = PrimPairs{};
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
    std::vector<double> va, vb, vPx, vPy, vPz, vK, varg, vKp, vhp;
    std::vector<int> pair_atomA;   // atom of the first centre of each primitive pair
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
                    vKp.push_back(vK.back() / p);
                    vhp.push_back(0.5 / p);
                    pair_atomA.push_back(sh[A].atom);
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
    PDG_CHECK(upload(ctx, "pp.a", &ctx->pp.a, va));
    PDG_CHECK(upload(ctx, "pp.b", &ctx->pp.b, vb));
    PDG_CHECK(upload(ctx, "pp.Px", &ctx->pp.Px, vPx));
    PDG_CHECK(upload(ctx, "pp.Py", &ctx->pp.Py, vPy));
    PDG_CHECK(upload(ctx, "pp.Pz", &ctx->pp.Pz, vPz));
    PDG_CHECK(upload(ctx, "pp.K", &ctx->pp.K, vK));
    PDG_CHECK(upload(ctx, "pp.arg", &ctx->pp.arg, varg));
    PDG_CHECK(upload(ctx, "pp.Kp", &ctx->pp.Kp, vKp));
    PDG_CHECK(upload(ctx, "pp.hp", &ctx->pp.hp, vhp));
    {
        std::vector<double> rec(8 * va.size());
        for (size_t i = 0; i < va.size(); ++i) {
            double *r = &rec[8 * i];
            r[0] = va[i] + vb[i]; r[1] = vPx[i]; r[2] = vPy[i]; r[3] = vPz[i];
            r[4] = vKp[i]; r[5] = vhp[i]; r[6] = varg[i]; r[7] = va[i];
        }
        double *drec = nullptr;
        PDG_CHECK(upload(ctx, "pp.rec", &drec, rec));
        ctx->pp.rec = reinterpret_cast<const double2 *>(drec);
        std::vector<float> rec32(8 * va.size());
        for (size_t i = 0; i < va.size(); ++i) {
            float *r = &rec32[8 * i];
            const double *rA = &ctx->xyz[3 * pair_atomA[i]];
            r[0] = (float)(va[i] + vb[i]);
            r[1] = (float)(vPx[i] - rA[0]); r[2] = (float)(vPy[i] - rA[1]); r[3] = (float)(vPz[i] - rA[2]);
            r[4] = (float)vKp[i]; r[5] = (float)vhp[i]; r[6] = (float)varg[i]; r[7] = 0.0f;
        }
        float *drec32 = nullptr;
        PDG_CHECK(upload(ctx, "pp.rec32", &drec32, rec32));
        ctx->pp.rec32 = reinterpret_cast<const float4 *>(drec32);
    }
    ctx->hostArg = varg;
    // Schwarz bounds on the unsorted lists, then sort each class by Q descending.
    for (int c = 0; c < PDG_NPAIRCLASS; ++c) {
        const int n = (int)cshA[c].size();
        ctx->hostQ[c].clear();
        ctx->bucket_start[c].assign(PDG_NBUCKET + 1, 0);
        ctx->qmax[c] = 0.0;
        if (n == 0) continue;
        int *dA = nullptr, *dB = nullptr, *dO = nullptr, *dN = nullptr;
        double *dQ = nullptr;
        PDG_CHECK(upload(ctx, "schwarz.A", &dA, cshA[c]));
        PDG_CHECK(upload(ctx, "schwarz.B", &dB, cshB[c]));
        PDG_CHECK(upload(ctx, "schwarz.O", &dO, cpoff[c]));
        PDG_CHECK(upload(ctx, "schwarz.N", &dN, cnp[c]));
        dQ = (double *)pdg_pool(ctx, "schwarz.Q", n * sizeof(double));
        if (!dQ) { pdg_set_error("device buffer allocation failed (schwarz.Q)"); return PDG_ERR_ALLOC; }
        schwarz_table[c](n, dA, dB, dO, dN, ctx->pp, ctx->dbasis, dQ, ctx->stream);
        PDG_CUDA(cudaGetLastError());
        std::vector<double> Q(n);
        PDG_CUDA(cudaMemcpyAsync(Q.data(), dQ, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        PDG_CUDA(cudaStreamSynchronize(ctx->stream));
        // by primitive-count bucket, then by Schwarz bound (descending) inside a bucket
        std::vector<int> order(n);
        std::iota(order.begin(), order.end(), 0);
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
            const int bx = np_bucket(cnp[c][x]), by = np_bucket(cnp[c][y]);
            return bx != by ? bx < by : Q[x] > Q[y];
        });
        std::vector<int> sA(n), sB(n), sO(n), sN(n);
        std::vector<double> sQ(n);
        for (int k = 0; k < n; ++k) {
            sA[k] = cshA[c][order[k]]; sB[k] = cshB[c][order[k]];
            sO[k] = cpoff[c][order[k]]; sN[k] = cnp[c][order[k]];
            sQ[k] = Q[order[k]];
        }
        PairList &pl = ctx->pairs[c];
        pl.n = n;
        PDG_CHECK(upload(ctx, cname("pairs.shA", c), &pl.shA, sA));
        PDG_CHECK(upload(ctx, cname("pairs.shB", c), &pl.shB, sB));
        PDG_CHECK(upload(ctx, cname("pairs.poff", c), &pl.poff, sO));
        PDG_CHECK(upload(ctx, cname("pairs.np", c), &pl.np, sN));
        PDG_CHECK(upload(ctx, cname("pairs.Q", c), &pl.Q, sQ));
        ctx->hostQ[c] = sQ;
        ctx->hostPoff[c] = sO;
        ctx->hostNp[c] = sN;
        ctx->qmax[c] = *std::max_element(sQ.begin(), sQ.end());
        auto &bs = ctx->bucket_start[c];
        bs.assign(PDG_NBUCKET + 1, n);
        for (int k = n - 1; k >= 0; --k) bs[np_bucket(sN[k])] = k;
        for (int k = PDG_NBUCKET - 1; k >= 0; --k) bs[k] = std::min(bs[k], bs[k + 1]);
    }
    return PDG_OK;
}

// cbra[k] = bra pair of quartet min(4k, total - 1) (binary search of the prefix sums).
__global__ void bra_map_kernel(const long long *__restrict__ offs, int nbra, long long total, long long nk,
                               int *__restrict__ cbra) {
    const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k >= nk) return;
    const long long t = min(4 * k, total - 1);
    int lo = 0, hi = nbra;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (offs[mid] <= t) lo = mid; else hi = mid;
    }
    cbra[k] = lo;
}

long long pdg_ket_count(const pdg_context *ctx, int cb, int ck, int ib, int k0, int nk, double thr) {
    const double qb = ctx->hostQ[cb][ib];
    if (!(qb > 0.0) || nk <= 0) return 0;
    const double need = thr / qb;
    const auto &Qk = ctx->hostQ[ck];
    // the bucket [k0, k0 + nk) is sorted by Q descending: the kets with Q >= need are a prefix
    long long cnt = std::upper_bound(Qk.begin() + k0, Qk.begin() + k0 + nk, need,
                                     [](double v, double e) { return v > e; }) - (Qk.begin() + k0);
    if (cb == ck) cnt = std::min<long long>(cnt, std::max<long long>(0, (long long)ib - k0 + 1));
    return cnt;
}

// Screened work list: for each (bra class >= ket class) block and each primitive-count bucket of the
// ket class, prefix sums over bra pairs of the number of ket pairs of the bucket with
// Q_bra * Q_ket >= thr; inside one class a quartet is counted once, with its ket at or before its bra
// in the class order.
int pdg_build_blocks(pdg_context *ctx, double thr) {
    if (ctx->blocks_thr == thr && !ctx->blocks.empty()) return PDG_OK;
    ctx->blocks.clear();
    int nbuf = 0;
    for (int cb = 0; cb < PDG_NPAIRCLASS; ++cb) {
        const auto &Qb = ctx->hostQ[cb];
        if (Qb.empty()) continue;
        for (int ck = 0; ck <= cb; ++ck) {
            if (ctx->hostQ[ck].empty()) continue;
            QuartetBlock qb{};
            qb.cb = cb;
            qb.ck = ck;
            for (int kb = 0; kb < PDG_NBUCKET; ++kb) {
                const int k0 = ctx->bucket_start[ck][kb], nk = ctx->bucket_start[ck][kb + 1] - k0;
                if (nk <= 0) continue;
                std::vector<long long> offs(Qb.size() + 1, 0);
                for (size_t i = 0; i < Qb.size(); ++i) offs[i + 1] = offs[i] + pdg_ket_count(ctx, cb, ck, (int)i, k0, nk, thr);
                if (offs.back() == 0) continue;
                auto &sb = qb.sub[qb.nsub++];
                sb.total = offs.back();
                sb.k0 = k0;
                sb.nk = nk;
                sb.bucket = kb;
                PDG_CHECK(upload(ctx, cname("blocks.offs", nbuf), &sb.offs, offs));
                const long long nmap = (sb.total - 1) / 4 + 2;
                sb.cbra = (int *)pdg_pool(ctx, cname("blocks.cbra", nbuf).c_str(), nmap * sizeof(int));
                if (!sb.cbra) { pdg_set_error("device buffer allocation failed (blocks.cbra)"); return PDG_ERR_ALLOC; }
                { bra_map_kernel<<<(unsigned)((nmap + 255) / 256), 256, 0, ctx->stream>>>(sb.offs, (int)Qb.size(), sb.total, nmap, sb.cbra); pdg_count_launch(); }
                PDG_CUDA(cudaGetLastError());
                qb.total += sb.total;
                ++nbuf;
            }
            if (qb.nsub > 0) ctx->blocks.push_back(qb);
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
    const bool mixed = ctx->precision_mode == 1;
    const int ns = (int)ctx->shells.size();
    if (mixed && !d_dmax) {
        // the precision partition needs the density bound even without density screening
        double *dm = (double *)pdg_pool(ctx, "jk_dmax", (size_t)ns * ns * sizeof(double));
        if (!dm) { pdg_set_error("pdg_eri_jk: device buffer allocation failed"); return PDG_ERR_ALLOC; }
        PDG_CHECK(pdg_shell_pair_dmax(ctx, d_D, dm));
        d_dmax = dm;
        dcut = 0.0;
    }
    if (mixed && !ctx->d_count32) {
        ctx->d_count32 = (unsigned long long *)pdg_pool(ctx, "count32", sizeof(unsigned long long));
        if (!ctx->d_count32) { pdg_set_error("pdg_eri_jk: device buffer allocation failed"); return PDG_ERR_ALLOC; }
        PDG_CUDA(cudaMemsetAsync(ctx->d_count32, 0, sizeof(unsigned long long), ctx->stream));
    }
    long long nq = 0;
    ProfScope prof(ctx, "eri_jk");
    for (const auto &b : ctx->blocks) {
        JKArgs a;
        a.bra = ctx->pairs[b.cb];
        a.ket = ctx->pairs[b.ck];
        a.same = (b.cb == b.ck);
        a.pp = ctx->pp;
        a.bs = ctx->dbasis;
        a.D = d_D;
        a.J = d_J;
        a.K = d_K;
        a.n = ctx->nbf;
        a.underflow = ctx->tei_underflow;
        a.dmax = d_dmax;
        a.nshell = ns;
        a.dcut = dcut;
        a.mixed_cut = ctx->mixed_cut;
        a.count32 = ctx->d_count32;
        a.variant = -1;
        if (mixed) {
            // quartets whose bound Q_AB Q_CD max|D| is below mixed_cut in FP32, the rest in FP64
            a.part = 1;
            jk_table[b.cb][b.ck](a, b, doJ, doK, false, ctx->stream);
            PDG_CUDA(cudaGetLastError());
            a.part = 2;
            jk_table[b.cb][b.ck](a, b, doJ, doK, true, ctx->stream);
        } else {
            a.part = 0;
            jk_table[b.cb][b.ck](a, b, doJ, doK, false, ctx->stream);
        }
        PDG_CUDA(cudaGetLastError());
        nq += b.total;
    }
    ctx->last_quartets = nq;
    return PDG_OK;
}

// Tile autotuner of the one-thread J+K kernels: for every (bra class, ket class) work list of the
// current geometry whose kernel splits quartets over lanes, time each candidate lanes-per-bucket
// table (one warm-up launch, then the best of two CUDA-event-timed launches of a full J+K build of
// the context's current density into scratch matrices) and keep the fastest in the process-wide
// table every later build of every context uses.  variants (36 ints, may be NULL) receives the
// choice per class pair (-1 where nothing was tuned).
extern "C" int pdg_autotune_eri(pdg_context *ctx, int *variants) {
    if (!ctx) { pdg_set_error("pdg_autotune_eri: invalid argument"); return PDG_ERR_ARG; }
    if (ctx->nbf == 0 || !ctx->have_geometry) { pdg_set_error("pdg_autotune_eri: basis and geometry required"); return PDG_ERR_STATE; }
    cudaSetDevice(ctx->device);
    PDG_CHECK(pdg_ensure_pairs(ctx));
    PDG_CHECK(pdg_build_blocks(ctx, ctx->schwarz_cut));
    const size_t nn = (size_t)ctx->nbf * ctx->nbf * sizeof(double);
    double *J = (double *)pdg_pool(ctx, "tune.J", nn), *K = (double *)pdg_pool(ctx, "tune.K", nn);
    if (!J || !K) { pdg_set_error("pdg_autotune_eri: device buffer allocation failed"); return PDG_ERR_ALLOC; }
    if (variants)
        for (int k = 0; k < PDG_NPAIRCLASS * PDG_NPAIRCLASS; ++k) variants[k] = -1;
    cudaEvent_t e0, e1;
    PDG_CUDA(cudaEventCreate(&e0));
    PDG_CUDA(cudaEventCreate(&e1));
    int status = PDG_OK;
    for (const auto &b : ctx->blocks) {
        const int la = PLA[b.cb], lb = PLB[b.cb], lc = PLA[b.ck], ld = PLB[b.ck];
        if (jk_group(la, lb, lc, ld) > 0 || !jk_split(la, lb, lc, ld)) continue;
        JKArgs a;
        a.bra = ctx->pairs[b.cb];
        a.ket = ctx->pairs[b.ck];
        a.same = (b.cb == b.ck);
        a.pp = ctx->pp;
        a.bs = ctx->dbasis;
        a.D = ctx->d_D;
        a.J = J;
        a.K = K;
        a.n = ctx->nbf;
        a.underflow = ctx->tei_underflow;
        a.dmax = nullptr;
        a.nshell = (int)ctx->shells.size();
        a.dcut = 0.0;
        a.mixed_cut = ctx->mixed_cut;
        a.count32 = nullptr;
        a.part = 0;
        int best = kDefaultLanesV[b.cb][b.ck];
        float best_ms = 1e30f;
        for (int v = 0; v < kNLanesV && status == PDG_OK; ++v) {
            a.variant = v;
            float ms_v = 1e30f;
            for (int rep = 0; rep < 3; ++rep) {
                cudaEventRecord(e0, ctx->stream);
                jk_table[b.cb][b.ck](a, b, true, true, false, ctx->stream);
                cudaEventRecord(e1, ctx->stream);
                if (cudaEventSynchronize(e1) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
                    pdg_set_error("pdg_autotune_eri: a timed launch failed");
                    status = PDG_ERR_CUDA;
                    break;
                }
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (rep > 0 && ms < ms_v) ms_v = ms;
            }
            if (ms_v < best_ms) { best_ms = ms_v; best = v; }
        }
        if (status != PDG_OK) break;
        g_jk_variant[b.cb][b.ck].store(best);
        if (variants) variants[b.cb * PDG_NPAIRCLASS + b.ck] = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return status;
}
