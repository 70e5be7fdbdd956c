// Rys two-dimensional integrals and horizontal transfers, written for compile-time
// angular momenta so that every array lives in registers.
//
// For one Rys node u = t^2 of a primitive quartet with bra exponent sum p (centre P),
// ket exponent sum q (centre Q) the 2D integrals G(e, f) of one Cartesian direction obey
// (Rys, Dupuis and King, J. Comput. Chem. 4, 154 (1983)):
//   G(0,0)   = 1
//   G(e+1,0) = C00 G(e,0) + e B10 G(e-1,0)
//   G(e,f+1) = C00' G(e,f) + f B01 G(e,f-1) + e B00 G(e-1,f)
// with C00 = (P-A) - q u (P-Q)/(p+q), C00' = (Q-C) + p u (P-Q)/(p+q),
// B00 = u/(2(p+q)), B10 = (1 - q u/(p+q))/(2p), B01 = (1 - p u/(p+q))/(2q).
// The transfer relations I(a,b+1) = I(a+1,b) + (A-B) I(a,b) (and the same on the ket)
// move angular momentum from the combined index to the second centre.  The reference
// performs the same steps with GaussianBasisSubsidiary_f1Cg1 / _f1Xg2i
// (GaussianBases/__extensions__/csource/GaussianBasisSubsidiary.c:88,480).
#pragma once
#include "common.cuh"

// T is the arithmetic type: double, or float for the quartets evaluated in single precision.
template <int LAB, int LCD, typename T = double>
__device__ __forceinline__ void rys_vrr(T (&G)[LAB + 1][LCD + 1], T g00, T c00, T c00p, T b10, T b01, T b00) {
    G[0][0] = g00;
    if constexpr (LAB > 0) {
        G[1][0] = c00 * g00;
#pragma unroll
        for (int e = 1; e < LAB; ++e) G[e + 1][0] = c00 * G[e][0] + e * b10 * G[e - 1][0];
    }
#pragma unroll
    for (int f = 0; f < LCD; ++f) {
        const int fm = f > 0 ? f - 1 : 0;
        const T fb01 = f * b01;
        G[0][f + 1] = c00p * G[0][f] + fb01 * G[0][fm];
#pragma unroll
        for (int e = 1; e <= LAB; ++e) G[e][f + 1] = c00p * G[e][f] + fb01 * G[e][fm] + e * b00 * G[e - 1][f];
    }
}

// Horizontal transfers on one direction: I[a][b][c][d] for a<=LA, b<=LB, c<=LC, d<=LD
// from G[e][f], e<=LA+LB, f<=LC+LD.  AB = A-B, CD = C-D.
template <int LA, int LB, int LC, int LD, typename R = double>
__device__ __forceinline__ void rys_hrr(const R (&G)[LA + LB + 1][LC + LD + 1], R AB, R CD,
                                        R (&I)[LA + 1][LB + 1][LC + 1][LD + 1]) {
    constexpr int LAB = LA + LB, LCD = LC + LD;
    R T[LAB + 1][LB + 1][LCD + 1];
#pragma unroll
    for (int a = 0; a <= LAB; ++a)
#pragma unroll
        for (int f = 0; f <= LCD; ++f) T[a][0][f] = G[a][f];
#pragma unroll
    for (int b = 1; b <= LB; ++b)
#pragma unroll
        for (int a = 0; a <= LAB - b; ++a)
#pragma unroll
            for (int f = 0; f <= LCD; ++f) T[a][b][f] = T[a + 1][b - 1][f] + AB * T[a][b - 1][f];
    R U[LA + 1][LB + 1][LCD + 1][LD + 1];
#pragma unroll
    for (int a = 0; a <= LA; ++a)
#pragma unroll
        for (int b = 0; b <= LB; ++b)
#pragma unroll
            for (int c = 0; c <= LCD; ++c) U[a][b][c][0] = T[a][b][c];
#pragma unroll
    for (int d = 1; d <= LD; ++d)
#pragma unroll
        for (int a = 0; a <= LA; ++a)
#pragma unroll
            for (int b = 0; b <= LB; ++b)
#pragma unroll
                for (int c = 0; c <= LCD - d; ++c) U[a][b][c][d] = U[a][b][c + 1][d - 1] + CD * U[a][b][c][d - 1];
#pragma unroll
    for (int a = 0; a <= LA; ++a)
#pragma unroll
        for (int b = 0; b <= LB; ++b)
#pragma unroll
            for (int c = 0; c <= LC; ++c)
#pragma unroll
                for (int d = 0; d <= LD; ++d) I[a][b][c][d] = U[a][b][c][d];
}
