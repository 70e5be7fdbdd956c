// Spin-unpolarised exchange-correlation functionals for the device (and host), written from
// their published definitions with the parameter values of the libxc 1.2.0 copy the reference
// vendors (pMolecule/QCModel/__extensions__/cxc), including its density and gradient floors
// (MIN_DENS = MIN_GRAD = 5e-13, cxc/util.h:81-82; exchange: cxc/work_gga_x.i, correlation:
// cxc/work_gga_c.i).  Each functional returns the energy per volume F(rho, sigma) = rho e(rho, sigma)
// and its partial derivatives vrho = dF/drho, vsigma = dF/dsigma, obtained exactly by forward-mode
// dual numbers.  rho is the total density and sigma = |grad rho|^2.
//
//   LDA_X   Dirac/Slater exchange.
//   B88     A.D. Becke, Phys. Rev. A 38, 3098 (1988); beta = 0.0042, gamma = 6.
//   PBE_X   J.P. Perdew, K. Burke, M. Ernzerhof, PRL 77, 3865 (1996); kappa = 0.804,
//           mu = 0.2195149727645171.
//   PW92    J.P. Perdew, Y. Wang, PRB 45, 13244 (1992), zeta = 0, the "modified" parameters
//           libxc uses inside PBE correlation (A = 0.0310907).
//   PBE_C   PBE correlation, beta = 0.06672455060314922, gamma = (1 - ln 2)/pi^2.
//   VWN_RPA S.H. Vosko, L. Wilk, M. Nusair, Can. J. Phys. 58, 1200 (1980), RPA parameters.
//   LYP     C. Lee, W. Yang, R.G. Parr, PRB 37, 785 (1988) in the form of B. Miehlich,
//           A. Savin, H. Stoll, H. Preuss, CPL 157, 200 (1989); a = 0.04918, b = 0.132,
//           c = 0.2533, d = 0.349.
// Combinations (pMolecule/QCModel/DFTDefinitions.py:212-222, cxc/hyb_gga_xc_b3lyp.c:57-63):
//   pbe = PBE_X + PBE_C ; blyp = B88 + LYP ; lda = LDA_X + VWN(5) is not provided ;
//   b3lyp = 0.08 LDA_X + 0.72 B88 + 0.19 VWN_RPA + 0.81 LYP with 0.20 exact exchange.
#pragma once
#include <math.h>

#ifdef __CUDACC__
#define XC_HD __host__ __device__ __forceinline__
#else
#define XC_HD inline
#endif

namespace xc {

// Dual number with partial derivatives with respect to rho (d0) and sigma (d1).
struct D2 {
    double v, d0, d1;
};
XC_HD D2 mk(double v) { return {v, 0.0, 0.0}; }
XC_HD D2 operator+(D2 a, D2 b) { return {a.v + b.v, a.d0 + b.d0, a.d1 + b.d1}; }
XC_HD D2 operator-(D2 a, D2 b) { return {a.v - b.v, a.d0 - b.d0, a.d1 - b.d1}; }
XC_HD D2 operator-(D2 a) { return {-a.v, -a.d0, -a.d1}; }
XC_HD D2 operator*(D2 a, D2 b) { return {a.v * b.v, a.d0 * b.v + a.v * b.d0, a.d1 * b.v + a.v * b.d1}; }
XC_HD D2 operator/(D2 a, D2 b) {
    const double r = 1.0 / b.v, q = a.v * r;
    return {q, (a.d0 - q * b.d0) * r, (a.d1 - q * b.d1) * r};
}
XC_HD D2 operator+(D2 a, double b) { return {a.v + b, a.d0, a.d1}; }
XC_HD D2 operator+(double b, D2 a) { return {a.v + b, a.d0, a.d1}; }
XC_HD D2 operator-(D2 a, double b) { return {a.v - b, a.d0, a.d1}; }
XC_HD D2 operator-(double b, D2 a) { return {b - a.v, -a.d0, -a.d1}; }
XC_HD D2 operator*(D2 a, double b) { return {a.v * b, a.d0 * b, a.d1 * b}; }
XC_HD D2 operator*(double b, D2 a) { return {a.v * b, a.d0 * b, a.d1 * b}; }
XC_HD D2 operator/(D2 a, double b) { return {a.v / b, a.d0 / b, a.d1 / b}; }
XC_HD D2 operator/(double b, D2 a) {
    const double r = 1.0 / a.v, q = b * r;
    return {q, -q * r * a.d0, -q * r * a.d1};
}
XC_HD D2 chain(D2 a, double f, double df) { return {f, df * a.d0, df * a.d1}; }
XC_HD D2 dlog(D2 a) { return chain(a, log(a.v), 1.0 / a.v); }
XC_HD D2 dexp(D2 a) {
    const double e = exp(a.v);
    return chain(a, e, e);
}
XC_HD D2 dsqrt(D2 a) {
    const double s = sqrt(a.v);
    return chain(a, s, 0.5 / s);
}
XC_HD D2 dcbrt(D2 a) {
    const double c = cbrt(a.v);
    return chain(a, c, c / (3.0 * a.v));
}
XC_HD D2 datan(D2 a) { return chain(a, atan(a.v), 1.0 / (1.0 + a.v * a.v)); }
XC_HD D2 dasinh(D2 a) { return chain(a, asinh(a.v), 1.0 / sqrt(1.0 + a.v * a.v)); }

constexpr double MIN_DENS = 5.0e-13;
constexpr double MIN_GRAD = 5.0e-13;
constexpr double X_FACTOR_C = 0.9305257363491000250020102180716672510262;  // 3/8 (3/pi)^(1/3) 4^(2/3)
constexpr double X2S = 0.1282782438530421943003109254455883701296;         // 1/(2 (6 pi^2)^(1/3))
constexpr double PI = 3.14159265358979323846;

// Exchange functionals of the reduced gradient x = |grad rho_s| / rho_s^(4/3) of one spin channel
// (rho_s = rho/2), F = 2 (-X_FACTOR_C) rho_s^(4/3) f(x).  The gradient floor of work_gga_x.i keeps
// |grad rho_s| >= MIN_GRAD, and vsigma vanishes below it.
template <typename Fx>
XC_HD D2 gga_exchange(D2 rho, D2 sigma, Fx fx) {
    const D2 ds = rho * 0.5;
    const D2 rho43 = ds * dcbrt(ds);  // rho_s^(4/3)
    D2 gdm;
    if (sqrt(sigma.v) * 0.5 > MIN_GRAD) gdm = dsqrt(sigma) * 0.5;
    else gdm = mk(MIN_GRAD);
    const D2 x = gdm / rho43;
    return 2.0 * (-X_FACTOR_C) * rho43 * fx(x);
}

struct B88F {
    XC_HD D2 operator()(D2 x) const {
        const double beta = 0.0042, gamma = 6.0;
        return 1.0 + (beta / X_FACTOR_C) * x * x / (1.0 + gamma * beta * x * dasinh(x));
    }
};
struct PBEXF {
    XC_HD D2 operator()(D2 x) const {
        const double kappa = 0.8040, mu = 0.2195149727645171;
        const D2 s = X2S * x;
        return 1.0 + kappa - kappa / (1.0 + (mu / kappa) * s * s);
    }
};
struct LDAXF {
    XC_HD D2 operator()(D2) const { return mk(1.0); }
};

XC_HD D2 lda_x(D2 rho) {
    // -3/4 (3/pi)^(1/3) rho^(4/3)
    return -0.7385587663820224058 * rho * dcbrt(rho);
}

XC_HD D2 rs_of(D2 rho) { return dcbrt(3.0 / (4.0 * PI * rho)); }

// PW92 paramagnetic correlation energy per particle (modified parameters).
XC_HD D2 pw92_ec(D2 rs) {
    const double A = 0.0310907, a1 = 0.21370, b1 = 7.5957, b2 = 3.5876, b3 = 1.6382, b4 = 0.49294;
    const D2 srs = dsqrt(rs);
    const D2 den = 2.0 * A * (b1 * srs + b2 * rs + b3 * rs * srs + b4 * rs * rs);
    return -2.0 * A * (1.0 + a1 * rs) * dlog(1.0 + 1.0 / den);
}

XC_HD D2 pbe_c(D2 rho, D2 sigma) {
    const double beta = 0.06672455060314922, gamma = (1.0 - 0.69314718055994530942) / (PI * PI);
    const D2 rs = rs_of(rho);
    const D2 ec = pw92_ec(rs);
    // work_gga_c.i clamps the value of sigma at MIN_GRAD^2 but keeps its derivative chain.
    D2 sg = sigma;
    if (sg.v < MIN_GRAD * MIN_GRAD) sg.v = MIN_GRAD * MIN_GRAD;
    const D2 xt = dsqrt(sg) / (rho * dcbrt(rho));
    const double tconv = 4.0 * 1.2599210498948731648;  // 4 2^(1/3)
    const D2 t = xt / (tconv * dsqrt(rs));
    const D2 A = (beta / gamma) / (dexp(-1.0 * ec / gamma) - 1.0);
    const D2 t2 = t * t;
    const D2 at2 = A * t2;
    const D2 H = gamma * dlog(1.0 + (beta / gamma) * t2 * (1.0 + at2) / (1.0 + at2 + at2 * at2));
    return rho * (ec + H);
}

XC_HD D2 vwn_rpa(D2 rho) {
    const double A = 0.0310907, b = 13.0720, c = 42.7198, x0 = -0.409286;
    const double Q = sqrt(4.0 * c - b * b);
    const double X0 = x0 * x0 + b * x0 + c;
    const double f1 = 2.0 * b / Q, f2 = b * x0 / X0, f3 = 2.0 * (2.0 * x0 + b) / Q;
    const D2 x = dsqrt(rs_of(rho));
    const D2 X = x * x + b * x + c;
    const D2 q = datan(Q / (2.0 * x + b));
    const D2 xx0 = x - x0;
    const D2 ec = A * (dlog(x * x / X) + (f1 - f2 * f3) * q - f2 * dlog(xx0 * xx0 / X));
    return rho * ec;
}

// LYP correlation for rho_a = rho_b = rho/2 and |grad rho_a|^2 = |grad rho_b|^2 = grad rho_a . grad rho_b = sigma/4.
XC_HD D2 lyp(D2 rho, D2 sigma) {
    const double a = 0.04918, b = 0.132, c = 0.2533, d = 0.349;
    const double CF = 0.3 * 9.5707800006273661;  // (3/10)(3 pi^2)^(2/3)
    const D2 rm13 = 1.0 / dcbrt(rho);
    const D2 den = 1.0 + d * rm13;
    const D2 omega = dexp(-c * rm13) / den / (rho * rho * rho * rho) * dcbrt(rho);  // rho^(-11/3)
    const D2 delta = c * rm13 + d * rm13 / den;
    const D2 ra = rho * 0.5;
    const D2 ga = sigma * 0.25;  // |grad rho_a|^2
    const D2 ra83 = ra * ra * dcbrt(ra * ra);  // ra^(8/3)
    const D2 t1 = -4.0 * a / den * ra * ra / rho;
    const D2 inner = 12.699208415745595 * CF * (ra83 + ra83) +
                     (47.0 / 18.0 - 7.0 / 18.0 * delta) * sigma - (2.5 - delta / 18.0) * (ga + ga) -
                     (delta - 11.0) / 9.0 * (ra / rho * ga + ra / rho * ga);
    const D2 t2 = ra * ra * inner - (2.0 / 3.0) * rho * rho * sigma + ((2.0 / 3.0) * rho * rho - ra * ra) * ga +
                  ((2.0 / 3.0) * rho * rho - ra * ra) * ga;
    return t1 - a * b * omega * t2;
}

enum Kind { NONE = 0, PBE = 1, BLYP = 2, B3LYP = 3, LDA_X_ONLY = 4, PW92_ONLY = 5, VWNRPA_ONLY = 6, LYP_ONLY = 7,
            B88_ONLY = 8, PBEX_ONLY = 9, PBEC_ONLY = 10 };

// Energy per volume and derivatives of the functional combination `kind` at one point.
// Points below the density floor contribute nothing (work_lda.i / work_gga_*.i skip them).
XC_HD void evaluate(int kind, double rho_v, double sigma_v, double *f, double *vrho, double *vsigma) {
    *f = 0.0;
    *vrho = 0.0;
    *vsigma = 0.0;
    if (rho_v < MIN_DENS) return;
    const D2 rho = {rho_v, 1.0, 0.0};
    const D2 sigma = {sigma_v, 0.0, 1.0};
    D2 F = mk(0.0);
    switch (kind) {
        case PBE: F = gga_exchange(rho, sigma, PBEXF()) + pbe_c(rho, sigma); break;
        case BLYP: F = gga_exchange(rho, sigma, B88F()) + lyp(rho, sigma); break;
        case B3LYP:
            F = 0.08 * lda_x(rho) + 0.72 * gga_exchange(rho, sigma, B88F()) + 0.19 * vwn_rpa(rho) + 0.81 * lyp(rho, sigma);
            break;
        case LDA_X_ONLY: F = lda_x(rho); break;
        case PW92_ONLY: F = rho * pw92_ec(rs_of(rho)); break;
        case VWNRPA_ONLY: F = vwn_rpa(rho); break;
        case LYP_ONLY: F = lyp(rho, sigma); break;
        case B88_ONLY: F = gga_exchange(rho, sigma, B88F()); break;
        case PBEX_ONLY: F = gga_exchange(rho, sigma, PBEXF()); break;
        case PBEC_ONLY: F = pbe_c(rho, sigma); break;
        default: break;
    }
    *f = F.v;
    *vrho = F.d0;
    *vsigma = F.d1;
}

}  // namespace xc
