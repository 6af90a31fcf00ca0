// PBE exchange-correlation (not in the reference; written from the published
// papers): J. P. Perdew, K. Burke, M. Ernzerhof, Phys. Rev. Lett. 77, 3865 (1996)
// for the gradient corrections, and J. P. Perdew, Y. Wang, Phys. Rev. B 45, 13244
// (1992) for the local correlation energy, with the parameter values of the PBE
// authors' reference implementation.
//
// Open-shell form f(rhoA, rhoB, gAA, gAB, gBB), energy per volume:
//   exchange    f_x = sum_s 1/2 e_x^unif(2 rho_s) F_x(s_s),  e_x^unif(n) = -3/4 (3/pi)^(1/3) n^(4/3),
//               s_s^2 = gamma_ss / ((3 pi^2 2 rho_s)^(2/3) (2 rho_s)^2),
//               F_x = 1 + kappa - kappa / (1 + mu s^2 / kappa)   (spin scaling of exchange);
//   correlation f_c = rho (eps_c(rs, zeta) + H(rs, zeta, t)),
//               eps_c = e0 + alpha_c f(zeta)/f''(0) (1 - zeta^4) + (e1 - e0) f(zeta) zeta^4 (PW92),
//               e0, e1, -alpha_c = G(rs; A, a1, b1..b4)
//                 = -2A (1 + a1 rs) ln(1 + 1 / (2A (b1 rs^1/2 + b2 rs + b3 rs^3/2 + b4 rs^2))),
//               H = gamma phi^3 ln(1 + beta/gamma t^2 (1 + A t^2) / (1 + A t^2 + A^2 t^4)),
//               A = beta/gamma / (exp(-eps_c / (gamma phi^3)) - 1),
//               phi = ((1 + zeta)^(2/3) + (1 - zeta)^(2/3)) / 2,
//               t^2 = |grad rho|^2 / (4 phi^2 k_s^2 rho^2), k_s^2 = 4 k_F / pi, k_F = (3 pi^2 rho)^(1/3),
//               |grad rho|^2 = gAA + 2 gAB + gBB.
// The five first derivatives come from forward-mode dual numbers through the same
// expression (one value and five tangents per operation), so energy and potential
// are one code path.
#pragma once

namespace pdfxc {

struct Dual5 {
    double v;
    double d[5];
};

__host__ __device__ inline Dual5 dconst(double c) {
    Dual5 r;
    r.v = c;
    for (int i = 0; i < 5; ++i) r.d[i] = 0.0;
    return r;
}
__host__ __device__ inline Dual5 dvar(double x, int k) {
    Dual5 r = dconst(x);
    r.d[k] = 1.0;
    return r;
}
// y = f(x) with f'(x) = fp: the chain rule on every tangent
__host__ __device__ inline Dual5 dchain(const Dual5& x, double fv, double fp) {
    Dual5 r;
    r.v = fv;
    for (int i = 0; i < 5; ++i) r.d[i] = fp * x.d[i];
    return r;
}
__host__ __device__ inline Dual5 operator+(const Dual5& a, const Dual5& b) {
    Dual5 r;
    r.v = a.v + b.v;
    for (int i = 0; i < 5; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
__host__ __device__ inline Dual5 operator-(const Dual5& a, const Dual5& b) {
    Dual5 r;
    r.v = a.v - b.v;
    for (int i = 0; i < 5; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
__host__ __device__ inline Dual5 operator*(const Dual5& a, const Dual5& b) {
    Dual5 r;
    r.v = a.v * b.v;
    for (int i = 0; i < 5; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
__host__ __device__ inline Dual5 operator/(const Dual5& a, const Dual5& b) {
    Dual5 r;
    const double ib = 1.0 / b.v;
    r.v = a.v * ib;
    for (int i = 0; i < 5; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
__host__ __device__ inline Dual5 operator+(const Dual5& a, double c) { return dchain(a, a.v + c, 1.0); }
__host__ __device__ inline Dual5 operator+(double c, const Dual5& a) { return dchain(a, a.v + c, 1.0); }
__host__ __device__ inline Dual5 operator-(const Dual5& a, double c) { return dchain(a, a.v - c, 1.0); }
__host__ __device__ inline Dual5 operator-(double c, const Dual5& a) { return dchain(a, c - a.v, -1.0); }
__host__ __device__ inline Dual5 operator-(const Dual5& a) { return dchain(a, -a.v, -1.0); }
__host__ __device__ inline Dual5 operator*(const Dual5& a, double c) { return dchain(a, a.v * c, c); }
__host__ __device__ inline Dual5 operator*(double c, const Dual5& a) { return dchain(a, a.v * c, c); }
__host__ __device__ inline Dual5 operator/(const Dual5& a, double c) { return dchain(a, a.v / c, 1.0 / c); }
__host__ __device__ inline Dual5 operator/(double c, const Dual5& a) {
    const double v = c / a.v;
    return dchain(a, v, -v / a.v);
}
__host__ __device__ inline Dual5 dexp(const Dual5& a) {
    const double e = exp(a.v);
    return dchain(a, e, e);
}
__host__ __device__ inline Dual5 dlog(const Dual5& a) { return dchain(a, log(a.v), 1.0 / a.v); }
__host__ __device__ inline Dual5 dsqrt(const Dual5& a) {
    const double s = sqrt(a.v);
    return dchain(a, s, 0.5 / s);
}
// a^c for a > 0
__host__ __device__ inline Dual5 dpow(const Dual5& a, double c) {
    const double p = pow(a.v, c);
    return dchain(a, p, c * p / a.v);
}

// scalar overloads so that the functional template also runs on plain doubles
__host__ __device__ inline double dexp(double a) { return exp(a); }
__host__ __device__ inline double dlog(double a) { return log(a); }
__host__ __device__ inline double dsqrt(double a) { return sqrt(a); }
__host__ __device__ inline double dpow(double a, double c) { return pow(a, c); }
__host__ __device__ inline double dval(double a) { return a; }
__host__ __device__ inline double dval(const Dual5& a) { return a.v; }
__host__ __device__ inline double dconst_like(double, double c) { return c; }
__host__ __device__ inline Dual5 dconst_like(const Dual5&, double c) { return dconst(c); }

namespace pbe {

constexpr double kPi = 3.14159265358979323846;
constexpr double kKappa = 0.804;
constexpr double kBeta = 0.06672455060314922;
constexpr double kMu = kBeta * kPi * kPi / 3.0;
constexpr double kGamma = 0.03109069086965489503494086371273;  // (1 - ln 2) / pi^2
constexpr double kGam = 0.5198420997897463295344212145565;      // 2^(4/3) - 2
constexpr double kFzz = 8.0 / (9.0 * kGam);                        // f''(0)
constexpr double kTiny = 1e-30;

template <class T>
__host__ __device__ inline T pw92_g(const T& rs, double A, double a1, double b1, double b2, double b3, double b4) {
    const T srs = dsqrt(rs);
    const T den = 2.0 * A * (b1 * srs + b2 * rs + b3 * rs * srs + b4 * rs * rs);
    return -2.0 * A * (1.0 + a1 * rs) * dlog(1.0 + 1.0 / den);
}

// exchange of one spin channel: 1/2 e_x^unif(2 rho_s) F_x(s_s)
template <class T>
__host__ __device__ inline T exchange_spin(const T& rs_, const T& g_) {
    const T n = 2.0 * rs_;
    const double cx = -0.75 * pow(3.0 / kPi, 1.0 / 3.0);
    const T n43 = dpow(n, 4.0 / 3.0);
    const T kf2n2 = dpow(3.0 * kPi * kPi * n, 2.0 / 3.0) * n * n;
    const T s2 = g_ / kf2n2;
    const T fx = 1.0 + kKappa - kKappa / (1.0 + kMu * s2 / kKappa);
    return 0.5 * cx * n43 * fx;
}

template <class T>
__host__ __device__ inline T pbe(const T& ra, const T& rb, const T& gaa, const T& gab, const T& gbb) {
    T f = dconst_like(ra, 0.0);
    if (dval(ra) > kTiny) f = f + exchange_spin(ra, gaa);
    if (dval(rb) > kTiny) f = f + exchange_spin(rb, gbb);
    const T rho = ra + rb;
    if (dval(rho) <= kTiny) return f;
    T zeta = (ra - rb) / rho;
    // fully polarised limits: keep (1 -+ zeta) positive for the fractional powers
    const double zmax = 1.0 - 1e-12;
    if (dval(zeta) > zmax) zeta = dconst_like(ra, zmax);
    if (dval(zeta) < -zmax) zeta = dconst_like(ra, -zmax);
    const T rs = dpow(3.0 / (4.0 * kPi) / rho, 1.0 / 3.0);
    const T e0 = pw92_g(rs, 0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294);
    const T e1 = pw92_g(rs, 0.01554535, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517);
    const T ac = -pw92_g(rs, 0.0168869, 0.11125, 10.357, 3.6231, 0.88026, 0.49671);
    const T opz = 1.0 + zeta, omz = 1.0 - zeta;
    const T fz = (dpow(opz, 4.0 / 3.0) + dpow(omz, 4.0 / 3.0) - 2.0) / kGam;
    const T z4 = zeta * zeta * zeta * zeta;
    const T ec = e0 + ac * fz * (1.0 - z4) / kFzz + (e1 - e0) * fz * z4;
    const T phi = 0.5 * (dpow(opz, 2.0 / 3.0) + dpow(omz, 2.0 / 3.0));
    const T phi3 = phi * phi * phi;
    const T kf = dpow(3.0 * kPi * kPi * rho, 1.0 / 3.0);
    const T ks2 = 4.0 * kf / kPi;
    const T grad2 = gaa + 2.0 * gab + gbb;
    const T t2 = grad2 / (4.0 * phi * phi * ks2 * rho * rho);
    const T A = (kBeta / kGamma) / (dexp(-ec / (kGamma * phi3)) - 1.0);
    const T at2 = A * t2;
    const T H = kGamma * phi3 * dlog(1.0 + (kBeta / kGamma) * t2 * (1.0 + at2) / (1.0 + at2 + at2 * at2));
    return f + rho * (ec + H);
}

}  // namespace pbe
}  // namespace pdfxc
