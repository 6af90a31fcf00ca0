// Device-side exchange-correlation functionals (FP64).
//
// Each functional is written in its open-shell form f(rhoA, rhoB, gAA, gAB, gBB)
// with first derivatives, following the reference's formulas; the closed-shell
// grid path evaluates it at rhoB = rhoA, gAB = gBB = gAA exactly as
// DfFunctional_{LDA,GGA}'s closed-shell overloads do
// (src/libpdf/DfFunctional.h:98-126, :182-233).
//   Slater       src/libpdf/DfFunctional_Slater.cpp:25-85
//   VWN5 / VWN3  src/libpdf/DfFunctional_VWN.cpp:19-340, DfFunctional_VWN3.cpp:21-54
//   Becke 88     src/libpdf/DfFunctional_Becke88.cpp:25-165 (+ _ExceptLDA.cpp:25-32)
//   LYP          src/libpdf/DfFunctional_LYP.cpp:25-675
//   composites   SVWN (DfFunctional_SVWN.cpp:25-41), B88LYP (DfFunctional_B88LYP.cpp),
//                B3LYP 0.80/0.72/0.19/0.81 (DfFunctional_B3LYP.cpp:25-150)
//   PBE          not in the reference: pbe.cuh (Perdew-Burke-Ernzerhof 1996, PW92 correlation)
// Transcendentals are CUDA's own pow/exp/log/atan/sqrt.
#pragma once

#include "pbe.cuh"

namespace pdfxc {

struct XcOut {
    double f, va, vb, vgaa, vgab, vgbb;
};

namespace fdetail {

__device__ __forceinline__ void slater(double ra, double rb, double& f, double& va, double& vb) {
    const double k = 3.0 / (4.0 * M_PI);
    const double ck = pow(k, 1.0 / 3.0);
    const double coef = -(9.0 / 4.0) * ck * (2.0 / 3.0);
    const double dcoef = -3.0 * ck * (2.0 / 3.0);
    f = coef * (pow(ra, 4.0 / 3.0) + pow(rb, 4.0 / 3.0));
    va = dcoef * pow(ra, 1.0 / 3.0);
    vb = dcoef * pow(rb, 1.0 / 3.0);
}

struct VwnPar {
    double A, b, c, x0;
};

__device__ __forceinline__ double vwn_eps(const VwnPar p, double x) {
    const double X = x * (x + p.b) + p.c;
    const double X0 = p.x0 * (p.x0 + p.b) + p.c;
    const double Q = sqrt(4 * p.c - p.b * p.b);
    const double at = atan(Q / (2.0 * x + p.b));
    const double xx0 = x - p.x0;
    return p.A * (log(x * x / X) + 2.0 * p.b / Q * at -
                  p.b * p.x0 / X0 * (log(xx0 * xx0 / X) + 2.0 * (2.0 * p.x0 + p.b) / Q * at));
}

__device__ __forceinline__ double vwn_eps_prime(const VwnPar p, double x) {
    const double X = x * (x + p.b) + p.c;
    const double X0 = p.x0 * (p.x0 + p.b) + p.c;
    const double Q = sqrt(4 * p.c - p.b * p.b);
    const double x2b = 2.0 * x + p.b;
    const double inv = 1.0 / (x2b * x2b + Q * Q);
    return p.A * (2.0 / x - x2b / X - 4.0 * p.b * inv -
                  p.b * p.x0 / X0 * (2.0 / (x - p.x0) - x2b / X - 4.0 * (2.0 * p.x0 + p.b) * inv));
}

// v3 = true: the VWN3 paramagnetic/ferromagnetic sets (B3LYP); false: VWN5.
__device__ __forceinline__ void vwn(bool v3, double ra, double rb, double& f, double& va, double& vb) {
    const VwnPar P = v3 ? VwnPar{0.0310907, 13.0720, 42.7198, -0.409286}
                        : VwnPar{0.0310907, 3.72744, 12.9352, -0.10498};
    const VwnPar F = v3 ? VwnPar{0.01554535, 20.1231, 101.578, -0.743294}
                        : VwnPar{0.01554535, 7.06042, 18.0578, -0.325};
    const VwnPar A = VwnPar{-1.0 / (6.0 * M_PI * M_PI), 1.13107, 13.0045, -0.0047584};
    const double ec_coef = 4.0 / (9.0 * (pow(2.0, 1.0 / 3.0) - 1.0));
    const double rho = ra + rb;
    const double inv = 1.0 / rho;
    const double x = pow(3.0 / (4.0 * M_PI) * inv, 1.0 / 6.0);
    const double zeta = (ra - rb) * inv;
    const double ep = vwn_eps(P, x), ef = vwn_eps(F, x), ea = vwn_eps(A, x);
    const double g = 9.0 / 8.0 * (pow(1.0 + zeta, 4.0 / 3.0) + pow(1.0 - zeta, 4.0 / 3.0) - 2.0);
    const double z3 = zeta * zeta * zeta, z4 = z3 * zeta;
    const double EC = ep + ea * g * (1.0 + (ec_coef * (ef - ep) / ea - 1.0) * z4);
    f = rho * EC;
    const double epp = vwn_eps_prime(P, x), efp = vwn_eps_prime(F, x), eap = vwn_eps_prime(A, x);
    const double gp = 1.5 * (pow(1.0 + zeta, 1.0 / 3.0) - pow(1.0 - zeta, 1.0 / 3.0));
    const double h = ec_coef * ((ef - ep) / ea) - 1.0;
    const double hp = ec_coef / ea * (efp - epp - (ef - ep) / ea * eap);
    const double t1 = -x / (6.0 * rho) * (epp + eap * g * (1.0 + h * z4) + ea * g * hp * z4);
    const double t2c = ea * (gp * (1.0 + h * z4) + 4.0 * g * h * z3);
    va = (ra > 1.0e-20) ? EC + rho * (t1 + t2c * (inv * (1.0 - zeta))) : 0.0;
    vb = (rb > 1.0e-20) ? EC + rho * (t1 + t2c * (-inv * (1.0 + zeta))) : 0.0;
}

__device__ __forceinline__ double b88_g(double x, bool full) {
    const double beta = 0.0042;
    const double G = -(3.0 / 2.0) * pow(3.0 / (4.0 * M_PI), 1.0 / 3.0);
    const double bx = beta * x;
    const double as = log(x + sqrt(x * x + 1));
    return (full ? G : 0.0) - (bx * x) / (1.0 + 6.0 * bx * as);
}

__device__ __forceinline__ double b88_gp(double x) {
    const double beta = 0.0042;
    const double bx = beta * x;
    const double as = log(x + sqrt(x * x + 1));
    const double M = 1.0 + 6.0 * bx * as;
    return 6.0 * bx * bx * (as + x / sqrt(x * x + 1.0)) / (M * M) - 2.0 * bx / M;
}

__device__ __forceinline__ void b88(bool full, double ra, double rb, double gaa, double gbb, double& f,
                                    double& va, double& vb, double& vgaa, double& vgbb) {
    const double EPS = 1.0e-16;
    double tA = 0.0, tB = 0.0;
    if (ra > EPS) tA = pow(ra, 4.0 / 3.0) * b88_g(sqrt(gaa) / pow(ra, 4.0 / 3.0), full);
    if (rb > EPS) tB = pow(rb, 4.0 / 3.0) * b88_g(sqrt(gbb) / pow(rb, 4.0 / 3.0), full);
    f = tA + tB;
    va = vb = vgaa = vgbb = 0.0;
    if (ra > EPS && gaa > EPS) {
        const double x = sqrt(gaa) / pow(ra, 4.0 / 3.0);
        const double g = b88_g(x, full), gp = b88_gp(x);
        va = 4.0 / 3.0 * pow(ra, 1.0 / 3.0) * (g - x * gp);
        vgaa = 0.5 / sqrt(gaa) * gp;
    }
    if (rb > EPS && gbb > EPS) {
        const double x = sqrt(gbb) / pow(rb, 4.0 / 3.0);
        const double g = b88_g(x, full), gp = b88_gp(x);
        vb = 4.0 / 3.0 * pow(rb, 1.0 / 3.0) * (g - x * gp);
        vgbb = 0.5 / sqrt(gbb) * gp;
    }
}

constexpr double LA = 0.04918, LB = 0.132, LC = 0.2533, LD = 0.349;

__device__ __forceinline__ double lyp_coef() {
    return pow(2.0, 11.0 / 3.0) * 0.3 * pow(3.0 * M_PI * M_PI, 2.0 / 3.0);
}
__device__ __forceinline__ double lyp_omega(double rho) {
    const double m13 = pow(rho, -1.0 / 3.0);
    return exp(-LC * m13) * pow(rho, -11.0 / 3.0) / (1.0 + LD * m13);
}
__device__ __forceinline__ double lyp_delta(double rho) {
    const double m13 = pow(rho, -1.0 / 3.0);
    return LC * m13 + LD * m13 / (1.0 + LD * m13);
}
__device__ __forceinline__ void lyp_dgamma(double rho, double ra, double rb, double om, double de,
                                           double& gaa, double& gab, double& gbb) {
    const double rab = ra * rb, abo = LA * LB * om;
    gaa = -abo * (1.0 / 9.0 * rab * (1.0 - 3.0 * de - (de - 11.0) * ra / rho) - rb * rb);
    gbb = -abo * (1.0 / 9.0 * rab * (1.0 - 3.0 * de - (de - 11.0) * rb / rho) - ra * ra);
    gab = -abo * (1.0 / 9.0 * rab * (47.0 - 7.0 * de) - 4.0 / 3.0 * rho * rho);
}

__device__ __forceinline__ double lyp_f(double ra, double rb, double gaa, double gab, double gbb) {
    const double rho = ra + rb, rab = ra * rb;
    const double om = lyp_omega(rho), de = lyp_delta(rho);
    double daa, dab, dbb;
    lyp_dgamma(rho, ra, rb, om, de, daa, dab, dbb);
    const double t1 = -4.0 * LA / (1.0 + LD * pow(rho, -1.0 / 3.0)) * rab / rho;
    const double t2 = -lyp_coef() * LA * LB * om * rab * (pow(ra, 8.0 / 3.0) + pow(rb, 8.0 / 3.0));
    return t1 + t2 + daa * gaa + dab * gab + dbb * gbb;
}

__device__ __forceinline__ void lyp_v(double ra, double rb, double gaa, double gab, double gbb,
                                      double& va, double& vb, double& vgaa, double& vgab,
                                      double& vgbb) {
    const double TOL = 1.0e-20;
    va = vb = vgaa = vgab = vgbb = 0.0;
    if (!(fabs(ra) > TOL && fabs(rb) > TOL)) return;
    const double rho = ra + rb, rab = ra * rb, ir = 1.0 / rho;
    const double r13 = pow(rho, 1.0 / 3.0), rm13 = 1.0 / r13, rm43 = pow(rho, -4.0 / 3.0);
    const double ra83 = pow(ra, 8.0 / 3.0), rb83 = pow(rb, 8.0 / 3.0);
    const double om = lyp_omega(rho), abo = LA * LB * om;
    const double omp = -1.0 / 3.0 * (ir * rm13) * om * (11.0 * r13 - LC - LD / (1.0 + LD * rm13));
    const double de = lyp_delta(rho);
    const double d1 = 1.0 + LD * pow(rho, -1.0 / 3.0);
    const double dep = 1.0 / 3.0 * (LD * LD * pow(rho, -5.0 / 3.0) / (d1 * d1) - ir * de);
    const double opo = -1.0 / 3.0 * pow(rho, -4.0 / 3.0) *
                       (11.0 * pow(rho, 1.0 / 3.0) - LC - LD / (1.0 + LD * pow(rho, -1.0 / 3.0)));
    double daa, dab, dbb;
    lyp_dgamma(rho, ra, rb, om, de, daa, dab, dbb);
    const double ra_aa = opo * daa - abo * (1.0 / 9.0 * rb * (1.0 - 3.0 * de - (de - 11.0) * ra * ir) -
                                            1.0 / 9.0 * rab * ((3.0 + ra * ir) * dep + (de - 11.0) * rb * ir * ir));
    const double rb_bb = opo * dbb - abo * (1.0 / 9.0 * ra * (1.0 - 3.0 * de - (de - 11.0) * rb * ir) -
                                            1.0 / 9.0 * rab * ((3.0 + rb * ir) * dep + (de - 11.0) * ra * ir * ir));
    const double t21 = 1.0 / 9.0 * (47.0 - 7.0 * de), t22 = -7.0 / 9.0 * rab * dep - 8.0 / 3.0 * rho;
    const double ra_ab = opo * dab - abo * (t21 * rb + t22);
    const double rb_ab = opo * dab - abo * (t21 * ra + t22);
    const double ra_bb = opo * dbb - abo * (1.0 / 9.0 * rb * (1.0 - 3.0 * de - (de - 11.0) * rb * ir) -
                                            1.0 / 9.0 * rab * ((3.0 + rb * ir) * dep - (de - 11.0) * rb * ir * ir) -
                                            2.0 * ra);
    const double rb_aa = opo * daa - abo * (1.0 / 9.0 * ra * (1.0 - 3.0 * de - (de - 11.0) * ra * ir) -
                                            1.0 / 9.0 * rab * ((3.0 + ra * ir) * dep - (de - 11.0) * ra * ir * ir) -
                                            2.0 * rb);
    const double a1c = -4.0 * LA / (1.0 + LD * rm13) * rab / rho;
    const double a1A = a1c * (1.0 / 3.0 * LD * rm43 / (1.0 + LD * rm13) + 1.0 / ra - ir);
    const double a1B = a1c * (1.0 / 3.0 * LD * rm43 / (1.0 + LD * rm13) + 1.0 / rb - ir);
    const double lc = lyp_coef();
    const double a2A = -lc * LA * LB * (omp * rab * (ra83 + rb83) + om * rb * (11.0 / 3.0 * ra83 + rb83));
    const double a2B = -lc * LA * LB * (omp * rab * (rb83 + ra83) + om * ra * (11.0 / 3.0 * rb83 + ra83));
    if (ra > TOL) {
        va = a1A + a2A + ra_aa * gaa + ra_ab * gab + ra_bb * gbb;
        vgaa = daa;
    }
    if (rb > TOL) {
        vb = a1B + a2B + rb_aa * gaa + rb_ab * gab + rb_bb * gbb;
        vgbb = dbb;
    }
    if (ra > TOL && rb > TOL) vgab = dab;
}

}  // namespace fdetail

__host__ __device__ constexpr bool functional_is_gga(int fn) { return fn == 2 || fn == 3 || fn == 4 || fn == 5; }

__device__ __forceinline__ XcOut eval_functional(int fn, double ra, double rb, double gaa, double gab,
                                                 double gbb) {
    using namespace fdetail;
    XcOut o{0, 0, 0, 0, 0, 0};
    double f1, a1, b1, f2, a2, b2, g1, g2, g3, g4, g5;
    switch (fn) {
        case 0:  // SVWN
            slater(ra, rb, f1, a1, b1);
            vwn(false, ra, rb, f2, a2, b2);
            o.f = f1 + f2, o.va = a1 + a2, o.vb = b1 + b2;
            break;
        case 1:  // HFS
            slater(ra, rb, o.f, o.va, o.vb);
            break;
        case 2:  // HFB
            b88(true, ra, rb, gaa, gbb, o.f, o.va, o.vb, o.vgaa, o.vgbb);
            break;
        case 3:  // BLYP
            b88(true, ra, rb, gaa, gbb, f1, a1, b1, g1, g3);
            f2 = lyp_f(ra, rb, gaa, gab, gbb);
            lyp_v(ra, rb, gaa, gab, gbb, a2, b2, g2, g4, g5);
            o.f = f1 + f2, o.va = a1 + a2, o.vb = b1 + b2;
            o.vgaa = g1 + g2, o.vgab = g4, o.vgbb = g3 + g5;
            break;
        case 5: {  // PBE: value and the five first derivatives through dual numbers
            const Dual5 f = pbe::pbe(dvar(ra, 0), dvar(rb, 1), dvar(gaa, 2), dvar(gab, 3), dvar(gbb, 4));
            o.f = f.v, o.va = f.d[0], o.vb = f.d[1], o.vgaa = f.d[2], o.vgab = f.d[3], o.vgbb = f.d[4];
            break;
        }
        default: {  // B3LYP
            double fs, as, bs, fv, av, bv, fb, ab, bb, gba, gbb2, fl, al, bl, gla, glab, glb;
            slater(ra, rb, fs, as, bs);
            vwn(true, ra, rb, fv, av, bv);
            b88(false, ra, rb, gaa, gbb, fb, ab, bb, gba, gbb2);
            fl = lyp_f(ra, rb, gaa, gab, gbb);
            lyp_v(ra, rb, gaa, gab, gbb, al, bl, gla, glab, glb);
            o.f = 0.80 * fs + 0.72 * fb + 0.19 * fv + 0.81 * fl;
            o.va = 0.80 * as + 0.72 * ab + 0.19 * av + 0.81 * al;
            o.vb = 0.80 * bs + 0.72 * bb + 0.19 * bv + 0.81 * bl;
            o.vgaa = 0.72 * gba + 0.81 * gla;
            o.vgab = 0.81 * glab;
            o.vgbb = 0.72 * gbb2 + 0.81 * glb;
        }
    }
    return o;
}

}  // namespace pdfxc
