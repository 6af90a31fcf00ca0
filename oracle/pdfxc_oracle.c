/*
 * pdfxc_oracle.c -- CPU restatement of ProteinDF's grid XC quadrature.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the oracle the CUDA path is checked
 * against: tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it through ctypes; the product (libpdfxc.so) never links or calls it.
 * It restates, in plain FP64 C, the arithmetic of the reference files cited
 * beside each function, and is itself pinned against the reference (the
 * functional known-answer tests of src/unit_test/DfFunctional_*Test.cpp and
 * the outputs of the reference harness oracle/_ref/pdfxc_ref).
 *
 * Functionals are evaluated through their open-shell forms
 * f(rhoA, rhoB, gAA, gAB, gBB); the closed-shell grid path calls them with
 * rhoB = rhoA and gAB = gBB = gAA, exactly as DfFunctional_{LDA,GGA}'s
 * closed-shell overloads do (src/libpdf/DfFunctional.h:98-126, :182-233).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { FN_SVWN = 0, FN_HFS = 1, FN_HFB = 2, FN_BLYP = 3, FN_B3LYP = 4, FN_PBE = 5 };

/* ---------------- PBE (not in the reference): Perdew, Burke, Ernzerhof, Phys. Rev.
 * Lett. 77, 3865 (1996) with the PW92 local correlation (Perdew, Wang, Phys. Rev. B
 * 45, 13244 (1992)), restated from the papers in complex arithmetic so that the
 * first derivatives follow by complex-step differentiation (Squire, Trapp 1998):
 * df/dx = Im f(x + i h) / h, h = 1e-30, exact to rounding for this analytic f.
 * Parity is unpinned (no reference implementation); the device's dual-number
 * derivatives and this restatement are independent. */
static double complex pbe_g(double complex rs, double A, double a1, double b1, double b2, double b3, double b4) {
    const double complex srs = csqrt(rs);
    const double complex den = 2.0 * A * (b1 * srs + b2 * rs + b3 * rs * srs + b4 * rs * rs);
    return -2.0 * A * (1.0 + a1 * rs) * clog(1.0 + 1.0 / den);
}

static double complex pbe_x_spin(double complex r, double complex g) {
    const double pi = M_PI, kappa = 0.804, mu = 0.06672455060314922 * M_PI * M_PI / 3.0;
    const double complex n = 2.0 * r;
    const double complex s2 = g / (cpow(3.0 * pi * pi * n, 2.0 / 3.0) * n * n);
    const double complex fx = 1.0 + kappa - kappa / (1.0 + mu * s2 / kappa);
    return 0.5 * (-0.75 * pow(3.0 / pi, 1.0 / 3.0)) * cpow(n, 4.0 / 3.0) * fx;
}

static double complex pbe_c(double complex ra, double complex rb, double complex gaa, double complex gab,
                            double complex gbb) {
    const double pi = M_PI, beta = 0.06672455060314922, gam = (1.0 - log(2.0)) / (pi * pi);
    const double tiny = 1e-30, zmax = 1.0 - 1e-12;
    const double fden = pow(2.0, 4.0 / 3.0) - 2.0, fzz = 8.0 / (9.0 * fden);
    double complex f = 0.0;
    if (creal(ra) > tiny) f += pbe_x_spin(ra, gaa);
    if (creal(rb) > tiny) f += pbe_x_spin(rb, gbb);
    const double complex rho = ra + rb;
    if (creal(rho) <= tiny) return f;
    double complex z = (ra - rb) / rho;
    if (creal(z) > zmax) z = zmax;
    if (creal(z) < -zmax) z = -zmax;
    const double complex rs = cpow(3.0 / (4.0 * pi * rho), 1.0 / 3.0);
    const double complex e0 = pbe_g(rs, 0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294);
    const double complex e1 = pbe_g(rs, 0.01554535, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517);
    const double complex ac = -pbe_g(rs, 0.0168869, 0.11125, 10.357, 3.6231, 0.88026, 0.49671);
    const double complex fz = (cpow(1.0 + z, 4.0 / 3.0) + cpow(1.0 - z, 4.0 / 3.0) - 2.0) / fden;
    const double complex z4 = z * z * z * z;
    const double complex ec = e0 + ac * fz * (1.0 - z4) / fzz + (e1 - e0) * fz * z4;
    const double complex phi = 0.5 * (cpow(1.0 + z, 2.0 / 3.0) + cpow(1.0 - z, 2.0 / 3.0));
    const double complex phi3 = phi * phi * phi;
    const double complex ks2 = 4.0 * cpow(3.0 * pi * pi * rho, 1.0 / 3.0) / pi;
    const double complex t2 = (gaa + 2.0 * gab + gbb) / (4.0 * phi * phi * ks2 * rho * rho);
    const double complex A = (beta / gam) / (cexp(-ec / (gam * phi3)) - 1.0);
    const double complex at2 = A * t2;
    const double complex H = gam * phi3 * clog(1.0 + (beta / gam) * t2 * (1.0 + at2) / (1.0 + at2 + at2 * at2));
    return f + rho * (ec + H);
}

static void pbe(double ra, double rb, double gaa, double gab, double gbb, double* o) {
    const double h = 1e-30;
    const double x[5] = {ra, rb, gaa, gab, gbb};
    o[0] = creal(pbe_c(ra, rb, gaa, gab, gbb));
    for (int k = 0; k < 5; ++k) {
        double complex y[5];
        for (int i = 0; i < 5; ++i) y[i] = x[i] + (i == k ? h * I : 0.0);
        o[1 + k] = cimag(pbe_c(y[0], y[1], y[2], y[3], y[4])) / h;
    }
}

/* ---------------- Slater exchange: src/libpdf/DfFunctional_Slater.cpp:25-85 ---- */
static double slater_coef(void) { return -(9.0 / 4.0) * pow(3.0 / (4.0 * M_PI), 1.0 / 3.0) * (2.0 / 3.0); }
static double slater_dcoef(void) { return -3.0 * pow(3.0 / (4.0 * M_PI), 1.0 / 3.0) * (2.0 / 3.0); }

static void slater(double ra, double rb, double* f, double* va, double* vb) {
    *f = slater_coef() * (pow(ra, 4.0 / 3.0) + pow(rb, 4.0 / 3.0));
    *va = slater_dcoef() * pow(ra, 1.0 / 3.0);
    *vb = slater_dcoef() * pow(rb, 1.0 / 3.0);
}

/* ---------------- VWN correlation: src/libpdf/DfFunctional_VWN.cpp:19-340 ------ */
/* parameter sets (A, b, c, x0): paramagnetic, ferromagnetic, spin stiffness.
 * VWN5 (DfFunctional_VWN.cpp:34-46) and VWN3 (DfFunctional_VWN3.cpp:21-28;
 * VWN3 keeps VWN5's spin-stiffness set). */
typedef struct { double A, b, c, x0; } vwn_par;
static const vwn_par VWN5_P = {0.0310907, 3.72744, 12.9352, -0.10498};
static const vwn_par VWN5_F = {0.01554535, 7.06042, 18.0578, -0.325};
static const vwn_par VWN3_P = {0.0310907, 13.0720, 42.7198, -0.409286};
static const vwn_par VWN3_F = {0.01554535, 20.1231, 101.578, -0.743294};

static vwn_par vwn_anti(void) {
    vwn_par p = {-1.0 / (6.0 * M_PI * M_PI), 1.13107, 13.0045, -0.0047584};
    return p;
}

/* eq. A13 (:181-208) */
static double vwn_eps(vwn_par p, double x) {
    const double X = x * (x + p.b) + p.c;
    const double X0 = p.x0 * (p.x0 + p.b) + p.c;
    const double Q = sqrt(4 * p.c - p.b * p.b);
    const double at = atan(Q / (2.0 * x + p.b));
    const double a1 = log(x * x / X);
    const double a2 = 2.0 * p.b / Q * at;
    const double xx0 = x - p.x0;
    const double a3 = -p.b * p.x0 / X0 * (log(xx0 * xx0 / X) + 2.0 * (2.0 * p.x0 + p.b) / Q * at);
    return p.A * (a1 + a2 + a3);
}

/* eq. A18 (:219-244) */
static double vwn_eps_prime(vwn_par p, double x) {
    const double X = x * (x + p.b) + p.c;
    const double X0 = p.x0 * (p.x0 + p.b) + p.c;
    const double Q = sqrt(4 * p.c - p.b * p.b);
    const double x2b = 2.0 * x + p.b;
    const double inv = 1.0 / (x2b * x2b + Q * Q);
    return p.A * (2.0 / x - x2b / X - 4.0 * p.b * inv -
                  p.b * p.x0 / X0 * (2.0 / (x - p.x0) - x2b / X - 4.0 * (2.0 * p.x0 + p.b) * inv));
}

static void vwn(int v3, double ra, double rb, double* f, double* va, double* vb) {
    const vwn_par P = v3 ? VWN3_P : VWN5_P, F = v3 ? VWN3_F : VWN5_F, A = vwn_anti();
    const double ec_coef = 4.0 / (9.0 * (pow(2.0, 1.0 / 3.0) - 1.0));
    const double rho = ra + rb;
    const double inv = 1.0 / rho;
    const double x = pow(3.0 / (4.0 * M_PI) * inv, 1.0 / 6.0);
    const double zeta = (ra - rb) * inv;
    const double ep = vwn_eps(P, x), ef = vwn_eps(F, x), ea = vwn_eps(A, x);
    const double g = 9.0 / 8.0 * (pow(1.0 + zeta, 4.0 / 3.0) + pow(1.0 - zeta, 4.0 / 3.0) - 2.0);
    const double z3 = zeta * zeta * zeta, z4 = z3 * zeta;
    const double EC = ep + ea * g * (1.0 + (ec_coef * (ef - ep) / ea - 1.0) * z4);
    *f = rho * EC;
    /* derivative, :278-338 */
    const double epp = vwn_eps_prime(P, x), efp = vwn_eps_prime(F, x), eap = vwn_eps_prime(A, x);
    const double gp = 1.5 * (pow(1.0 + zeta, 1.0 / 3.0) - pow(1.0 - zeta, 1.0 / 3.0));
    const double h = ec_coef * ((ef - ep) / ea) - 1.0;
    const double hp = ec_coef / ea * (efp - epp - (ef - ep) / ea * eap);
    const double t1 = -x / (6.0 * rho) * (epp + eap * g * (1.0 + h * z4) + ea * g * hp * z4);
    const double t2c = ea * (gp * (1.0 + h * z4) + 4.0 * g * h * z3);
    const double dzA = inv * (1.0 - zeta), dzB = -inv * (1.0 + zeta);
    *va = (ra > 1.0e-20) ? EC + rho * (t1 + t2c * dzA) : 0.0;
    *vb = (rb > 1.0e-20) ? EC + rho * (t1 + t2c * dzB) : 0.0;
}

/* ---------------- Becke 88 exchange: src/libpdf/DfFunctional_Becke88.cpp:25-165,
 * the "except LDA" variant drops the constant term of g
 * (src/libpdf/DfFunctional_Becke88_ExceptLDA.cpp:25-32). ------------------------ */
static double b88_g(double x, int full) {
    const double beta = 0.0042;
    const double G = -(3.0 / 2.0) * pow(3.0 / (4.0 * M_PI), 1.0 / 3.0);
    const double bx = beta * x;
    const double as = log(x + sqrt(x * x + 1));
    return (full ? G : 0.0) - (bx * x) / (1.0 + 6.0 * bx * as);
}

static double b88_gp(double x) {
    const double beta = 0.0042;
    const double bx = beta * x;
    const double as = log(x + sqrt(x * x + 1));
    const double M = 1.0 + 6.0 * bx * as;
    return 6.0 * bx * bx * (as + x / sqrt(x * x + 1.0)) / (M * M) - 2.0 * bx / M;
}

static void b88(int full, double ra, double rb, double gaa, double gbb, double* f, double* va,
                double* vb, double* vgaa, double* vgbb) {
    const double EPS = 1.0e-16;
    double tA = 0.0, tB = 0.0;
    if (ra > EPS) tA = pow(ra, 4.0 / 3.0) * b88_g(sqrt(gaa) / pow(ra, 4.0 / 3.0), full);
    if (rb > EPS) tB = pow(rb, 4.0 / 3.0) * b88_g(sqrt(gbb) / pow(rb, 4.0 / 3.0), full);
    *f = tA + tB;
    *va = *vb = *vgaa = *vgbb = 0.0;
    if (ra > EPS && gaa > EPS) {
        const double x = sqrt(gaa) / pow(ra, 4.0 / 3.0);
        const double g = b88_g(x, full), gp = b88_gp(x);
        *va = 4.0 / 3.0 * pow(ra, 1.0 / 3.0) * (g - x * gp);
        *vgaa = 0.5 / sqrt(gaa) * gp;
    }
    if (rb > EPS && gbb > EPS) {
        const double x = sqrt(gbb) / pow(rb, 4.0 / 3.0);
        const double g = b88_g(x, full), gp = b88_gp(x);
        *vb = 4.0 / 3.0 * pow(rb, 1.0 / 3.0) * (g - x * gp);
        *vgbb = 0.5 / sqrt(gbb) * gp;
    }
}

/* ---------------- LYP correlation: src/libpdf/DfFunctional_LYP.cpp:25-675 ----- */
static const double LA = 0.04918, LB = 0.132, LC = 0.2533, LD = 0.349;

static double lyp_coef(void) { return pow(2.0, 11.0 / 3.0) * 0.3 * pow(3.0 * M_PI * M_PI, 2.0 / 3.0); }

static double lyp_omega(double rho) {
    const double m13 = pow(rho, -1.0 / 3.0);
    return exp(-LC * m13) * pow(rho, -11.0 / 3.0) / (1.0 + LD * m13);
}

static double lyp_delta(double rho) {
    const double m13 = pow(rho, -1.0 / 3.0);
    return LC * m13 + LD * m13 / (1.0 + LD * m13);
}

static void lyp_dgamma(double rho, double ra, double rb, double om, double de, double* gaa,
                       double* gab, double* gbb) {
    const double rab = ra * rb, abo = LA * LB * om;
    *gaa = -abo * (1.0 / 9.0 * rab * (1.0 - 3.0 * de - (de - 11.0) * ra / rho) - rb * rb);
    *gbb = -abo * (1.0 / 9.0 * rab * (1.0 - 3.0 * de - (de - 11.0) * rb / rho) - ra * ra);
    *gab = -abo * (1.0 / 9.0 * rab * (47.0 - 7.0 * de) - 4.0 / 3.0 * rho * rho);
}

/* energy density, :340-366 */
static double lyp_f(double ra, double rb, double gaa, double gab, double gbb) {
    const double rho = ra + rb, rab = ra * rb;
    const double om = lyp_omega(rho), de = lyp_delta(rho);
    double daa, dab, dbb;
    lyp_dgamma(rho, ra, rb, om, de, &daa, &dab, &dbb);
    const double t1 = -4.0 * LA / (1.0 + LD * pow(rho, -1.0 / 3.0)) * rab / rho;
    const double t2 = -lyp_coef() * LA * LB * om * rab * (pow(ra, 8.0 / 3.0) + pow(rb, 8.0 / 3.0));
    return t1 + t2 + daa * gaa + dab * gab + dbb * gbb;
}

/* first derivatives, :63-185 with the mixed second derivatives of :507-595 */
static void lyp_v(double ra, double rb, double gaa, double gab, double gbb, double* va, double* vb,
                  double* vgaa, double* vgab, double* vgbb) {
    const double TOL = 1.0e-20;
    *va = *vb = *vgaa = *vgab = *vgbb = 0.0;
    if (!(fabs(ra) > TOL && fabs(rb) > TOL)) return;
    const double rho = ra + rb, rab = ra * rb, ir = 1.0 / rho;
    const double r13 = pow(rho, 1.0 / 3.0), rm13 = 1.0 / r13, rm43 = pow(rho, -4.0 / 3.0);
    const double ra83 = pow(ra, 8.0 / 3.0), rb83 = pow(rb, 8.0 / 3.0);
    const double om = lyp_omega(rho), abo = LA * LB * om;
    const double omp = -1.0 / 3.0 * (ir * rm13) * om * (11.0 * r13 - LC - LD / (1.0 + LD * rm13));
    const double de = lyp_delta(rho);
    const double d1 = 1.0 + LD * pow(rho, -1.0 / 3.0);
    const double dep = 1.0 / 3.0 * (LD * LD * pow(rho, -5.0 / 3.0) / (d1 * d1) - ir * de);
    /* mixed derivatives d2 f / d rho_s d gamma_t */
    const double opo = -1.0 / 3.0 * pow(rho, -4.0 / 3.0) *
                       (11.0 * pow(rho, 1.0 / 3.0) - LC - LD / (1.0 + LD * pow(rho, -1.0 / 3.0)));
    double daa, dab, dbb;
    lyp_dgamma(rho, ra, rb, om, de, &daa, &dab, &dbb);
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
    const double a2A = -lyp_coef() * LA * LB * (omp * rab * (ra83 + rb83) + om * rb * (11.0 / 3.0 * ra83 + rb83));
    const double a2B = -lyp_coef() * LA * LB * (omp * rab * (rb83 + ra83) + om * ra * (11.0 / 3.0 * rb83 + ra83));
    if (ra > TOL) {
        *va = a1A + a2A + ra_aa * gaa + ra_ab * gab + ra_bb * gbb;
        *vgaa = daa;
    }
    if (rb > TOL) {
        *vb = a1B + a2B + rb_aa * gaa + rb_ab * gab + rb_bb * gbb;
        *vgbb = dbb;
    }
    if (ra > TOL && rb > TOL) *vgab = dab;
}

/* ---------------- composites ----------------------------------------------------
 * SVWN = Slater + VWN5 (src/libpdf/DfFunctional_SVWN.cpp:25-41)
 * HFS  = Slater (src/libpdf/DfFunctional_HFS.cpp)
 * HFB  = Becke88 with the LDA term (DfXCFunctional.cpp:80-84 -> DfFunctional_Becke88)
 * BLYP = Becke88 + LYP (src/libpdf/DfFunctional_B88LYP.cpp:21-60)
 * B3LYP = 0.80 Slater + 0.72 B88(except LDA) + 0.19 VWN3 + 0.81 LYP
 *         (src/libpdf/DfFunctional_B3LYP.cpp:25-28, :50-150)
 * out: f, vrhoA, vrhoB, vgAA, vgAB, vgBB */
int pdfxc_oracle_functional(int fn, double ra, double rb, double gaa, double gab, double gbb,
                            double* out) {
    double f = 0, va = 0, vb = 0, vgaa = 0, vgab = 0, vgbb = 0;
    double f1, a1, b1, f2, a2, b2, g1, g2, g3, g4, g5;
    switch (fn) {
        case FN_SVWN:
            slater(ra, rb, &f1, &a1, &b1);
            vwn(0, ra, rb, &f2, &a2, &b2);
            f = f1 + f2, va = a1 + a2, vb = b1 + b2;
            break;
        case FN_HFS:
            slater(ra, rb, &f, &va, &vb);
            break;
        case FN_HFB:
            b88(1, ra, rb, gaa, gbb, &f, &va, &vb, &vgaa, &vgbb);
            break;
        case FN_BLYP:
            b88(1, ra, rb, gaa, gbb, &f1, &a1, &b1, &g1, &g3);
            f2 = lyp_f(ra, rb, gaa, gab, gbb);
            lyp_v(ra, rb, gaa, gab, gbb, &a2, &b2, &g2, &g4, &g5);
            f = f1 + f2, va = a1 + a2, vb = b1 + b2, vgaa = g1 + g2, vgab = g4, vgbb = g3 + g5;
            break;
        case FN_B3LYP: {
            double fs, as, bs, fv, av, bv, fb, ab, bb, gba, gbb2, fl, al, bl, gla, glab, glb;
            slater(ra, rb, &fs, &as, &bs);
            vwn(1, ra, rb, &fv, &av, &bv);
            b88(0, ra, rb, gaa, gbb, &fb, &ab, &bb, &gba, &gbb2);
            fl = lyp_f(ra, rb, gaa, gab, gbb);
            lyp_v(ra, rb, gaa, gab, gbb, &al, &bl, &gla, &glab, &glb);
            f = 0.80 * fs + 0.72 * fb + 0.19 * fv + 0.81 * fl;
            va = 0.80 * as + 0.72 * ab + 0.19 * av + 0.81 * al;
            vb = 0.80 * bs + 0.72 * bb + 0.19 * bv + 0.81 * bl;
            vgaa = 0.72 * gba + 0.81 * gla;
            vgab = 0.72 * 0.0 + 0.81 * glab;
            vgbb = 0.72 * gbb2 + 0.81 * glb;
            break;
        }
        case FN_PBE:
            pbe(ra, rb, gaa, gab, gbb, out);
            return 0;
        default:
            return -1;
    }
    out[0] = f, out[1] = va, out[2] = vb, out[3] = vgaa, out[4] = vgab, out[5] = vgbb;
    return 0;
}

int pdfxc_oracle_is_gga(int fn) { return fn == FN_HFB || fn == FN_BLYP || fn == FN_B3LYP || fn == FN_PBE; }

/* Single components, for the reference's per-class known-answer tests:
 * 0 Slater, 1 VWN5, 2 VWN3, 3 Becke88, 4 Becke88 except LDA, 5 LYP. */
int pdfxc_oracle_component(int comp, double ra, double rb, double gaa, double gab, double gbb,
                           double* out) {
    double f = 0, va = 0, vb = 0, vgaa = 0, vgab = 0, vgbb = 0;
    switch (comp) {
        case 0: slater(ra, rb, &f, &va, &vb); break;
        case 1: vwn(0, ra, rb, &f, &va, &vb); break;
        case 2: vwn(1, ra, rb, &f, &va, &vb); break;
        case 3: b88(1, ra, rb, gaa, gbb, &f, &va, &vb, &vgaa, &vgbb); break;
        case 4: b88(0, ra, rb, gaa, gbb, &f, &va, &vb, &vgaa, &vgbb); break;
        case 5:
            f = lyp_f(ra, rb, gaa, gab, gbb);
            lyp_v(ra, rb, gaa, gab, gbb, &va, &vb, &vgaa, &vgab, &vgbb);
            break;
        default: return -1;
    }
    out[0] = f, out[1] = va, out[2] = vb, out[3] = vgaa, out[4] = vgab, out[5] = vgbb;
    return 0;
}

/* ---------------- AO values: src/libpdf/DfCalcGridX.cpp:103-235, :667-769 ------
 * Shell table: per shell atom, L (0..2), first AO, nprim, first primitive.
 * Component order s; px py pz; dxy dxz dyz d(x2-y2) dz2. A primitive is skipped
 * when alpha*r^2 > 30 (TOOBIG, :42, :690). */
typedef struct {
    int nshell, nao;
    const int *sh_atom, *sh_l, *sh_ao0, *sh_nprim, *sh_p0;
    const double *p_exp, *p_coef, *atom_xyz;
} shells_t;

static void ang(int t, double x, double y, double z, double a2, double* v, double* dx, double* dy,
                double* dz) {
    const double s3 = 1.0 / sqrt(3.0);
    switch (t) {
        case 0: *v = 1; *dx = -a2 * x; *dy = -a2 * y; *dz = -a2 * z; break;
        case 1: *v = x; *dx = -a2 * x * x + 1.0; *dy = -a2 * x * y; *dz = -a2 * x * z; break;
        case 2: *v = y; *dx = -a2 * y * x; *dy = -a2 * y * y + 1.0; *dz = -a2 * y * z; break;
        case 3: *v = z; *dx = -a2 * z * x; *dy = -a2 * z * y; *dz = -a2 * z * z + 1.0; break;
        case 4: *v = x * y; *dx = -a2 * x * y * x + y; *dy = -a2 * x * y * y + x; *dz = -a2 * x * y * z; break;
        case 5: *v = z * x; *dx = -a2 * x * z * x + z; *dy = -a2 * x * z * y; *dz = -a2 * x * z * z + x; break;
        case 6: *v = y * z; *dx = -a2 * y * z * x; *dy = -a2 * y * z * y + z; *dz = -a2 * y * z * z + y; break;
        case 7: {
            *v = 0.5 * (x * x - y * y);
            const double xxX = -a2 * x * x * x + 2.0 * x, xxY = -a2 * x * x * y, xxZ = -a2 * x * x * z;
            const double yyX = -a2 * y * y * x, yyY = -a2 * y * y * y + 2.0 * y, yyZ = -a2 * y * y * z;
            *dx = 0.5 * (xxX - yyX); *dy = 0.5 * (xxY - yyY); *dz = 0.5 * (xxZ - yyZ);
            break;
        }
        default: {
            *v = s3 * (z * z - 0.5 * (x * x + y * y));
            const double xxX = -a2 * x * x * x + 2.0 * x, xxY = -a2 * x * x * y, xxZ = -a2 * x * x * z;
            const double yyX = -a2 * y * y * x, yyY = -a2 * y * y * y + 2.0 * y, yyZ = -a2 * y * y * z;
            const double zzX = -a2 * z * z * x, zzY = -a2 * z * z * y, zzZ = -a2 * z * z * z + 2.0 * z;
            *dx = s3 * (zzX - 0.5 * (xxX + yyX));
            *dy = s3 * (zzY - 0.5 * (xxY + yyY));
            *dz = s3 * (zzZ - 0.5 * (xxZ + yyZ));
        }
    }
}

static void eval_aos(const shells_t* S, const double* r, double* phi, double* gx, double* gy,
                     double* gz) {
    for (int s = 0; s < S->nshell; ++s) {
        const double* A = S->atom_xyz + 3 * S->sh_atom[s];
        const double x = r[0] - A[0], y = r[1] - A[1], z = r[2] - A[2];
        const double d2 = x * x + y * y + z * z;
        const int L = S->sh_l[s], n = 2 * L + 1;
        for (int c = 0; c < n; ++c) {
            const int t = L * L + c, mu = S->sh_ao0[s] + c;
            double v = 0, dx = 0, dy = 0, dz = 0;
            for (int k = 0; k < S->sh_nprim[s]; ++k) {
                const double a = S->p_exp[S->sh_p0[s] + k];
                if (a * d2 <= 30.0) {
                    const double g = S->p_coef[S->sh_p0[s] + k] * exp(-a * d2);
                    double pv, px, py, pz;
                    ang(t, x, y, z, 2.0 * a, &pv, &px, &py, &pz);
                    v += pv * g, dx += px * g, dy += py * g, dz += pz * g;
                }
            }
            phi[mu] = v;
            if (gx) gx[mu] = dx, gy[mu] = dy, gz[mu] = dz;
        }
    }
}

int pdfxc_oracle_aos(int nshell, int nao, const int* sh_atom, const int* sh_l, const int* sh_ao0,
                     const int* sh_nprim, const int* sh_p0, const double* p_exp, const double* p_coef,
                     const double* atom_xyz, long npts, const double* xyz, double* phi, double* dphi) {
    shells_t S = {nshell, nao, sh_atom, sh_l, sh_ao0, sh_nprim, sh_p0, p_exp, p_coef, atom_xyz};
#pragma omp parallel
    {
        double* g = (double*)malloc(sizeof(double) * 3 * (size_t)nao);
#pragma omp for schedule(static)
        for (long i = 0; i < npts; ++i) {
            eval_aos(&S, xyz + 3 * i, phi + (size_t)i * nao, g, g + nao, g + 2 * nao);
            if (dphi)
                for (int m = 0; m < nao; ++m)
                    for (int k = 0; k < 3; ++k) dphi[((size_t)i * nao + m) * 3 + k] = g[k * nao + m];
        }
        free(g);
    }
    return 0;
}

/* ---------------- the quadrature: src/libpdf/DfCalcGridX.cpp:865-931 (rho, grad rho),
 * :2056-2193 (Vxc pass, closed shell), :2351-2368 and :2455-2500 (Vxc element
 * formula), :2502-2537 (electron count).
 * rho_A = sum_ij PA_ij phi_i phi_j;  grad rho_A = 2 sum_ij PA_ij phi_i grad phi_j.
 * Points with rho_A <= rho_cut (1e-16) contribute nothing.
 * V_ij += w vrho phi_i phi_j + phi_i (c . grad phi_j) + phi_j (c . grad phi_i),
 *   c = w (2 vgAA + vgAB) grad rho_A (GGA).
 * Exc  += w f(rhoA, rhoA, gAA, gAA, gAA).
 * Outputs: exc, nelec_alpha = sum w rhoA, vxc (nao x nao, full), rho (npts x 1|4).
 * The per-point sums are accumulated in FP64 in point order within each
 * thread, then reduced across threads. ------------------------------------------- */
int pdfxc_oracle_xc(int fn, int nshell, int nao, const int* sh_atom, const int* sh_l,
                    const int* sh_ao0, const int* sh_nprim, const int* sh_p0, const double* p_exp,
                    const double* p_coef, const double* atom_xyz, long npts, const double* xyzw,
                    const double* PA, double rho_cut, double* exc, double* nelec, double* vxc,
                    double* rho_out, int nthreads) {
    shells_t S = {nshell, nao, sh_atom, sh_l, sh_ao0, sh_nprim, sh_p0, p_exp, p_coef, atom_xyz};
    const int gga = pdfxc_oracle_is_gga(fn);
    const size_t N = (size_t)nao;
    double E = 0.0, NE = 0.0;
    memset(vxc, 0, sizeof(double) * N * N);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel reduction(+ : E, NE)
    {
        double* phi = (double*)malloc(sizeof(double) * N * 5);
        double *gx = phi + N, *gy = phi + 2 * N, *gz = phi + 3 * N, *X = phi + 4 * N;
        double* V = (double*)calloc(N * N, sizeof(double));
#pragma omp for schedule(dynamic, 64)
        for (long i = 0; i < npts; ++i) {
            const double* r = xyzw + 4 * i;
            const double w = r[3];
            eval_aos(&S, r, phi, gga ? gx : NULL, gy, gz);
            for (size_t a = 0; a < N; ++a) {
                double s = 0.0;
                const double* Pa = PA + a * N;
                for (size_t b = 0; b < N; ++b) s += Pa[b] * phi[b];
                X[a] = s;
            }
            double rho = 0.0, grx = 0.0, gry = 0.0, grz = 0.0;
            for (size_t a = 0; a < N; ++a) rho += phi[a] * X[a];
            if (gga)
                for (size_t a = 0; a < N; ++a) grx += gx[a] * X[a], gry += gy[a] * X[a], grz += gz[a] * X[a];
            grx *= 2.0, gry *= 2.0, grz *= 2.0;
            if (rho_out) {
                double* ro = rho_out + (size_t)i * (gga ? 4 : 1);
                ro[0] = rho;
                if (gga) ro[1] = grx, ro[2] = gry, ro[3] = grz;
            }
            NE += w * rho;
            if (!(rho > rho_cut)) continue;
            const double gam = grx * grx + gry * gry + grz * grz;
            double o[6];
            pdfxc_oracle_functional(fn, rho, rho, gam, gam, gam, o);
            E += w * o[0];
            const double c1 = w * o[1];
            const double cc = w * (2.0 * o[3] + o[4]);
            const double cx = cc * grx, cy = cc * gry, cz = cc * grz;
            for (size_t a = 0; a < N; ++a) {
                const double ta = gga ? (cx * gx[a] + cy * gy[a] + cz * gz[a]) : 0.0;
                double* Va = V + a * N;
                for (size_t b = 0; b <= a; ++b) {
                    const double tb = gga ? (cx * gx[b] + cy * gy[b] + cz * gz[b]) : 0.0;
                    Va[b] += c1 * phi[a] * phi[b] + phi[a] * tb + phi[b] * ta;
                }
            }
        }
#pragma omp critical
        for (size_t a = 0; a < N; ++a)
            for (size_t b = 0; b <= a; ++b) vxc[a * N + b] += V[a * N + b];
        free(V);
        free(phi);
    }
    for (size_t a = 0; a < N; ++a)
        for (size_t b = 0; b < a; ++b) vxc[b * N + a] = vxc[a * N + b];
    *exc = E;
    *nelec = NE;
    return 0;
}

/* ---------------- Becke partition weights: src/libpdf/DfGenerateGrid.cpp:1811-1876,
 * :1958-1977, :2043-2086. For point r owned by atom A:
 *   P_m(r) = prod_{n != m} s(nu_mn),  s = (1 - f3(nu)) / 2,  f3 = f1(f1(f1(.))),
 *   f1(x) = x (3 - x^2) / 2,  mu_mn = (|r-R_m| - |r-R_n|) / |R_m - R_n|,
 *   nu_mn = mu_mn + a_mn (1 - mu_mn^2),  a = u/(u^2-1), u = (R_m-R_n)/(R_m+R_n),
 *   clamped to [-1/2, 1/2] (atomic size adjustment, radii brad),
 *   weight factor = P_A / sum_m P_m. --------------------------------------------- */
static double becke_f3(double x) {
    for (int k = 0; k < 3; ++k) x = 0.5 * x * (3.0 - x * x);
    return x;
}

int pdfxc_oracle_becke(int natom, const double* atom_xyz, const double* brad, int size_adjust,
                       long npts, const double* xyz, const int* owner, const int* ghost, double* factor) {
#pragma omp parallel
    {
        double* P = (double*)malloc(sizeof(double) * (size_t)natom);
        double* rr = (double*)malloc(sizeof(double) * (size_t)natom);
#pragma omp for schedule(static)
        for (long i = 0; i < npts; ++i) {
            const double* r = xyz + 3 * i;
            for (int m = 0; m < natom; ++m) {
                const double* A = atom_xyz + 3 * m;
                rr[m] = sqrt((r[0] - A[0]) * (r[0] - A[0]) + (r[1] - A[1]) * (r[1] - A[1]) +
                             (r[2] - A[2]) * (r[2] - A[2]));
            }
            double tot = 0.0;
            for (int m = 0; m < natom; ++m) {
                double p = 1.0;
                for (int n = 0; n < natom; ++n) {
                    /* partners with atomic number <= 0 (dummy atoms) are left out (:2056) */
                    if (n == m || (ghost && ghost[n])) continue;
                    const double* A = atom_xyz + 3 * m;
                    const double* B = atom_xyz + 3 * n;
                    const double Rmn = sqrt((A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) +
                                            (A[2] - B[2]) * (A[2] - B[2]));
                    double u = (rr[m] - rr[n]) * (1.0 / Rmn);
                    if (size_adjust) {
                        const double au = (brad[m] - brad[n]) / (brad[m] + brad[n]);
                        double a = au / (au * au - 1.0);
                        if (a < -0.5) a = -0.5;
                        else if (a > 0.5) a = 0.5;
                        u = u + a * (1.0 - u * u);
                    }
                    p *= 0.5 * (1.0 - becke_f3(u));
                }
                P[m] = p;
                tot += p;
            }
            factor[i] = P[owner[i]] / tot;
        }
        free(P);
        free(rr);
    }
    return 0;
}

/* ---------------- XC nuclear gradient, AO-centre term:
 * src/libpdf/DfCalcGridX.cpp:1073-1415 (energyGradient, energyGradient_part) with
 * the AO second derivatives of :237-385 and :792-863.
 * Per point g (owner atom A, weight w) with rho_A > rho_cut and per AO i on atom B:
 *   X_i = sum_j P_ij phi_j,  Y_ki = sum_j P_ij d_k phi_j,
 *   G_i = vrho grad phi_i X_i + sum_k c_k (grad d_k phi_i X_i + grad phi_i Y_ki)   (GGA terms)
 *   c = 2 vgAA grad rho_A + vgAB grad rho_A,
 *   grad[B] += -2 w G_i,  grad[A] -= -2 w G_i   (the grid moves with its atom),
 * and the result is doubled for the closed shell (:1090, :1237).
 * The AO second derivatives use d_k d_l (A e^{-a r^2}) =
 *   (A_kl - 2a (x_l A_k + x_k A_l) - 2a delta_kl A + 4a^2 x_k x_l A) e^{-a r^2}
 * for the angular polynomial A of each component, the same functions the
 * reference expands term by term. ---------------------------------------------- */
static void ang_poly(int t, double x, double y, double z, double* A, double* Ak, double* Akl) {
    /* A, dA/d(x,y,z), d2A/(xx, xy, xz, yy, yz, zz) */
    const double s3 = 1.0 / sqrt(3.0);
    for (int k = 0; k < 3; ++k) Ak[k] = 0.0;
    for (int k = 0; k < 6; ++k) Akl[k] = 0.0;
    switch (t) {
        case 0: *A = 1.0; break;
        case 1: *A = x; Ak[0] = 1.0; break;
        case 2: *A = y; Ak[1] = 1.0; break;
        case 3: *A = z; Ak[2] = 1.0; break;
        case 4: *A = x * y; Ak[0] = y; Ak[1] = x; Akl[1] = 1.0; break;
        case 5: *A = z * x; Ak[0] = z; Ak[2] = x; Akl[2] = 1.0; break;
        case 6: *A = y * z; Ak[1] = z; Ak[2] = y; Akl[4] = 1.0; break;
        case 7: *A = 0.5 * (x * x - y * y); Ak[0] = x; Ak[1] = -y; Akl[0] = 1.0; Akl[3] = -1.0; break;
        default:
            *A = s3 * (z * z - 0.5 * (x * x + y * y));
            Ak[0] = -s3 * x; Ak[1] = -s3 * y; Ak[2] = 2.0 * s3 * z;
            Akl[0] = -s3; Akl[3] = -s3; Akl[5] = 2.0 * s3;
    }
}

/* phi, d phi (3 x nao), d2 phi (6 x nao: xx xy xz yy yz zz) at one point */
static void eval_aos_d2(const shells_t* S, const double* r, double* phi, double* d1, double* d2) {
    const int N = S->nao;
    static const int KL[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
    for (int s = 0; s < S->nshell; ++s) {
        const double* C = S->atom_xyz + 3 * S->sh_atom[s];
        const double q[3] = {r[0] - C[0], r[1] - C[1], r[2] - C[2]};
        const double d2r = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
        const int L = S->sh_l[s], n = 2 * L + 1;
        for (int c = 0; c < n; ++c) {
            const int t = L * L + c, mu = S->sh_ao0[s] + c;
            double A, Ak[3], Akl[6];
            ang_poly(t, q[0], q[1], q[2], &A, Ak, Akl);
            double v = 0.0, g[3] = {0, 0, 0}, h[6] = {0, 0, 0, 0, 0, 0};
            for (int k = 0; k < S->sh_nprim[s]; ++k) {
                const double a = S->p_exp[S->sh_p0[s] + k];
                if (a * d2r > 30.0) continue;
                const double e = S->p_coef[S->sh_p0[s] + k] * exp(-a * d2r);
                const double a2 = 2.0 * a;
                v += A * e;
                for (int m = 0; m < 3; ++m) g[m] += (Ak[m] - a2 * q[m] * A) * e;
                for (int m = 0; m < 6; ++m) {
                    const int kk = KL[m][0], ll = KL[m][1];
                    double tv = Akl[m] - a2 * (q[ll] * Ak[kk] + q[kk] * Ak[ll]) + a2 * a2 * q[kk] * q[ll] * A;
                    if (kk == ll) tv -= a2 * A;
                    h[m] += tv * e;
                }
            }
            phi[mu] = v;
            for (int m = 0; m < 3; ++m) d1[m * N + mu] = g[m];
            for (int m = 0; m < 6; ++m) d2[m * N + mu] = h[m];
        }
    }
}

int pdfxc_oracle_aos_d2(int nshell, int nao, const int* sh_atom, const int* sh_l, const int* sh_ao0,
                        const int* sh_nprim, const int* sh_p0, const double* p_exp, const double* p_coef,
                        const double* atom_xyz, long npts, const double* xyz, double* out /* npts x 10 x nao */) {
    shells_t S = {nshell, nao, sh_atom, sh_l, sh_ao0, sh_nprim, sh_p0, p_exp, p_coef, atom_xyz};
#pragma omp parallel for schedule(static)
    for (long i = 0; i < npts; ++i) {
        double* o = out + (size_t)i * 10 * nao;
        eval_aos_d2(&S, xyz + 3 * i, o, o + nao, o + 4 * (size_t)nao);
    }
    return 0;
}

int pdfxc_oracle_xc_grad(int fn, int nshell, int nao, const int* sh_atom, const int* sh_l, const int* sh_ao0,
                         const int* sh_nprim, const int* sh_p0, const double* p_exp, const double* p_coef,
                         const double* atom_xyz, int natom, long npts, const double* xyzw, const int* owner,
                         const double* PA, double rho_cut, double* grad /* natom x 3 */, double* exc,
                         double* fdens /* npts, energy density f per point, or NULL */, int nthreads) {
    shells_t S = {nshell, nao, sh_atom, sh_l, sh_ao0, sh_nprim, sh_p0, p_exp, p_coef, atom_xyz};
    const int gga = pdfxc_oracle_is_gga(fn);
    const size_t N = (size_t)nao;
    int* ao_atom = (int*)malloc(sizeof(int) * N);
    for (int s = 0; s < nshell; ++s)
        for (int c = 0; c < 2 * sh_l[s] + 1; ++c) ao_atom[sh_ao0[s] + c] = sh_atom[s];
    memset(grad, 0, sizeof(double) * 3 * (size_t)natom);
    double E = 0.0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel reduction(+ : E)
    {
        double* phi = (double*)malloc(sizeof(double) * N * 14);
        double *d1 = phi + N, *d2 = phi + 4 * N, *X = phi + 10 * N; /* X, Yx, Yy, Yz */
        double* G = (double*)calloc(3 * (size_t)natom, sizeof(double));
#pragma omp for schedule(dynamic, 64)
        for (long i = 0; i < npts; ++i) {
            const double* r = xyzw + 4 * i;
            const double w = r[3];
            if (fdens) fdens[i] = 0.0;
            eval_aos_d2(&S, r, phi, d1, d2);
            for (size_t a = 0; a < N; ++a) {
                const double* Pa = PA + a * N;
                double s0 = 0, sx = 0, sy = 0, sz = 0;
                for (size_t b = 0; b < N; ++b) {
                    s0 += Pa[b] * phi[b];
                    sx += Pa[b] * d1[b], sy += Pa[b] * d1[N + b], sz += Pa[b] * d1[2 * N + b];
                }
                X[a] = s0, X[N + a] = sx, X[2 * N + a] = sy, X[3 * N + a] = sz;
            }
            double rho = 0.0, gr[3] = {0, 0, 0};
            for (size_t a = 0; a < N; ++a) {
                rho += phi[a] * X[a];
                for (int k = 0; k < 3; ++k) gr[k] += d1[k * N + a] * X[a];
            }
            for (int k = 0; k < 3; ++k) gr[k] *= 2.0;
            if (!(rho > rho_cut)) continue;
            const double gam = gga ? gr[0] * gr[0] + gr[1] * gr[1] + gr[2] * gr[2] : 0.0;
            double o[6];
            pdfxc_oracle_functional(fn, rho, rho, gam, gam, gam, o);
            E += w * o[0];
            if (fdens) fdens[i] = o[0];
            double c[3] = {0, 0, 0};
            if (gga)
                for (int k = 0; k < 3; ++k) c[k] = (2.0 * o[3] + o[4]) * gr[k];
            /* d2 index of (m, k): xx xy xz / xy yy yz / xz yz zz */
            static const int H[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
            const int A = owner[i];
            for (size_t a = 0; a < N; ++a) {
                double gv[3];
                for (int m = 0; m < 3; ++m) {
                    double t = o[1] * d1[m * N + a] * X[a];
                    if (gga)
                        for (int k = 0; k < 3; ++k)
                            t += c[k] * (d2[H[m][k] * N + a] * X[a] + d1[m * N + a] * X[(1 + k) * N + a]);
                    gv[m] = -2.0 * w * t;
                }
                const int B = ao_atom[a];
                for (int m = 0; m < 3; ++m) G[3 * B + m] += gv[m], G[3 * A + m] -= gv[m];
            }
        }
#pragma omp critical
        for (int k = 0; k < 3 * natom; ++k) grad[k] += 2.0 * G[k]; /* closed shell */
        free(G);
        free(phi);
    }
    free(ao_atom);
    *exc = E;
    return 0;
}

/* ---------------- XC nuclear gradient, grid-weight term: the derivative of the
 * Becke partition of pdfxc_oracle_becke with respect to the nuclei (Johnson, Gill
 * and Pople, J. Chem. Phys. 98, 5612 (1993), appendix B), written here from the
 * partition function itself. For point r owned by atom A with coefficient
 * c = w_single f(r):
 *   omega_A = P_A / Z,  Z = sum_i P_i,  P_i = prod_{j != i} s(nu_ij),
 *   grad_B omega_A = (grad_B P_A - omega_A grad_B Z) / Z        (B != A, point fixed),
 *   grad_B P_i   = prod_{j != i, B} s_ij  s'(nu_iB) grad_B nu_iB         (i != B),
 *   grad_B P_B   = sum_{j != B} prod_{k != B, j} s_Bk  s'(nu_Bj) grad_B nu_Bj,
 *   grad_B mu_iB = -(u_B + mu_iB e_iB) / R_iB,  grad_B mu_Bj = (u_B - mu_Bj e_jB) / R_Bj,
 *   u_B = (R_B - r)/|R_B - r|,  e_iB = (R_B - R_i)/R_iB,  d nu / d mu = 1 - 2 a mu,
 *   s'(nu) = -(27/16) (1 - p2^2)(1 - p1^2)(1 - nu^2),  p1 = f1(nu), p2 = f1(p1);
 *   grad[B] += c grad_B omega_A,  grad[A] -= c grad_B omega_A (the point moves with A).
 * The reference's own weight term (JGP_nablaB_omegaA, src/libpdf/DfGenerateGrid.cpp:
 * 2259-2393) evaluates to zero: its JGP_t returns 0 unless |mu| > 1. ----------- */
int pdfxc_oracle_becke_grad(int natom, const double* atom_xyz, const double* brad, int size_adjust, long npts,
                            const double* xyz, const int* owner, const double* coef, double* grad) {
    const int n = natom;
    memset(grad, 0, sizeof(double) * 3 * (size_t)n);
#pragma omp parallel
    {
        double* rr = (double*)malloc(sizeof(double) * n);
        double* s = (double*)malloc(sizeof(double) * (size_t)n * n);
        double* ds = (double*)malloc(sizeof(double) * (size_t)n * n); /* d s / d mu, size adjustment folded in */
        double* mu = (double*)malloc(sizeof(double) * (size_t)n * n);
        double* P = (double*)malloc(sizeof(double) * n);
        double* pre = (double*)malloc(sizeof(double) * (n + 1));
        double* G = (double*)calloc(3 * (size_t)n, sizeof(double));
#pragma omp for schedule(dynamic, 16)
        for (long g = 0; g < npts; ++g) {
            const double c = coef[g];
            if (c == 0.0) continue;
            const double* r = xyz + 3 * g;
            const int A = owner[g];
            for (int m = 0; m < n; ++m) {
                const double* R = atom_xyz + 3 * m;
                rr[m] = sqrt((r[0] - R[0]) * (r[0] - R[0]) + (r[1] - R[1]) * (r[1] - R[1]) + (r[2] - R[2]) * (r[2] - R[2]));
            }
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j) {
                    if (i == j) { s[i * n + j] = 1.0; ds[i * n + j] = 0.0; mu[i * n + j] = 0.0; continue; }
                    const double* Ri = atom_xyz + 3 * i;
                    const double* Rj = atom_xyz + 3 * j;
                    const double Rij = sqrt((Ri[0] - Rj[0]) * (Ri[0] - Rj[0]) + (Ri[1] - Rj[1]) * (Ri[1] - Rj[1]) +
                                            (Ri[2] - Rj[2]) * (Ri[2] - Rj[2]));
                    const double m_ = (rr[i] - rr[j]) * (1.0 / Rij);
                    double nu = m_, dnu = 1.0;
                    if (size_adjust) {
                        const double au = (brad[i] - brad[j]) / (brad[i] + brad[j]);
                        double a = au / (au * au - 1.0);
                        if (a < -0.5) a = -0.5;
                        else if (a > 0.5) a = 0.5;
                        nu = m_ + a * (1.0 - m_ * m_);
                        dnu = 1.0 - 2.0 * a * m_;
                    }
                    const double p1 = 0.5 * nu * (3.0 - nu * nu), p2 = 0.5 * p1 * (3.0 - p1 * p1);
                    s[i * n + j] = 0.5 * (1.0 - becke_f3(nu));
                    ds[i * n + j] = -(27.0 / 16.0) * (1.0 - p2 * p2) * (1.0 - p1 * p1) * (1.0 - nu * nu) * dnu;
                    mu[i * n + j] = m_;
                }
            double Z = 0.0;
            for (int i = 0; i < n; ++i) {
                double p = 1.0;
                for (int j = 0; j < n; ++j) p *= s[i * n + j];
                P[i] = p;
                Z += p;
            }
            const double omega = P[A] / Z;
            for (int B = 0; B < n; ++B) {
                if (B == A) continue;
                const double* RB = atom_xyz + 3 * B;
                double uB[3];
                for (int k = 0; k < 3; ++k) uB[k] = (RB[k] - r[k]) / rr[B];
                double dZ[3] = {0, 0, 0}, dPA[3] = {0, 0, 0};
                /* i != B: one factor s_iB differentiated */
                for (int i = 0; i < n; ++i) {
                    if (i == B) continue;
                    double others = 1.0;
                    for (int j = 0; j < n; ++j)
                        if (j != B) others *= s[i * n + j];
                    const double* Ri = atom_xyz + 3 * i;
                    double e[3], RiB = 0.0;
                    for (int k = 0; k < 3; ++k) e[k] = RB[k] - Ri[k], RiB += e[k] * e[k];
                    RiB = sqrt(RiB);
                    const double f = others * ds[i * n + B];
                    for (int k = 0; k < 3; ++k) {
                        const double gmu = -(uB[k] + mu[i * n + B] * e[k] / RiB) / RiB;
                        dZ[k] += f * gmu;
                        if (i == A) dPA[k] += f * gmu;
                    }
                }
                /* i == B: every factor s_Bj in turn, prefix/suffix products of the rest */
                pre[0] = 1.0;
                for (int j = 0; j < n; ++j) pre[j + 1] = pre[j] * s[B * n + j];
                double suf = 1.0;
                for (int j = n - 1; j >= 0; --j) {
                    if (j != B) {
                        const double* Rj = atom_xyz + 3 * j;
                        double e[3], RBj = 0.0;
                        for (int k = 0; k < 3; ++k) e[k] = RB[k] - Rj[k], RBj += e[k] * e[k];
                        RBj = sqrt(RBj);
                        const double f = pre[j] * suf * ds[B * n + j];
                        for (int k = 0; k < 3; ++k) dZ[k] += f * (uB[k] - mu[B * n + j] * e[k] / RBj) / RBj;
                    }
                    suf *= s[B * n + j];
                }
                for (int k = 0; k < 3; ++k) {
                    const double d = c * (dPA[k] - omega * dZ[k]) / Z;
                    G[3 * B + k] += d;
                    G[3 * A + k] -= d;
                }
            }
        }
#pragma omp critical
        for (int k = 0; k < 3 * n; ++k) grad[k] += G[k];
        free(rr), free(s), free(ds), free(mu), free(P), free(pre), free(G);
    }
    return 0;
}

/* ---------------- open shell: src/libpdf/DfCalcGridX.cpp:2292-2303, :2317-2328
 * (calcXCIntegForFockAndEnergy(P_A, P_B, ...)), :1891-1922 and :1963-2016 (rho of
 * both spins), :2093-2135 and :2195-2278 (buildVxc with F_A, F_B).
 * A point contributes when rho_A > rho_cut or rho_B > rho_cut. For spin s,
 * build_XC_Matrix (:2455-2500) is given vrho_s, vgamma_ss, vgamma_AB and the
 * spin's own gradient, so c_s = w (2 vgamma_ss + vgamma_AB) grad rho_s.
 * Outputs: exc, nelec_a/b = sum w rho_s, vxc_a/b (nao x nao, full),
 * rho (npts x 2 LDA: rhoA rhoB; npts x 8 GGA: rhoA, grad A, rhoB, grad B). */
int pdfxc_oracle_xc_uks(int fn, int nshell, int nao, const int* sh_atom, const int* sh_l, const int* sh_ao0,
                        const int* sh_nprim, const int* sh_p0, const double* p_exp, const double* p_coef,
                        const double* atom_xyz, long npts, const double* xyzw, const double* PA, const double* PB,
                        double rho_cut, double* exc, double* nelec_a, double* nelec_b, double* vxc_a, double* vxc_b,
                        double* rho_out, int nthreads) {
    shells_t S = {nshell, nao, sh_atom, sh_l, sh_ao0, sh_nprim, sh_p0, p_exp, p_coef, atom_xyz};
    const int gga = pdfxc_oracle_is_gga(fn);
    const size_t N = (size_t)nao;
    double E = 0.0, NA = 0.0, NB = 0.0;
    memset(vxc_a, 0, sizeof(double) * N * N);
    memset(vxc_b, 0, sizeof(double) * N * N);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
#pragma omp parallel reduction(+ : E, NA, NB)
    {
        double* phi = (double*)malloc(sizeof(double) * N * 6);
        double *gx = phi + N, *gy = phi + 2 * N, *gz = phi + 3 * N, *XA = phi + 4 * N, *XB = phi + 5 * N;
        double* Va = (double*)calloc(N * N, sizeof(double));
        double* Vb = (double*)calloc(N * N, sizeof(double));
#pragma omp for schedule(dynamic, 64)
        for (long i = 0; i < npts; ++i) {
            const double* r = xyzw + 4 * i;
            const double w = r[3];
            eval_aos(&S, r, phi, gga ? gx : NULL, gy, gz);
            for (size_t a = 0; a < N; ++a) {
                double sa = 0.0, sb = 0.0;
                for (size_t b = 0; b < N; ++b) sa += PA[a * N + b] * phi[b], sb += PB[a * N + b] * phi[b];
                XA[a] = sa, XB[a] = sb;
            }
            double ra = 0.0, rb = 0.0, ga[3] = {0, 0, 0}, gb[3] = {0, 0, 0};
            for (size_t a = 0; a < N; ++a) {
                ra += phi[a] * XA[a], rb += phi[a] * XB[a];
                if (gga) {
                    ga[0] += gx[a] * XA[a], ga[1] += gy[a] * XA[a], ga[2] += gz[a] * XA[a];
                    gb[0] += gx[a] * XB[a], gb[1] += gy[a] * XB[a], gb[2] += gz[a] * XB[a];
                }
            }
            for (int k = 0; k < 3; ++k) ga[k] *= 2.0, gb[k] *= 2.0;
            if (rho_out) {
                double* ro = rho_out + (size_t)i * (gga ? 8 : 2);
                if (gga) {
                    ro[0] = ra, ro[1] = ga[0], ro[2] = ga[1], ro[3] = ga[2];
                    ro[4] = rb, ro[5] = gb[0], ro[6] = gb[1], ro[7] = gb[2];
                } else {
                    ro[0] = ra, ro[1] = rb;
                }
            }
            NA += w * ra, NB += w * rb;
            if (!(ra > rho_cut || rb > rho_cut)) continue;
            const double gaa = ga[0] * ga[0] + ga[1] * ga[1] + ga[2] * ga[2];
            const double gbb = gb[0] * gb[0] + gb[1] * gb[1] + gb[2] * gb[2];
            const double gab = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
            double o[6];
            pdfxc_oracle_functional(fn, ra, rb, gaa, gab, gbb, o);
            E += w * o[0];
            for (int spin = 0; spin < 2; ++spin) {
                const double c1 = w * (spin ? o[2] : o[1]);
                const double cc = w * (2.0 * (spin ? o[5] : o[3]) + o[4]);
                const double* g = spin ? gb : ga;
                const double cx = cc * g[0], cy = cc * g[1], cz = cc * g[2];
                double* V = spin ? Vb : Va;
                for (size_t a = 0; a < N; ++a) {
                    const double ta = gga ? (cx * gx[a] + cy * gy[a] + cz * gz[a]) : 0.0;
                    for (size_t b = 0; b <= a; ++b) {
                        const double tb = gga ? (cx * gx[b] + cy * gy[b] + cz * gz[b]) : 0.0;
                        V[a * N + b] += c1 * phi[a] * phi[b] + phi[a] * tb + phi[b] * ta;
                    }
                }
            }
        }
#pragma omp critical
        for (size_t a = 0; a < N; ++a)
            for (size_t b = 0; b <= a; ++b) vxc_a[a * N + b] += Va[a * N + b], vxc_b[a * N + b] += Vb[a * N + b];
        free(Va), free(Vb), free(phi);
    }
    for (size_t a = 0; a < N; ++a)
        for (size_t b = 0; b < a; ++b) vxc_a[b * N + a] = vxc_a[a * N + b], vxc_b[b * N + a] = vxc_b[a * N + b];
    *exc = E;
    *nelec_a = NA;
    *nelec_b = NB;
    return 0;
}

/* ---------------- SS partition weights: src/libpdf/DfGenerateGrid.cpp:1878-1956
 * (calcMultiCenterWeight_SS). For point r owned by atom A:
 *   P_m(r) = prod_{n != m} s(mu_mn),  mu_mn = (|r-R_m| - |r-R_n|) / |R_m - R_n| (no size adjustment),
 *   s = (1 - g)/2,  g = -1 (mu < -a), 1 (mu > a), else (35 z - 35 z^3 + 21 z^5 - 5 z^7)/16, z = mu/a,
 *   a = 0.64;  factor = P_A / sum_m P_m. */
int pdfxc_oracle_ss(int natom, const double* atom_xyz, long npts, const double* xyz, const int* owner,
                    double* factor) {
#pragma omp parallel
    {
        double* rr = (double*)malloc(sizeof(double) * (size_t)natom);
#pragma omp for schedule(static)
        for (long i = 0; i < npts; ++i) {
            const double* r = xyz + 3 * i;
            for (int m = 0; m < natom; ++m) {
                const double* A = atom_xyz + 3 * m;
                rr[m] = sqrt((r[0] - A[0]) * (r[0] - A[0]) + (r[1] - A[1]) * (r[1] - A[1]) +
                             (r[2] - A[2]) * (r[2] - A[2]));
            }
            double tot = 0.0, pown = 0.0;
            for (int m = 0; m < natom; ++m) {
                double p = 1.0;
                for (int n = 0; n < natom; ++n) {
                    if (n == m) continue;
                    const double* A = atom_xyz + 3 * m;
                    const double* B = atom_xyz + 3 * n;
                    const double Rmn = sqrt((A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) +
                                            (A[2] - B[2]) * (A[2] - B[2]));
                    const double u = (rr[m] - rr[n]) * (1.0 / Rmn);
                    const double a = 0.64;
                    double g;
                    if (u < -a) g = -1.0;
                    else if (u > a) g = 1.0;
                    else {
                        const double z = u / a, z2 = z * z, z3 = z2 * z, z5 = z2 * z3;
                        g = (1.0 / 16.0) * (35.0 * z - 35.0 * z3 + 21.0 * z5 - 5.0 * z5 * z2);
                    }
                    p *= 0.5 * (1.0 - g);
                }
                tot += p;
                if (m == owner[i]) pown = p;
            }
            factor[i] = pown / tot;
        }
        free(rr);
    }
    return 0;
}
