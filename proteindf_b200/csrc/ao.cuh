// AO values of the XC build, shared by the FP64 and the INT8 paths: a shell's radial
// sums at a point and the angular polynomial of each component. A component's value
// and gradient are phi = A S0 and grad phi = grad A S0 - 2 r A S1 with
// S0 = sum_k c_k e^{-a_k r^2}, S1 = sum_k c_k a_k e^{-a_k r^2} (primitives with
// a r^2 > 30 skipped, DfCalcGridX.cpp:42, :690): the reference's per-primitive
// prefactors (getPrefactor / getPrefactorForDerivative, DfCalcGridX.cpp:103-235)
// summed in another order.
#pragma once

#include "pdfxc_internal.cuh"

namespace pdfxc {

// Angular polynomial A of component t = L^2 + c (the reference's prefactors,
// DfCalcGridX.cpp:103-141) and its gradient.
__device__ __forceinline__ void ang_poly1(int t, double x, double y, double z, double& A, double& Ax, double& Ay,
                                          double& Az) {
    const double s3 = 0.57735026918962576451;  // 1/sqrt(3)
    switch (t) {
        case 0: A = 1.0; Ax = Ay = Az = 0.0; break;
        case 1: A = x; Ax = 1.0; Ay = Az = 0.0; break;
        case 2: A = y; Ay = 1.0; Ax = Az = 0.0; break;
        case 3: A = z; Az = 1.0; Ax = Ay = 0.0; break;
        case 4: A = x * y; Ax = y; Ay = x; Az = 0.0; break;
        case 5: A = z * x; Ax = z; Az = x; Ay = 0.0; break;
        case 6: A = y * z; Ay = z; Az = y; Ax = 0.0; break;
        case 7: A = 0.5 * (x * x - y * y); Ax = x; Ay = -y; Az = 0.0; break;
        default: A = s3 * (z * z - 0.5 * (x * x + y * y)); Ax = -s3 * x; Ay = -s3 * y; Az = 2.0 * s3 * z;
    }
}

// Radial sums S0 and (GGA) S1 of shell s at squared distance d2 from its atom.
template <bool GGA>
__device__ __forceinline__ void shell_radial(const BasisView& bas, int s, double d2, double& S0, double& S1) {
    const int np = bas.sh_nprim[s], p0 = bas.sh_p0[s];
    S0 = 0.0, S1 = 0.0;
    for (int k = 0; k < np; ++k) {  // exponents ascend within a shell: the rest are cut too
        const double al = bas.p_exp[p0 + k];
        if (al * d2 > 30.0) break;
        const double e = bas.p_coef[p0 + k] * exp(-al * d2);
        S0 += e;
        if (GGA) S1 += al * e;
    }
}

// A shell as the AO kernels read it from shared memory (every thread of a CTA walks the same
// shells, so broadcasts replace chains of dependent global loads): its atom, L and primitives.
constexpr int kStagedPrims = 10;
struct ShellRec {
    double ax, ay, az;
    int lq, np;  // np < 0: more than kStagedPrims primitives, read from the global tables
    int sh, row0;
    double alpha[kStagedPrims], coef[kStagedPrims];
};

__device__ __forceinline__ void stage_shell(const BasisView& bas, int sh, int row0, ShellRec& r) {
    const int a = bas.sh_atom[sh], np = bas.sh_nprim[sh], p0 = bas.sh_p0[sh];
    r.ax = bas.atom_xyz[3 * a], r.ay = bas.atom_xyz[3 * a + 1], r.az = bas.atom_xyz[3 * a + 2];
    r.lq = bas.sh_l[sh], r.sh = sh, r.row0 = row0;
    r.np = np <= kStagedPrims ? np : -1;
    if (np <= kStagedPrims)
        for (int k = 0; k < np; ++k) r.alpha[k] = bas.p_exp[p0 + k], r.coef[k] = bas.p_coef[p0 + k];
}

// shell_radial on a staged shell (the same operations in the same order)
template <bool GGA>
__device__ __forceinline__ void shell_radial_staged(const BasisView& bas, const ShellRec& r, double d2, double& S0,
                                                    double& S1) {
    if (r.np < 0) {
        shell_radial<GGA>(bas, r.sh, d2, S0, S1);
        return;
    }
    S0 = 0.0, S1 = 0.0;
    for (int k = 0; k < r.np; ++k) {  // exponents ascend within a shell: the rest are cut too
        const double al = r.alpha[k];
        if (al * d2 > 30.0) break;
        const double e = r.coef[k] * exp(-al * d2);
        S0 += e;
        if (GGA) S1 += al * e;
    }
}

// Value and (GGA) gradient of component t at displacement (x, y, z) from the shell's atom.
template <bool GGA>
__device__ __forceinline__ void ao_from_radial(int t, double x, double y, double z, double S0, double S1, double& v,
                                               double& gx, double& gy, double& gz) {
    double A, Ax, Ay, Az;
    ang_poly1(t, x, y, z, A, Ax, Ay, Az);
    v = A * S0;
    if (GGA) {
        const double u = 2.0 * A * S1;
        gx = Ax * S0 - x * u;
        gy = Ay * S0 - y * u;
        gz = Az * S0 - z * u;
    }
}

// All components of a shell of angular momentum L at once (L = 0, 1, 2; the component order
// and prefactors of ang_poly1): v[c] = A_c S0 and g[c] = grad A_c S0 - 2 r A_c S1, c < 2L + 1.
// One branch per shell instead of one per component.
__device__ __forceinline__ void shell_components(int L, double x, double y, double z, double S0, double S1,
                                                 double v[5], double gx[5], double gy[5], double gz[5]) {
    const double u = 2.0 * S1;
    if (L == 0) {
        v[0] = S0;
        gx[0] = -x * u, gy[0] = -y * u, gz[0] = -z * u;
        return;
    }
    if (L == 1) {
        const double r[3] = {x, y, z};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double t = r[c] * u;
            v[c] = r[c] * S0;
            gx[c] = (c == 0 ? S0 : 0.0) - x * t;
            gy[c] = (c == 1 ? S0 : 0.0) - y * t;
            gz[c] = (c == 2 ? S0 : 0.0) - z * t;
        }
        return;
    }
    const double s3 = 0.57735026918962576451;  // 1/sqrt(3)
    const double A[5] = {x * y, z * x, y * z, 0.5 * (x * x - y * y), s3 * (z * z - 0.5 * (x * x + y * y))};
    const double Ax[5] = {y, z, 0.0, x, -s3 * x};
    const double Ay[5] = {x, 0.0, z, -y, -s3 * y};
    const double Az[5] = {0.0, x, y, 0.0, 2.0 * s3 * z};
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        const double t = A[c] * u;
        v[c] = A[c] * S0;
        gx[c] = Ax[c] * S0 - x * t;
        gy[c] = Ay[c] * S0 - y * t;
        gz[c] = Az[c] * S0 - z * t;
    }
}

// The Vxc operand Z = a phi + c . grad phi of every component of a shell (a = 0.5 w v_rho, c the
// gradient coefficients; zero c for an LDA). With phi = A S0 and grad phi = grad A S0 - 2 r A S1,
// Z = A alpha + S0 (c . grad A) with alpha = a S0 - 2 S1 (c . r) once per shell and point.
__device__ __forceinline__ void shell_z(int L, double x, double y, double z, double S0, double S1, double a,
                                        double cx, double cy, double cz, double zc[5]) {
    const double alpha = a * S0 - 2.0 * S1 * (cx * x + cy * y + cz * z);
    if (L == 0) {
        zc[0] = alpha;
    } else if (L == 1) {
        zc[0] = x * alpha + S0 * cx;
        zc[1] = y * alpha + S0 * cy;
        zc[2] = z * alpha + S0 * cz;
    } else {
        const double s3 = 0.57735026918962576451;  // 1/sqrt(3)
        zc[0] = x * y * alpha + S0 * (cx * y + cy * x);
        zc[1] = z * x * alpha + S0 * (cx * z + cz * x);
        zc[2] = y * z * alpha + S0 * (cy * z + cz * y);
        zc[3] = 0.5 * (x * x - y * y) * alpha + S0 * (cx * x - cy * y);
        zc[4] = s3 * (z * z - 0.5 * (x * x + y * y)) * alpha + S0 * s3 * (2.0 * cz * z - cx * x - cy * y);
    }
}

// rho and grad rho contributions of a shell's components with coefficients X[c] (c < 2L + 1; zero
// for a component that is not added): with phi = A S0 and grad phi = grad A S0 - 2 r A S1,
// sum_c X_c phi_c = S0 PA and sum_c X_c grad phi_c = S0 PG - 2 r S1 PA, with PA = sum_c X_c A_c and
// PG = sum_c X_c grad A_c, so a component costs a few FMAs.
template <bool GGA>
__device__ __forceinline__ void shell_rho(int L, double x, double y, double z, double S0, double S1, const double X[5],
                                          double& r, double& gx, double& gy, double& gz) {
    double PA, Px = 0.0, Py = 0.0, Pz = 0.0;
    if (L == 0) {
        PA = X[0];
    } else if (L == 1) {
        PA = x * X[0] + y * X[1] + z * X[2];
        Px = X[0], Py = X[1], Pz = X[2];
    } else {
        const double s3 = 0.57735026918962576451;  // 1/sqrt(3)
        PA = X[0] * (x * y) + X[1] * (z * x) + X[2] * (y * z) + X[3] * (0.5 * (x * x - y * y)) +
             X[4] * (s3 * (z * z - 0.5 * (x * x + y * y)));
        if (GGA) {
            Px = X[0] * y + X[1] * z + (X[3] - s3 * X[4]) * x;
            Py = X[0] * x + X[2] * z - (X[3] + s3 * X[4]) * y;
            Pz = X[1] * x + X[2] * y + 2.0 * s3 * X[4] * z;
        }
    }
    r = fma(S0, PA, r);
    if (GGA) {
        const double w = 2.0 * S1 * PA;
        gx += S0 * Px - x * w;
        gy += S0 * Py - y * w;
        gz += S0 * Pz - z * w;
    }
}

}  // namespace pdfxc
