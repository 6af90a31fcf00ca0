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
    for (int k = 0; k < np; ++k) {
        const double al = bas.p_exp[p0 + k];
        if (al * d2 <= 30.0) {
            const double e = bas.p_coef[p0 + k] * exp(-al * d2);
            S0 += e;
            if (GGA) S1 += al * e;
        }
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

}  // namespace pdfxc
