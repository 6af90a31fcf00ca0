// Atom-centred grid points on the device (DfGenerateGrid::getSphericalGrids,
// src/libpdf/DfGenerateGrid.cpp:1715-1734): the unit grid of a shell's angular order is
// rotated by O, scaled by the shell's abscissa and moved to the atom; the weight is the
// unit weight times the radial weight. The operations follow the reference's order
// (O u, then * r, then + centre) without fused multiply-adds, so the points are those
// of a host generator that forms them the same way.
#include <cuda_runtime.h>

#include "pdfxc_internal.cuh"

namespace pdfxc {

namespace {

__global__ void __launch_bounds__(128) k_grid_points(const GridShell* __restrict__ shells,
                                                     const double* __restrict__ unit, const double* __restrict__ O,
                                                     const double* __restrict__ atom_xyz, double* __restrict__ xyz,
                                                     double* __restrict__ w, int* __restrict__ owner) {
    const GridShell s = shells[blockIdx.x];
    const double ax = atom_xyz[3 * s.atom], ay = atom_xyz[3 * s.atom + 1], az = atom_xyz[3 * s.atom + 2];
    double o[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) o[k] = O[k];
    for (int k = threadIdx.x; k < s.n; k += blockDim.x) {
        const double* u = unit + 4 * (s.u0 + k);
        const double ux = __dadd_rn(__dadd_rn(__dmul_rn(o[0], u[0]), __dmul_rn(o[1], u[1])), __dmul_rn(o[2], u[2]));
        const double uy = __dadd_rn(__dadd_rn(__dmul_rn(o[3], u[0]), __dmul_rn(o[4], u[1])), __dmul_rn(o[5], u[2]));
        const double uz = __dadd_rn(__dadd_rn(__dmul_rn(o[6], u[0]), __dmul_rn(o[7], u[1])), __dmul_rn(o[8], u[2]));
        const int64_t i = s.p0 + k;
        xyz[3 * i] = __dadd_rn(__dmul_rn(ux, s.r), ax);
        xyz[3 * i + 1] = __dadd_rn(__dmul_rn(uy, s.r), ay);
        xyz[3 * i + 2] = __dadd_rn(__dmul_rn(uz, s.r), az);
        w[i] = __dmul_rn(u[3], s.wr);
        owner[i] = s.atom;
    }
}

}  // namespace

void launch_grid_points(const GridShell* shells, int nshell, const double* unit, const double* O,
                        const double* atom_xyz, double* xyz, double* w, int* owner, cudaStream_t s) {
    if (nshell > 0) k_grid_points<<<nshell, 128, 0, s>>>(shells, unit, O, atom_xyz, xyz, w, owner);
}

}  // namespace pdfxc
