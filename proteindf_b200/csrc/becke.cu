// Becke partition weights on the device (K7).
//
// For point r owned by atom A (DfGenerateGrid::calcMultiCenterWeight_Becke,
// src/libpdf/DfGenerateGrid.cpp:1811-1876, Ps_uij :2043-2086):
//   P_m(r) = prod_{n != m} s(nu_mn),  s(nu) = (1 - f(f(f(nu)))) / 2,  f(x) = x (3 - x^2) / 2
//   mu_mn  = (|r - R_m| - |r - R_n|) / |R_m - R_n|
//   nu_mn  = mu_mn + a_mn (1 - mu_mn^2), a = u / (u^2 - 1), u = (R_m - R_n)/(R_m + R_n),
//            a clamped to [-1/2, 1/2] (atomic size adjustment, Becke radii)
//   w(r)   = w_single(r) * P_A(r) / sum_m P_m(r).
// Partner atoms n with atomic number <= 0 (dummy atoms, `ghost`) are left out of
// every product, as Ps_uij does (:2056); a dummy atom m still has its own P_m.
// One thread per point; the atoms (coordinates and radius) are staged in
// shared memory once per CTA. All arithmetic is FP64, and this file is compiled
// without fused multiply-adds, so that every operation rounds once in the order
// written: the weights then equal the CPU restatement's (plain IEEE operations in
// the same order) bit for bit, and the weight screen keeps the same points.
#include <cuda_runtime.h>

#include <algorithm>

#include "pdfxc_internal.cuh"

namespace pdfxc {

namespace {

__device__ __forceinline__ double becke_s(double nu) {
#pragma unroll
    for (int k = 0; k < 3; ++k) nu = 0.5 * nu * (3.0 - nu * nu);
    return 0.5 * (1.0 - nu);
}

__global__ void __launch_bounds__(128) k_becke(const double* __restrict__ atom_xyz, const double* __restrict__ brad,
                                               const int* __restrict__ ghost, int natom, int size_adjust,
                                               int64_t npts, const double* __restrict__ xyz,
                                               const int* __restrict__ owner, const double* __restrict__ w_single,
                                               double* __restrict__ w_out) {
    extern __shared__ double4 atoms[];  // x, y, z, radius (negative: a dummy partner, left out)
    for (int a = threadIdx.x; a < natom; a += blockDim.x)
        atoms[a] = make_double4(atom_xyz[3 * a], atom_xyz[3 * a + 1], atom_xyz[3 * a + 2],
                                ghost && ghost[a] ? -1.0 : brad[a]);
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npts; i += (int64_t)gridDim.x * blockDim.x) {
        const double rx = xyz[3 * i], ry = xyz[3 * i + 1], rz = xyz[3 * i + 2];
        const int own = owner[i];
        double tot = 0.0, pown = 0.0;
        for (int m = 0; m < natom; ++m) {
            const double4 A = atoms[m];
            const double rm = sqrt((rx - A.x) * (rx - A.x) + (ry - A.y) * (ry - A.y) + (rz - A.z) * (rz - A.z));
            double p = 1.0;
            for (int n = 0; n < natom && p != 0.0; ++n) {
                if (n == m) continue;
                const double4 B = atoms[n];
                if (B.w < 0.0) continue;
                const double Am = A.w < 0.0 ? brad[m] : A.w;
                const double rn = sqrt((rx - B.x) * (rx - B.x) + (ry - B.y) * (ry - B.y) + (rz - B.z) * (rz - B.z));
                const double Rmn = sqrt((A.x - B.x) * (A.x - B.x) + (A.y - B.y) * (A.y - B.y) + (A.z - B.z) * (A.z - B.z));
                double u = (rm - rn) * (1.0 / Rmn);
                if (size_adjust) {
                    const double au = (Am - B.w) / (Am + B.w);
                    double a = au / (au * au - 1.0);
                    a = a < -0.5 ? -0.5 : (a > 0.5 ? 0.5 : a);
                    u = u + a * (1.0 - u * u);
                }
                p *= becke_s(u);
            }
            tot += p;
            if (m == own) pown = p;
        }
        w_out[i] = w_single[i] * (pown / tot);
    }
}

// Pair constants: inv[m*n_atom + n] = 1/|R_m - R_n|, adj[m*n_atom + n] = a_mn (0 without size adjustment).
// A dummy partner n (ghost[n] != 0) gets inv = 0 and adj = -1: then nu = -1 and its factor
// s = (1 - f3(-1)) / 2 is exactly 1 (f(-1) = -1 in IEEE arithmetic), the same as leaving it out.
__global__ void k_becke_pairs(const double* __restrict__ atom_xyz, const double* __restrict__ brad,
                              const int* __restrict__ ghost, int natom, int size_adjust, double* inv, double* adj) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < natom * natom; e += gridDim.x * blockDim.x) {
        const int m = e / natom, n = e % natom;
        if (m == n) {
            inv[e] = adj[e] = 0.0;
            continue;
        }
        if (ghost && ghost[n]) {
            inv[e] = 0.0, adj[e] = -1.0;
            continue;
        }
        const double dx = atom_xyz[3 * m] - atom_xyz[3 * n], dy = atom_xyz[3 * m + 1] - atom_xyz[3 * n + 1],
                     dz = atom_xyz[3 * m + 2] - atom_xyz[3 * n + 2];
        inv[e] = 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
        double a = 0.0;
        if (size_adjust) {
            const double au = (brad[m] - brad[n]) / (brad[m] + brad[n]);
            a = au / (au * au - 1.0);
            a = a < -0.5 ? -0.5 : (a > 0.5 ? 0.5 : a);
        }
        adj[e] = a;
    }
}

// Same weights as k_becke, one point per thread, with each thread's point-atom distances kept in
// shared memory ([atom][thread]) and the pair constants read from the table: one multiply per
// pair instead of two square roots and a division. Its shared memory per CTA grows with the atom
// count, so it is the form for small molecules (becke_small_atoms), k_becke_warp the one above.
constexpr int BECKE_T = 64;
__global__ void __launch_bounds__(BECKE_T) k_becke_tab(const double* __restrict__ atom_xyz, int natom,
                                                       const double* __restrict__ inv, const double* __restrict__ adj,
                                                       int64_t npts, const double* __restrict__ xyz,
                                                       const int* __restrict__ owner,
                                                       const double* __restrict__ w_single, double* __restrict__ w_out) {
    extern __shared__ double rr[];  // [natom][BECKE_T]
    const int t = threadIdx.x;
    for (int64_t i0 = blockIdx.x * (int64_t)BECKE_T; i0 < npts; i0 += (int64_t)gridDim.x * BECKE_T) {
        const int64_t i = i0 + t;
        const bool live = i < npts;
        const double rx = live ? xyz[3 * i] : 0.0, ry = live ? xyz[3 * i + 1] : 0.0, rz = live ? xyz[3 * i + 2] : 0.0;
        for (int m = 0; m < natom; ++m) {
            const double ax = atom_xyz[3 * m] - rx, ay = atom_xyz[3 * m + 1] - ry, az = atom_xyz[3 * m + 2] - rz;
            rr[m * BECKE_T + t] = sqrt(ax * ax + ay * ay + az * az);
        }
        if (live) {
            const int own = owner[i];
            double tot = 0.0, pown = 0.0;
            for (int m = 0; m < natom; ++m) {
                const double rm = rr[m * BECKE_T + t];
                const double* im = inv + (size_t)m * natom;
                const double* am = adj + (size_t)m * natom;
                double p = 1.0;
                for (int n = 0; n < natom && p != 0.0; ++n) {
                    if (n == m) continue;
                    double u = (rm - rr[n * BECKE_T + t]) * __ldg(im + n);
                    u = u + __ldg(am + n) * (1.0 - u * u);
                    p *= becke_s(u);
                }
                tot += p;
                if (m == own) pown = p;
            }
            w_out[i] = w_single[i] * (pown / tot);
        }
    }
}

// Stratmann-Scuseria partition (DfGenerateGrid::calcMultiCenterWeight_SS,
// src/libpdf/DfGenerateGrid.cpp:1878-1956): s = (1 - g(mu))/2 with g the
// piecewise polynomial of a = 0.64, no size adjustment. s is exactly 0 for
// mu >= a and exactly 1 for mu <= -a (the polynomial is -1 / +1 at z = -1 / +1),
// which bounds the atoms that matter at a point (k_ss); 1/R_mn from the pair table.
__device__ __forceinline__ double ss_s(double u) {
    constexpr double a = 0.64;
    double g;
    if (u < -a) {
        g = -1.0;
    } else if (u > a) {
        g = 1.0;
    } else {
        const double z = u / a, z2 = z * z, z3 = z2 * z, z5 = z2 * z3;
        g = (1.0 / 16.0) * (35.0 * z - 35.0 * z3 + 21.0 * z5 - 5.0 * z5 * z2);
    }
    return 0.5 * (1.0 - g);
}

// One thread per point. For a point r owned by atom A at distance d, an atom m can have
// P_m = prod_n s(mu_mn) != 0 only if |A - m| < 2 d / (1 - a) (otherwise mu_mA >= a, s = 0), and
// a factor s(mu_mn) can differ from 1 only if |m - n| < 2 |r - m| / (1 - a) (otherwise
// mu_mn <= -a, s = 1): both bounds from |r - n| >= |m - n| - |r - m|, and s is exactly 0 / 1 at
// +-a. So the candidates m are A and A's neighbours up to 2 d / (1 - a), and the factors of P_m
// come from m's neighbours up to 2 |r - m| / (1 - a), each list sorted by distance; the
// skipped factors are exactly 1 and the skipped terms exactly 0. Points deep inside their
// owner's cell see no candidate and no factor (w = w_single). nbr_idx / nbr_dist: per atom the
// other atoms in ascending distance (natom - 1 entries).
__global__ void __launch_bounds__(128) k_ss(const double* __restrict__ atom_xyz, int natom,
                                            const double* __restrict__ inv, const int* __restrict__ nbr_idx,
                                            const double* __restrict__ nbr_dist, int64_t npts,
                                            const double* __restrict__ xyz, const int* __restrict__ owner,
                                            const double* __restrict__ w_single, double* __restrict__ w_out) {
    constexpr double kReach = 2.0 / (1.0 - 0.64);
    const int nn = natom - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < npts; i += (int64_t)gridDim.x * blockDim.x) {
        const double rx = xyz[3 * i], ry = xyz[3 * i + 1], rz = xyz[3 * i + 2];
        const int own = owner[i];
        auto dist = [&](int a) {
            const double dx = rx - atom_xyz[3 * a], dy = ry - atom_xyz[3 * a + 1], dz = rz - atom_xyz[3 * a + 2];
            return sqrt(dx * dx + dy * dy + dz * dz);
        };
        const double lim_own = kReach * dist(own);
        double tot = 0.0, pown = 0.0;
        for (int k = -1; k < nn; ++k) {
            int m = own;
            if (k >= 0) {
                if (nbr_dist[(size_t)own * nn + k] >= lim_own) break;
                m = nbr_idx[(size_t)own * nn + k];
            }
            const double rm = dist(m), lim_m = kReach * rm;
            const double* im = inv + (size_t)m * natom;
            const int* ni = nbr_idx + (size_t)m * nn;
            const double* nd = nbr_dist + (size_t)m * nn;
            double p = 1.0;
            for (int j = 0; j < nn && p != 0.0; ++j) {
                if (nd[j] >= lim_m) break;
                const int n = ni[j];
                p *= ss_s((rm - dist(n)) * __ldg(im + n));
            }
            tot += p;
            if (m == own) pown = p;
        }
        w_out[i] = w_single[i] * (pown / tot);
    }
}

}  // namespace

void launch_ss(const double* atom_xyz, int natom, double* inv, double* adj, const int* nbr_idx,
               const double* nbr_dist, int64_t npts, const double* xyz, const int* owner, const double* w_single,
               double* w_out, cudaStream_t s) {
    k_becke_pairs<<<(natom * natom + 255) / 256, 256, 0, s>>>(atom_xyz, atom_xyz, nullptr, natom, 0, inv, adj);
    const int threads = 128;
    int64_t blocks = (npts + threads - 1) / threads;
    if (blocks > 148 * 64) blocks = 148 * 64;
    if (blocks < 1) blocks = 1;
    k_ss<<<(unsigned)blocks, threads, 0, s>>>(atom_xyz, natom, inv, nbr_idx, nbr_dist, npts, xyz, owner, w_single,
                                              w_out);
}

void launch_becke_pairs(const double* atom_xyz, const double* brad, int natom, int size_adjust, double* inv,
                        double* adj, cudaStream_t s) {
    k_becke_pairs<<<(natom * natom + 255) / 256, 256, 0, s>>>(atom_xyz, brad, nullptr, natom, size_adjust, inv, adj);
}

// The weights of k_becke with the pair constants from the table (one multiply per pair instead of
// two square roots and a division) and a warp per point: lane l forms P_m for m = l, l + 32, ...
// with the factors in ascending partner order, and lane 0 sums the P_m in ascending m, the
// operations and order of k_becke. The pair constants are read from the transposed table
// (invT[n][m] = inv[m][n], adjT[n][m] = adj[m][n]), so that the lanes' loads for one partner n
// are consecutive; per warp, the point's distances and the P_m sit in shared memory, 16 bytes
// per atom. (k_becke_tab keeps one point per thread, with that point's natom distances per thread
// in shared memory: at 100 atoms a few warps per SM and twice this kernel's time.)
constexpr int BECKE_WW = 8;  // warps per CTA
__global__ void __launch_bounds__(32 * BECKE_WW) k_becke_warp(const double* __restrict__ atom_xyz, int natom,
                                                              const double* __restrict__ invT,
                                                              const double* __restrict__ adjT, int64_t npts,
                                                              const double* __restrict__ xyz,
                                                              const int* __restrict__ owner,
                                                              const double* __restrict__ w_single,
                                                              double* __restrict__ w_out) {
    extern __shared__ double smw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* rr = smw + (size_t)warp * 2 * natom;  // [natom]: |r - R_m|
    double* ps = rr + natom;                      // [natom]: P_m(r)
    for (int64_t i = blockIdx.x * (int64_t)BECKE_WW + warp; i < npts; i += (int64_t)gridDim.x * BECKE_WW) {
        const double rx = xyz[3 * i], ry = xyz[3 * i + 1], rz = xyz[3 * i + 2];
        for (int m = lane; m < natom; m += 32) {
            const double ax = atom_xyz[3 * m] - rx, ay = atom_xyz[3 * m + 1] - ry, az = atom_xyz[3 * m + 2] - rz;
            rr[m] = sqrt(ax * ax + ay * ay + az * az);
        }
        __syncwarp();
        for (int m = lane; m < natom; m += 32) {
            const double rm = rr[m];
            double p = 1.0;
            for (int n = 0; n < natom && p != 0.0; ++n) {
                if (n == m) continue;
                double u = (rm - rr[n]) * __ldg(invT + (size_t)n * natom + m);
                u = u + __ldg(adjT + (size_t)n * natom + m) * (1.0 - u * u);
                p *= becke_s(u);
            }
            ps[m] = p;
        }
        __syncwarp();
        if (lane == 0) {
            double tot = 0.0;
            for (int m = 0; m < natom; ++m) tot += ps[m];
            w_out[i] = w_single[i] * (ps[owner[i]] / tot);
        }
        __syncwarp();  // rr and ps are rewritten for the next point
    }
}

__global__ void k_transpose_n2(const double* __restrict__ a, double* __restrict__ at, int n) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)n * n;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int r = (int)(e / n), c = (int)(e % n);
        at[(int64_t)c * n + r] = a[e];
    }
}

void launch_becke_tab(const double* atom_xyz, const double* brad, const int* ghost, int natom, int size_adjust,
                      double* inv, double* adj, int64_t npts, const double* xyz, const int* owner,
                      const double* w_single, double* w_out, cudaStream_t s) {
    k_becke_pairs<<<(natom * natom + 255) / 256, 256, 0, s>>>(atom_xyz, brad, ghost, natom, size_adjust, inv, adj);
    int64_t blocks = (npts + BECKE_T - 1) / BECKE_T;
    if (blocks > 148 * 32) blocks = 148 * 32;
    if (blocks < 1) blocks = 1;
    const size_t smem = sizeof(double) * BECKE_T * natom;
    cudaFuncSetAttribute(k_becke_tab, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_becke_tab<<<(unsigned)blocks, BECKE_T, smem, s>>>(atom_xyz, natom, inv, adj, npts, xyz, owner, w_single,
                                                        w_out);
}

// Up to this many atoms the one-point-per-thread form; above it the warp form. Measured on seeded
// chains with USER 75 x 302 grids (ncu durations, table form / warp form): 20 atoms 0.28 / 0.48 ms,
// 32 atoms 1.07 / 1.15 ms, 48 atoms 4.57 / 4.66 ms, 64 atoms 15.8 / 8.2 ms, 100 atoms 77 / 39 ms.
constexpr int kBeckeSmallAtoms = 48;
size_t becke_small_atoms() { return kBeckeSmallAtoms; }

size_t becke_warp_max_atoms() { return (200u * 1024u) / (2 * sizeof(double) * BECKE_WW); }

// tab: 4 n_atom^2 doubles (the pair table, then its transpose)
void launch_becke_warp(const double* atom_xyz, const double* brad, const int* ghost, int natom, int size_adjust,
                       double* tab, int64_t npts, const double* xyz, const int* owner, const double* w_single,
                       double* w_out, cudaStream_t s) {
    const size_t n2 = (size_t)natom * natom;
    double *inv = tab, *adj = tab + n2, *invT = tab + 2 * n2, *adjT = tab + 3 * n2;
    k_becke_pairs<<<(unsigned)((n2 + 255) / 256), 256, 0, s>>>(atom_xyz, brad, ghost, natom, size_adjust, inv, adj);
    const unsigned tb = (unsigned)std::min<size_t>((n2 + 255) / 256, 148 * 8);
    k_transpose_n2<<<tb, 256, 0, s>>>(inv, invT, natom);
    k_transpose_n2<<<tb, 256, 0, s>>>(adj, adjT, natom);
    int64_t blocks = (npts + BECKE_WW - 1) / BECKE_WW;
    if (blocks > 148 * 64) blocks = 148 * 64;
    if (blocks < 1) blocks = 1;
    const size_t smem = 2 * sizeof(double) * BECKE_WW * natom;
    cudaFuncSetAttribute(k_becke_warp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_becke_warp<<<(unsigned)blocks, 32 * BECKE_WW, smem, s>>>(atom_xyz, natom, invT, adjT, npts, xyz, owner, w_single,
                                                               w_out);
}

void launch_becke(const double* atom_xyz, const double* brad, const int* ghost, int natom, int size_adjust,
                  int64_t npts, const double* xyz, const int* owner, const double* w_single, double* w_out,
                  cudaStream_t s) {
    const int threads = 128;
    int64_t blocks = (npts + threads - 1) / threads;
    if (blocks > 148 * 64) blocks = 148 * 64;
    if (blocks < 1) blocks = 1;
    const size_t smem = sizeof(double4) * natom;
    cudaFuncSetAttribute(k_becke, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_becke<<<(unsigned)blocks, threads, smem, s>>>(atom_xyz, brad, ghost, natom, size_adjust, npts, xyz, owner,
                                                    w_single, w_out);
}

size_t becke_max_atoms() { return (220u * 1024u) / sizeof(double4); }

}  // namespace pdfxc
