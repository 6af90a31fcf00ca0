// XC nuclear gradient on the device (FP64): DfCalcGridX::energyGradient /
// energyGradient_part (src/libpdf/DfCalcGridX.cpp:1073-1415).
//
// AO-centre term, per block of 128 points with its screened AO list:
//   ao_grad      phi, grad phi and (GGA) the six second derivatives of every
//                screened AO (the reference's getAOs/getDAOs/getD2AOs, :667-863)
//   gemm_x       X = P_sub phi and (GGA) Y_k = P_sub d_k phi on the FP64 tensor cores
//   grad_point   rho, grad rho, the functional, and per AO i on atom B
//                G_i = a grad phi_i X_i + sum_k c_k (grad d_k phi_i X_i + grad phi_i Y_ki),
//                a = w vrho, c = w (2 vgAA + vgAB) grad rho_A;
//                grad[B] -= 4 G_i (the reference's -2 w, doubled for the closed shell),
//                grad[owner] += 4 G_i (the grid moves with its atom).
// Grid-weight term, per point with coefficient c = w_single f (f the energy density):
//                the derivative of the Becke partition omega_A = P_A / sum_i P_i with
//                respect to every nucleus (Johnson, Gill and Pople, J. Chem. Phys. 98,
//                5612 (1993), appendix B), written from the partition function; the
//                reference's own version of this term evaluates to zero (its JGP_t,
//                src/libpdf/DfGenerateGrid.cpp:2357-2372, returns 0 unless |mu| > 1).
#include <cuda_runtime.h>

#include "functional.cuh"
#include "pdfxc_internal.cuh"

namespace pdfxc {

namespace {

// Angular polynomial A of component t (s; px py pz; dxy dxz dyz d(x2-y2) dz2, the
// reference's prefactors, :103-141), its gradient and its second derivatives
// (xx xy xz yy yz zz).
__device__ __forceinline__ void ang_poly(int t, double x, double y, double z, double& A, double* Ak, double* Akl) {
    const double s3 = 0.57735026918962576451;  // 1/sqrt(3)
#pragma unroll
    for (int k = 0; k < 3; ++k) Ak[k] = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) Akl[k] = 0.0;
    switch (t) {
        case 0: A = 1.0; break;
        case 1: A = x; Ak[0] = 1.0; break;
        case 2: A = y; Ak[1] = 1.0; break;
        case 3: A = z; Ak[2] = 1.0; break;
        case 4: A = x * y; Ak[0] = y; Ak[1] = x; Akl[1] = 1.0; break;
        case 5: A = z * x; Ak[0] = z; Ak[2] = x; Akl[2] = 1.0; break;
        case 6: A = y * z; Ak[1] = z; Ak[2] = y; Akl[4] = 1.0; break;
        case 7: A = 0.5 * (x * x - y * y); Ak[0] = x; Ak[1] = -y; Akl[0] = 1.0; Akl[3] = -1.0; break;
        default:
            A = s3 * (z * z - 0.5 * (x * x + y * y));
            Ak[0] = -s3 * x; Ak[1] = -s3 * y; Ak[2] = 2.0 * s3 * z;
            Akl[0] = -s3; Akl[3] = -s3; Akl[5] = 2.0 * s3;
    }
}

// Workspace planes of one block ([nbp][128] doubles each): 0 phi, 1-3 grad phi,
// 4-9 second derivatives (GGA); then X (and Y_x, Y_y, Y_z for GGA).
__host__ __device__ inline int grad_phi_planes(bool gga) { return gga ? 10 : 4; }

// One CTA per block, 256 threads: the point is threadIdx.x % 128, the two halves
// of the CTA take alternate shells. d_k d_l (A e^{-a r^2}) =
// (A_kl - 2a (x_l A_k + x_k A_l) - 2a delta_kl A + 4a^2 x_k x_l A) e^{-a r^2}.
template <bool GGA>
__global__ void __launch_bounds__(256) k_ao_grad(BasisView bas, GridView g, int blk0, char* ws) {
    const int blk = blk0 + blockIdx.x;
    const BlockMeta m = g.meta[blk];
    const int p = threadIdx.x & (BLOCK_PTS - 1);
    const int half = threadIdx.x >> 7;
    double* out = reinterpret_cast<double*>(ws + m.ws);
    const size_t plane = (size_t)m.nbp * BLOCK_PTS;
    const int gp = blk * BLOCK_PTS + p;
    const double rx = g.px[gp], ry = g.py[gp], rz = g.pz[gp];
    constexpr int KL[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
    for (int i = half; i < m.nsh; i += 2) {
        const int s = g.blk_shells[m.sh0 + i];
        const int row0 = g.blk_shell_row[m.sh0 + i];
        const int at = bas.sh_atom[s];
        const double q[3] = {rx - bas.atom_xyz[3 * at], ry - bas.atom_xyz[3 * at + 1], rz - bas.atom_xyz[3 * at + 2]};
        const double d2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
        const int L = bas.sh_l[s], n = 2 * L + 1, np = bas.sh_nprim[s], p0 = bas.sh_p0[s];
        double v[5], gd[5][3], hd[5][6];
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            v[c] = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) gd[c][k] = 0.0;
#pragma unroll
            for (int k = 0; k < 6; ++k) hd[c][k] = 0.0;
        }
        for (int k = 0; k < np; ++k) {
            const double al = bas.p_exp[p0 + k];
            if (al * d2 > 30.0) continue;  // TOOBIG, DfCalcGridX.cpp:42, :690
            const double e = bas.p_coef[p0 + k] * exp(-al * d2);
            const double a2 = 2.0 * al;
#pragma unroll
            for (int c = 0; c < 5; ++c) {
                if (c >= n) break;
                double A, Ak[3], Akl[6];
                ang_poly(L * L + c, q[0], q[1], q[2], A, Ak, Akl);
                v[c] += A * e;
#pragma unroll
                for (int k = 0; k < 3; ++k) gd[c][k] += (Ak[k] - a2 * q[k] * A) * e;
                if (GGA) {
#pragma unroll
                    for (int h = 0; h < 6; ++h) {
                        const int kk = KL[h][0], ll = KL[h][1];
                        double t = Akl[h] - a2 * (q[ll] * Ak[kk] + q[kk] * Ak[ll]) + a2 * a2 * q[kk] * q[ll] * A;
                        if (kk == ll) t -= a2 * A;
                        hd[c][h] += t * e;
                    }
                }
            }
        }
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            if (c >= n) break;
            const size_t o = (size_t)(row0 + c) * BLOCK_PTS + p;
            out[o] = v[c];
#pragma unroll
            for (int k = 0; k < 3; ++k) out[(1 + k) * plane + o] = gd[c][k];
            if (GGA) {
#pragma unroll
                for (int h = 0; h < 6; ++h) out[(4 + h) * plane + o] = hd[c][h];
            }
        }
    }
    // zero the padding rows of every plane
    for (int r = m.nb + half; r < m.nbp; r += 2) {
        const size_t o = (size_t)r * BLOCK_PTS + p;
        for (int k = 0; k < grad_phi_planes(GGA); ++k) out[k * plane + o] = 0.0;
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// grad[3 * atom + k] += scale * (sum over the warp of v[k]); every lane calls it with the same atom.
__device__ __forceinline__ void warp_add3(double* grad, int atom, double scale, double vx, double vy, double vz) {
    const double sx = warp_sum(vx), sy = warp_sum(vy), sz = warp_sum(vz);
    if ((threadIdx.x & 31) == 0 && (sx != 0.0 || sy != 0.0 || sz != 0.0)) {
        atomicAdd(&grad[3 * atom], scale * sx);
        atomicAdd(&grad[3 * atom + 1], scale * sy);
        atomicAdd(&grad[3 * atom + 2], scale * sz);
    }
}

// grad[3 * own + k] += scale * v[k], lanes with the same owner summed first (a warp's
// points usually share one or two owners).
__device__ __forceinline__ void warp_add3_by_owner(double* grad, int own, double scale, double vx, double vy,
                                                   double vz) {
    const int lane = threadIdx.x & 31;
    unsigned todo = 0xffffffffu;
    while (todo) {
        const int src = __ffs(todo) - 1;
        const int o = __shfl_sync(0xffffffffu, own, src);
        const bool mine = own == o;
        todo &= ~__ballot_sync(0xffffffffu, mine);
        const double sx = warp_sum(mine ? vx : 0.0), sy = warp_sum(mine ? vy : 0.0), sz = warp_sum(mine ? vz : 0.0);
        if (lane == src && (sx != 0.0 || sy != 0.0 || sz != 0.0)) {
            atomicAdd(&grad[3 * o], scale * sx);
            atomicAdd(&grad[3 * o + 1], scale * sy);
            atomicAdd(&grad[3 * o + 2], scale * sz);
        }
    }
}

// One CTA (128 threads, one per point) per block. fdens receives the energy density
// f(rho) per point slot (0 below the density cut-off, for the weight term), blk_sum the
// block's Exc and electron-count partials, grad the AO-centre term (natom x 3). Every
// derivative is scaled by `seed`, the cotangent of Exc (1 for the plain gradient). With
// want_z the adjoint of the density with respect to P replaces X in place:
// Z_i = 0.5 a phi_i + c . grad phi_i (a = seed w vrho, c = seed w (2 vgAA + vgAB) grad rho),
// so that phi Z^T + Z phi^T summed over the blocks is seed dExc/dP.
template <bool GGA>
__global__ void __launch_bounds__(BLOCK_PTS) k_grad_point(GridView g, const int* __restrict__ ao_atom,
                                                          const int* __restrict__ owner, int blk0, int fn,
                                                          double rho_cut, char* ws, double seed, int want_z,
                                                          double* fdens, double* blk_sum, double* grad) {
    const int blk = blk0 + blockIdx.x;
    const BlockMeta m = g.meta[blk];
    const int p = threadIdx.x;
    const size_t plane = (size_t)m.nbp * BLOCK_PTS;
    const double* phi = reinterpret_cast<const double*>(ws + m.ws);
    double* X = reinterpret_cast<double*>(ws + m.ws) + grad_phi_planes(GGA) * plane;
    double rho = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
    for (int r = 0; r < m.nb; ++r) {
        const size_t o = (size_t)r * BLOCK_PTS + p;
        const double x = X[o];
        rho = fma(phi[o], x, rho);
        if (GGA) {
            gx = fma(phi[plane + o], x, gx);
            gy = fma(phi[2 * plane + o], x, gy);
            gz = fma(phi[3 * plane + o], x, gz);
        }
    }
    gx *= 2.0, gy *= 2.0, gz *= 2.0;
    const size_t gp = (size_t)blk * BLOCK_PTS + p;
    const double w = g.pw[gp];
    double f = 0.0, a = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
    if (w != 0.0 && rho > rho_cut) {
        const double gam = GGA ? gx * gx + gy * gy + gz * gz : 0.0;
        const XcOut o = eval_functional(fn, rho, rho, gam, gam, gam);
        f = o.f;
        a = seed * w * o.va;
        if (GGA) {
            const double cc = seed * w * (2.0 * o.vgaa + o.vgab);
            cx = cc * gx, cy = cc * gy, cz = cc * gz;
        }
    }
    fdens[gp] = seed * f;

    // AO-centre term: the block's AO list is in shell order, so each atom's AOs form runs
    const int* aos = g.blk_aos + m.ao0;
    double ax = 0.0, ay = 0.0, az = 0.0, tx = 0.0, ty = 0.0, tz = 0.0;
    int cur = m.nb > 0 ? ao_atom[aos[0]] : 0;
    for (int r = 0; r < m.nb; ++r) {
        const int at = ao_atom[aos[r]];  // the same for every thread of the CTA
        if (at != cur) {
            warp_add3(grad, cur, -4.0, ax, ay, az);
            ax = ay = az = 0.0;
            cur = at;
        }
        const size_t o = (size_t)r * BLOCK_PTS + p;
        const double x = X[o];
        const double d1x = phi[plane + o], d1y = phi[2 * plane + o], d1z = phi[3 * plane + o];
        double Gx = a * d1x * x, Gy = a * d1y * x, Gz = a * d1z * x;
        if (GGA) {
            const double cY = cx * X[plane + o] + cy * X[2 * plane + o] + cz * X[3 * plane + o];
            const double hxx = phi[4 * plane + o], hxy = phi[5 * plane + o], hxz = phi[6 * plane + o];
            const double hyy = phi[7 * plane + o], hyz = phi[8 * plane + o], hzz = phi[9 * plane + o];
            Gx += (cx * hxx + cy * hxy + cz * hxz) * x + d1x * cY;
            Gy += (cx * hxy + cy * hyy + cz * hyz) * x + d1y * cY;
            Gz += (cx * hxz + cy * hyz + cz * hzz) * x + d1z * cY;
        }
        ax += Gx, ay += Gy, az += Gz;
        tx += Gx, ty += Gy, tz += Gz;
        if (want_z) X[o] = 0.5 * a * phi[o] + (GGA ? cx * d1x + cy * d1y + cz * d1z : 0.0);
    }
    if (m.nb > 0) warp_add3(grad, cur, -4.0, ax, ay, az);
    warp_add3_by_owner(grad, owner[gp], 4.0, tx, ty, tz);

    // block sums in FP64 (deterministic order): Exc, electron count
    __shared__ double red[2][BLOCK_PTS / 32];
    const double se = warp_sum(w * f), sn = warp_sum(w * rho);
    if ((p & 31) == 0) red[0][p >> 5] = se, red[1][p >> 5] = sn;
    __syncthreads();
    if (p == 0) {
        double E = 0.0, N = 0.0;
        for (int i = 0; i < BLOCK_PTS / 32; ++i) E += red[0][i], N += red[1][i];
        blk_sum[2 * blk] = E;
        blk_sum[2 * blk + 1] = N;
    }
}

__device__ __forceinline__ void becke_poly(double nu, double& p1, double& p2, double& p3) {
    p1 = 0.5 * nu * (3.0 - nu * nu);
    p2 = 0.5 * p1 * (3.0 - p1 * p1);
    p3 = 0.5 * p2 * (3.0 - p2 * p2);
}

// Grid-weight term. T points per CTA (one per thread); shared memory holds each
// point's atom distances and partition products, [natom][T] each. Pair constants
// (1/R_ij and the size adjustment a_ij) come from the table k_becke_pairs writes.
// For B != owner A and every other atom i, one evaluation of nu_iB gives
// s_iB = (1 - f3)/2, s_Bi = (1 + f3)/2 (nu_Bi = -nu_iB), s'(nu_iB) = s'(nu_Bi) and
// grad_B mu_iB = -grad_B mu_Bi, so that
//   grad_B Z += s' dnu grad_B mu_iB (P_i / s_iB - P_B / s_Bi),
//   grad_B P_A = s'(nu_AB) dnu grad_B mu_AB P_A / s_AB,
// where P_i / s_iB is the product of P_i's other factors (taken as 0 when s_iB has
// underflowed: the term is then below 1e-250).
//
// ROWS_IN_DRAM: the two [natom] rows of every thread live in a scratch array in
// device memory ([2][natom][gridDim.x * T], a thread's entries strided by the
// grid's thread count, so a warp's accesses stay coalesced) instead of shared
// memory; the form for systems whose rows do not fit shared memory.
template <int T, bool ROWS_IN_DRAM>
__global__ void __launch_bounds__(T) k_grad_weight(const double* __restrict__ atom_xyz, int natom,
                                                   const double* __restrict__ inv, const double* __restrict__ adj,
                                                   int64_t nslots, const double* __restrict__ px,
                                                   const double* __restrict__ py, const double* __restrict__ pz,
                                                   const int* __restrict__ owner, const double* __restrict__ wsingle,
                                                   const double* __restrict__ fdens, double* grad,
                                                   double* __restrict__ scratch) {
    extern __shared__ double sm[];
    const size_t stride = ROWS_IN_DRAM ? (size_t)gridDim.x * T : (size_t)T;
    double* rr = ROWS_IN_DRAM ? scratch + (size_t)blockIdx.x * T : sm;  // [natom][stride]
    double* Pm = rr + (size_t)natom * stride;                            // [natom][stride]
    const int t = threadIdx.x;
    constexpr double kTiny = 1e-250;
    for (int64_t i0 = blockIdx.x * (int64_t)T; i0 < nslots; i0 += (int64_t)gridDim.x * T) {
        const int64_t i = i0 + t;
        const bool live = i < nslots;
        const double c = live ? wsingle[i] * fdens[i] : 0.0;
        if (!__syncthreads_or(c != 0.0)) continue;
        const double rx = live ? px[i] : 0.0, ry = live ? py[i] : 0.0, rz = live ? pz[i] : 0.0;
        const int A = live ? owner[i] : 0;
        for (int m = 0; m < natom; ++m) {
            const double ax = __ldg(atom_xyz + 3 * m) - rx, ay = __ldg(atom_xyz + 3 * m + 1) - ry,
                         az = __ldg(atom_xyz + 3 * m + 2) - rz;
            rr[m * stride + t] = sqrt(ax * ax + ay * ay + az * az);
            Pm[m * stride + t] = 1.0;
        }
        // partition products, each unordered pair once
        for (int m = 0; m < natom; ++m) {
            const double rm = rr[m * stride + t];
            double pmv = Pm[m * stride + t];
            for (int n = m + 1; n < natom; ++n) {
                double mu = (rm - rr[n * stride + t]) * __ldg(inv + (size_t)m * natom + n);
                const double nu = mu + __ldg(adj + (size_t)m * natom + n) * (1.0 - mu * mu);
                double p1, p2, p3;
                becke_poly(nu, p1, p2, p3);
                pmv *= 0.5 * (1.0 - p3);
                Pm[n * stride + t] *= 0.5 * (1.0 + p3);
            }
            Pm[m * stride + t] = pmv;
        }
        double Z = 0.0;
        for (int m = 0; m < natom; ++m) Z += Pm[m * stride + t];
        const bool act = c != 0.0 && Z > 0.0;
        const double invZ = act ? 1.0 / Z : 0.0;
        const double PA = Pm[A * stride + t];
        const double omega = PA * invZ;
        double Tx = 0.0, Ty = 0.0, Tz = 0.0;
        for (int B = 0; B < natom; ++B) {
            double dx = 0.0, dy = 0.0, dz = 0.0;
            if (act && B != A) {
                const double RBx = __ldg(atom_xyz + 3 * B), RBy = __ldg(atom_xyz + 3 * B + 1),
                             RBz = __ldg(atom_xyz + 3 * B + 2);
                const double rB = rr[B * stride + t];
                const double irB = 1.0 / rB;
                const double ux = (RBx - rx) * irB, uy = (RBy - ry) * irB, uz = (RBz - rz) * irB;
                const double PB = Pm[B * stride + t];
                double zx = 0.0, zy = 0.0, zz = 0.0, ax = 0.0, ay = 0.0, az = 0.0;
                for (int n = 0; n < natom; ++n) {
                    if (n == B) continue;
                    const double iR = __ldg(inv + (size_t)n * natom + B);
                    const double a = __ldg(adj + (size_t)n * natom + B);
                    const double mu = (rr[n * stride + t] - rB) * iR;
                    const double nu = mu + a * (1.0 - mu * mu);
                    double p1, p2, p3;
                    becke_poly(nu, p1, p2, p3);
                    const double s_nB = 0.5 * (1.0 - p3), s_Bn = 0.5 * (1.0 + p3);
                    const double k = -(27.0 / 16.0) * (1.0 - p2 * p2) * (1.0 - p1 * p1) * (1.0 - nu * nu) *
                                     (1.0 - 2.0 * a * mu);
                    const double ex = (RBx - __ldg(atom_xyz + 3 * n)) * iR, ey = (RBy - __ldg(atom_xyz + 3 * n + 1)) * iR,
                                 ez = (RBz - __ldg(atom_xyz + 3 * n + 2)) * iR;
                    const double gmx = -(ux + mu * ex) * iR, gmy = -(uy + mu * ey) * iR, gmz = -(uz + mu * ez) * iR;
                    const double rn = s_nB > kTiny ? Pm[n * stride + t] / s_nB : 0.0;
                    const double rb = s_Bn > kTiny ? PB / s_Bn : 0.0;
                    const double f = k * (rn - rb);
                    zx += f * gmx, zy += f * gmy, zz += f * gmz;
                    if (n == A) ax = k * rn * gmx, ay = k * rn * gmy, az = k * rn * gmz;
                }
                dx = c * (ax - omega * zx) * invZ;
                dy = c * (ay - omega * zy) * invZ;
                dz = c * (az - omega * zz) * invZ;
            }
            warp_add3(grad, B, 1.0, dx, dy, dz);
            Tx += dx, Ty += dy, Tz += dz;
        }
        warp_add3_by_owner(grad, A, -1.0, Tx, Ty, Tz);
        __syncthreads();  // shared rows are rewritten by the next tile of points
    }
}

}  // namespace

int grad_workspace_planes(bool gga) { return grad_phi_planes(gga) + (gga ? 4 : 1); }

void launch_ao_grad(const BasisView& b, const GridView& g, int blk0, int nblk, bool gga, char* ws, cudaStream_t s) {
    if (gga)
        k_ao_grad<true><<<nblk, 256, 0, s>>>(b, g, blk0, ws);
    else
        k_ao_grad<false><<<nblk, 256, 0, s>>>(b, g, blk0, ws);
}

void launch_grad_x(const GridView& g, const double* P, int nao, int blk0, int nblk, int max_nbp, bool gga, char* ws,
                   cudaStream_t s) {
    // X = P_sub phi (LDA); X, Y_x, Y_y, Y_z = P_sub (phi, d_x phi, d_y phi, d_z phi) (GGA)
    launch_gemm_x_planes(g, P, nao, blk0, nblk, max_nbp, 0, grad_phi_planes(gga), gga ? 4 : 1, ws, s);
}

void launch_grad_point(const GridView& g, const int* ao_atom, const int* owner, int blk0, int nblk, int fn,
                       double rho_cut, char* ws, double seed, bool want_z, double* fdens, double* blk_sum,
                       double* grad, cudaStream_t s) {
    if (functional_is_gga(fn))
        k_grad_point<true><<<nblk, BLOCK_PTS, 0, s>>>(g, ao_atom, owner, blk0, fn, rho_cut, ws, seed, want_z ? 1 : 0,
                                                      fdens, blk_sum, grad);
    else
        k_grad_point<false><<<nblk, BLOCK_PTS, 0, s>>>(g, ao_atom, owner, blk0, fn, rho_cut, ws, seed,
                                                       want_z ? 1 : 0, fdens, blk_sum, grad);
}

int grad_z_plane(bool gga) { return grad_phi_planes(gga); }

// Shared memory per CTA: 2 * natom * T doubles; 64 points per CTA while that fits
// 200 KiB, else 32; beyond 400 atoms the rows live in device memory
// (grad_weight_scratch_doubles of scratch).
int grad_weight_max_atoms() { return (int)((200u * 1024u) / (2 * sizeof(double) * 32)); }

namespace {
constexpr int kWeightDramCtas = 148 * 4;
}

size_t grad_weight_scratch_doubles(int natom) { return (size_t)2 * natom * kWeightDramCtas * 32; }

void launch_grad_weight(const double* atom_xyz, int natom, const double* inv, const double* adj, int64_t nslots,
                        const double* px, const double* py, const double* pz, const int* owner, const double* wsingle,
                        const double* fdens, double* grad, double* scratch, cudaStream_t s) {
    const size_t smem64 = 2 * sizeof(double) * 64 * (size_t)natom;
    const size_t smem32 = 2 * sizeof(double) * 32 * (size_t)natom;
    if (scratch) {
        int64_t blocks = (nslots + 31) / 32;
        if (blocks > kWeightDramCtas) blocks = kWeightDramCtas;
        k_grad_weight<32, true><<<(unsigned)blocks, 32, 0, s>>>(atom_xyz, natom, inv, adj, nslots, px, py, pz, owner,
                                                               wsingle, fdens, grad, scratch);
    } else if (smem64 <= 200u * 1024u) {
        int64_t blocks = (nslots + 63) / 64;
        if (blocks > 148 * 16) blocks = 148 * 16;
        cudaFuncSetAttribute(k_grad_weight<64, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem64);
        k_grad_weight<64, false><<<(unsigned)blocks, 64, smem64, s>>>(atom_xyz, natom, inv, adj, nslots, px, py, pz,
                                                                     owner, wsingle, fdens, grad, nullptr);
    } else {
        int64_t blocks = (nslots + 31) / 32;
        if (blocks > 148 * 16) blocks = 148 * 16;
        cudaFuncSetAttribute(k_grad_weight<32, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem32);
        k_grad_weight<32, false><<<(unsigned)blocks, 32, smem32, s>>>(atom_xyz, natom, inv, adj, nslots, px, py, pz,
                                                                     owner, wsingle, fdens, grad, nullptr);
    }
}

}  // namespace pdfxc
