// FP64 drop-in kernels of the XC build.
//
// Per block of up to 128 grid points with its screened AO list (nb AOs, padded
// to nbp rows), one build runs
//   ao_eval      phi[mu][p], grad phi[k][mu][p]                (DfCalcGridX.cpp:667-769)
//   gemm_x       X = P_sub * phi, P_sub = P_A[aos, aos]
//   rho_functional  rho_A(p) = sum_mu phi X, grad rho_A = 2 sum_mu grad phi X
//                (:865-931), the functional, Exc and electron-count partials,
//                and the per-point Vxc coefficients (:2056-2193, :2455-2500)
//   gemm_v       Vacc[aos, aos] += phi * Z^T with
//                Z[nu][p] = 0.5 w vrho phi + c . grad phi, c = w (2 vgAA + vgAB) grad rho_A
//   finish       V = Vacc + Vacc^T, FP64 block sums of Exc and the electron count
// V = phi Z^T + Z phi^T reproduces the reference's element formula
// V_ij += w vrho phi_i phi_j + phi_i (c . grad phi_j) + phi_j (c . grad phi_i).
#include <cuda_runtime.h>

#include "ao.cuh"
#include "functional.cuh"
#include "pdfxc_internal.cuh"

namespace pdfxc {

namespace {

// One CTA per block, 256 threads: the point is threadIdx.x % 128, the two
// halves of the CTA take alternate shells. Stores are coalesced along points.
// Per shell the contraction is summed once (shell_radial), then every component
// is formed from the radial sums (ao_from_radial).
template <bool GGA>
__global__ void __launch_bounds__(256) k_ao_eval(BasisView bas, GridView g, int blk0, char* ws) {
    const int blk = blk0 + blockIdx.x;
    const BlockMeta m = g.meta[blk];
    const int p = threadIdx.x & (BLOCK_PTS - 1);
    const int half = threadIdx.x >> 7;
    double* phi = reinterpret_cast<double*>(ws + m.ws);
    double* dphi = phi + (size_t)m.nbp * BLOCK_PTS;
    const size_t plane = (size_t)m.nbp * BLOCK_PTS;
    const int gp = blk * BLOCK_PTS + p;
    const double rx = g.px[gp], ry = g.py[gp], rz = g.pz[gp];
    for (int i = half; i < m.nsh; i += 2) {
        const int s = g.blk_shells[m.sh0 + i];
        const int row0 = g.blk_shell_row[m.sh0 + i];
        const int a = bas.sh_atom[s];
        const double x = rx - bas.atom_xyz[3 * a], y = ry - bas.atom_xyz[3 * a + 1],
                     z = rz - bas.atom_xyz[3 * a + 2];
        const int L = bas.sh_l[s], n = 2 * L + 1;
        double S0, S1;
        shell_radial<GGA>(bas, s, x * x + y * y + z * z, S0, S1);
        for (int c = 0; c < n; ++c) {
            double v, gx, gy, gz;
            ao_from_radial<GGA>(L * L + c, x, y, z, S0, S1, v, gx, gy, gz);
            const size_t o = (size_t)(row0 + c) * BLOCK_PTS + p;
            phi[o] = v;
            if (GGA) {
                dphi[o] = gx;
                dphi[plane + o] = gy;
                dphi[2 * plane + o] = gz;
            }
        }
    }
    // zero the padding rows
    for (int r = m.nb + half; r < m.nbp; r += 2) {
        const size_t o = (size_t)r * BLOCK_PTS + p;
        phi[o] = 0.0;
        if (GGA) dphi[o] = dphi[plane + o] = dphi[2 * plane + o] = 0.0;
    }
}

// FP64 tensor-core MMA: D(8x8) += A(8x4, row-major) B(4x8, col-major), FP64 in and out.
// Per thread (g = lane / 4, t = lane % 4): a = A[g][t], b = B[t][g], d = {D[g][2t], D[g][2t+1]}.
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// X[m][p] = sum_k P[aos[m]][aos[k]] phi[k][p]: CTA tile 64 rows x 128 points, K step 16,
// 8 warps as 2 x 4 warp tiles of 32 x 32 (4 x 4 DMMA tiles). The next K step's operands
// are fetched into registers while the current one is multiplied. Planes are [nbp][128]
// arrays of the block's workspace: source plane src0 + z, destination plane dst0 + z for
// blockIdx.z = z (the build: one plane, phi -> X after the phi planes; the gradient:
// phi and its three derivatives -> X and Y_x, Y_y, Y_z).
constexpr int GX_BM = 64, GX_BK = 16, GX_AS = GX_BK + 2, GX_BS = BLOCK_PTS + 4;
__global__ void __launch_bounds__(256, 2) k_gemm_x(GridView g, const double* __restrict__ P, int nao,
                                                int blk0, char* ws, int src0, int dst0, int64_t t0) {
    int blk, m0;
    if (g.xtiles) {  // one CTA per tile of the list
        const int2 it = g.xtiles[t0 + blockIdx.x];
        blk = it.x, m0 = it.y * GX_BM;
    } else {
        blk = blk0 + blockIdx.y, m0 = blockIdx.x * GX_BM;
    }
    const BlockMeta m = g.meta[blk];
    if (m0 >= m.nbp) return;
    const size_t plane = (size_t)m.nbp * BLOCK_PTS;
    const double* phi = reinterpret_cast<const double*>(ws + m.ws) + (size_t)(src0 + blockIdx.z) * plane;
    double* X = reinterpret_cast<double*>(ws + m.ws) + (size_t)(dst0 + blockIdx.z) * plane;
    const int* aos = g.blk_aos + m.ao0;

    __shared__ double As[GX_BM * GX_AS];   // [m][k]
    __shared__ double Bs[GX_BK * GX_BS];   // [k][n]
    __shared__ int s_row[GX_BM];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int wm = warp >> 2, wn = warp & 3, gq = lane >> 2, tq = lane & 3;
    for (int r = t; r < GX_BM; r += 256) s_row[r] = (m0 + r < m.nb) ? aos[m0 + r] : -1;
    __syncthreads();

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

    double ra[4], rb[8];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {  // A: 64 x 16 gathered from P (L2-resident)
            const int e = t + q * 256, r = e >> 4, c = e & 15, gc = k0 + c;
            const int row = s_row[r];
            ra[q] = (row >= 0 && gc < m.nb) ? __ldg(P + (size_t)row * nao + aos[gc]) : 0.0;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {  // B: 16 x 128 of phi, coalesced
            const int e = t + q * 256, r = e >> 7, c = e & 127;
            rb[q] = phi[(size_t)(k0 + r) * BLOCK_PTS + c];
        }
    };
    fetch(0);
    for (int k0 = 0; k0 < m.nbp; k0 += GX_BK) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int e = t + q * 256;
            As[(e >> 4) * GX_AS + (e & 15)] = ra[q];
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int e = t + q * 256;
            Bs[(e >> 7) * GX_BS + (e & 127)] = rb[q];
        }
        __syncthreads();
        if (k0 + GX_BK < m.nbp) fetch(k0 + GX_BK);
#pragma unroll
        for (int kk = 0; kk < GX_BK; kk += 4) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[(wm * 32 + i * 8 + gq) * GX_AS + kk + tq];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[(kk + tq) * GX_BS + wn * 32 + j * 8 + gq];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            double2* dst = reinterpret_cast<double2*>(X + (size_t)(m0 + wm * 32 + i * 8 + gq) * BLOCK_PTS + wn * 32 +
                                                      j * 8 + 2 * tq);
            *dst = make_double2(acc[i][j][0], acc[i][j][1]);
        }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One CTA (128 threads, one per point) per block.
template <bool GGA>
__global__ void __launch_bounds__(BLOCK_PTS) k_rho_functional(GridView g, int blk0, int fn, int incremental,
                                                              double rho_cut, char* ws, double* rho_store,
                                                              double* coef, double* blk_sum) {
    const int blk = blk0 + blockIdx.x;
    const BlockMeta m = g.meta[blk];
    const int p = threadIdx.x;
    const int nplanes = GGA ? 4 : 1;
    const double* phi = reinterpret_cast<const double*>(ws + m.ws);
    const size_t plane = (size_t)m.nbp * BLOCK_PTS;
    const double* X = phi + nplanes * plane;
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
    double* rs = rho_store + gp * 4;
    if (incremental) {
        rho += rs[0];
        gx += rs[1], gy += rs[2], gz += rs[3];
    }
    rs[0] = rho, rs[1] = gx, rs[2] = gy, rs[3] = gz;
    const double w = g.pw[gp];
    double e = 0.0, a = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
    if (w != 0.0 && rho > rho_cut) {
        const double gam = gx * gx + gy * gy + gz * gz;
        const XcOut o = eval_functional(fn, rho, rho, gam, gam, gam);
        e = w * o.f;
        a = 0.5 * w * o.va;
        if (GGA) {
            const double cc = w * (2.0 * o.vgaa + o.vgab);
            cx = cc * gx, cy = cc * gy, cz = cc * gz;
        }
    }
    double* cf = coef + gp * 4;
    cf[0] = a, cf[1] = cx, cf[2] = cy, cf[3] = cz;
    // Z[nu][p] = 0.5 w vrho phi + c . grad phi, written over X (no longer needed), all nbp rows
    double* Z = const_cast<double*>(X);
    for (int r = 0; r < m.nbp; ++r) {
        const size_t o = (size_t)r * BLOCK_PTS + p;
        double z = a * phi[o];
        if (GGA) z += cx * phi[plane + o] + cy * phi[2 * plane + o] + cz * phi[3 * plane + o];
        Z[o] = z;
    }
    // block sums in FP64 (deterministic order)
    __shared__ double red[2][BLOCK_PTS / 32];
    double se = warp_sum(e), sn = warp_sum(w * rho);
    if ((p & 31) == 0) red[0][p >> 5] = se, red[1][p >> 5] = sn;
    __syncthreads();
    if (p == 0) {
        double E = 0.0, N = 0.0;
        for (int i = 0; i < BLOCK_PTS / 32; ++i) E += red[0][i], N += red[1][i];
        blk_sum[2 * blk] = E;
        blk_sum[2 * blk + 1] = N;
    }
}

// GGA closed-shell build without stored AO gradients. Layout of a block (doubles):
// phi [nbp][128], X then Z [nbp][128], then the radial sums S0 [nsh][128] and S1 [nsh][128]
// (block_ws_doubles_rad). k_ao_eval_rad writes phi and the radial sums; k_rho_functional_rad
// forms phi and grad phi of every component from the radial sums (ao_from_radial, the
// formulas of k_ao_eval) in row order, so rho and grad rho are summed as from stored planes,
// and reads 2 nsh + nb rows per point instead of 5 nbp (and 2 nsh + nbp instead of 4 nbp for Z).
// The shells (rows, angular momenta, atoms, primitives) are staged in shared memory, 64 at a time.
__global__ void __launch_bounds__(256) k_ao_eval_rad(BasisView bas, GridView g, int blk0, char* ws) {
    const int blk = blk0 + blockIdx.x;
    const BlockMeta m = g.meta[blk];
    const int p = threadIdx.x & (BLOCK_PTS - 1);
    const int half = threadIdx.x >> 7;
    double* phi = reinterpret_cast<double*>(ws + m.ws);
    const size_t plane = (size_t)m.nbp * BLOCK_PTS;
    double* S0p = phi + 2 * plane;
    double* S1p = S0p + (size_t)m.nsh * BLOCK_PTS;
    const int gp = blk * BLOCK_PTS + p;
    const double rx = g.px[gp], ry = g.py[gp], rz = g.pz[gp];
    __shared__ ShellRec recs[64];  // the block's shells, 64 at a time
    for (int i0 = 0; i0 < m.nsh; i0 += 64) {
        __syncthreads();
        for (int k = threadIdx.x; k < 64 && i0 + k < m.nsh; k += blockDim.x)
            stage_shell(bas, g.blk_shells[m.sh0 + i0 + k], g.blk_shell_row[m.sh0 + i0 + k], recs[k]);
        __syncthreads();
        for (int i = i0 + half; i < min(i0 + 64, m.nsh); i += 2) {
            const ShellRec& r = recs[i - i0];
            const double x = rx - r.ax, y = ry - r.ay, z = rz - r.az;
            const int L = r.lq, n = 2 * L + 1;
            double S0, S1;
            shell_radial_staged<true>(bas, r, x * x + y * y + z * z, S0, S1);
            S0p[(size_t)i * BLOCK_PTS + p] = S0;
            S1p[(size_t)i * BLOCK_PTS + p] = S1;
            for (int c = 0; c < n; ++c) {
                double v, gx, gy, gz;
                ao_from_radial<false>(L * L + c, x, y, z, S0, S1, v, gx, gy, gz);
                phi[(size_t)(r.row0 + c) * BLOCK_PTS + p] = v;
            }
        }
    }
    for (int r = m.nb + half; r < m.nbp; r += 2) phi[(size_t)r * BLOCK_PTS + p] = 0.0;
}

struct ShellStage {
    double ax[128], ay[128], az[128];
    int row0[128], lq[128];
};

__device__ __forceinline__ void stage_shells(const BasisView& bas, const GridView& g, const BlockMeta& m, int i0,
                                             ShellStage& st) {
    for (int k = threadIdx.x; k < 128 && i0 + k < m.nsh; k += blockDim.x) {
        const int s = g.blk_shells[m.sh0 + i0 + k];
        const int a = bas.sh_atom[s];
        st.ax[k] = bas.atom_xyz[3 * a], st.ay[k] = bas.atom_xyz[3 * a + 1], st.az[k] = bas.atom_xyz[3 * a + 2];
        st.row0[k] = g.blk_shell_row[m.sh0 + i0 + k];
        st.lq[k] = bas.sh_l[s];
    }
}

__global__ void __launch_bounds__(BLOCK_PTS) k_rho_functional_rad(BasisView bas, GridView g, int blk0, int fn,
                                                                  int incremental, double rho_cut, char* ws,
                                                                  double* rho_store, double* coef, double* blk_sum) {
    __shared__ ShellStage st;
    const int blk = blk0 + blockIdx.x;
    const BlockMeta m = g.meta[blk];
    const int p = threadIdx.x;
    const size_t plane = (size_t)m.nbp * BLOCK_PTS;
    double* X = reinterpret_cast<double*>(ws + m.ws) + plane;
    const double* S0p = X + plane;
    const double* S1p = S0p + (size_t)m.nsh * BLOCK_PTS;
    const size_t gp = (size_t)blk * BLOCK_PTS + p;
    const double px = g.px[gp], py = g.py[gp], pz = g.pz[gp];
    double rho = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
    double v[5], ax[5], ay[5], az[5];
    for (int i0 = 0; i0 < m.nsh; i0 += 128) {
        __syncthreads();
        stage_shells(bas, g, m, i0, st);
        __syncthreads();
        const int kn = min(128, m.nsh - i0);
        double S0n = S0p[(size_t)i0 * BLOCK_PTS + p], S1n = S1p[(size_t)i0 * BLOCK_PTS + p];
        for (int k = 0; k < kn; ++k) {
            const int i = i0 + k;
            const double S0 = S0n, S1 = S1n;
            if (k + 1 < kn) S0n = S0p[(size_t)(i + 1) * BLOCK_PTS + p], S1n = S1p[(size_t)(i + 1) * BLOCK_PTS + p];
            const int L = st.lq[k], row0 = st.row0[k];
            shell_components(L, px - st.ax[k], py - st.ay[k], pz - st.az[k], S0, S1, v, ax, ay, az);
#pragma unroll
            for (int c = 0; c < 5; ++c) {
                if (c < 2 * L + 1) {
                    const double xv = X[(size_t)(row0 + c) * BLOCK_PTS + p];
                    rho = fma(v[c], xv, rho);
                    gx = fma(ax[c], xv, gx);
                    gy = fma(ay[c], xv, gy);
                    gz = fma(az[c], xv, gz);
                }
            }
        }
    }
    gx *= 2.0, gy *= 2.0, gz *= 2.0;
    double* rs = rho_store + gp * 4;
    if (incremental) {
        rho += rs[0];
        gx += rs[1], gy += rs[2], gz += rs[3];
    }
    rs[0] = rho, rs[1] = gx, rs[2] = gy, rs[3] = gz;
    const double w = g.pw[gp];
    double e = 0.0, a = 0.0, cx = 0.0, cy = 0.0, cz = 0.0;
    if (w != 0.0 && rho > rho_cut) {
        const double gam = gx * gx + gy * gy + gz * gz;
        const XcOut o = eval_functional(fn, rho, rho, gam, gam, gam);
        e = w * o.f;
        a = 0.5 * w * o.va;
        const double cc = w * (2.0 * o.vgaa + o.vgab);
        cx = cc * gx, cy = cc * gy, cz = cc * gz;
    }
    double* cf = coef + gp * 4;
    cf[0] = a, cf[1] = cx, cf[2] = cy, cf[3] = cz;
    // Z[nu][p] = 0.5 w vrho phi + c . grad phi over X (every row of X has been read by this thread)
    for (int i0 = 0; i0 < m.nsh; i0 += 128) {
        __syncthreads();
        stage_shells(bas, g, m, i0, st);
        __syncthreads();
        const int kn = min(128, m.nsh - i0);
        double S0n = S0p[(size_t)i0 * BLOCK_PTS + p], S1n = S1p[(size_t)i0 * BLOCK_PTS + p];
        for (int k = 0; k < kn; ++k) {
            const int i = i0 + k;
            const double S0 = S0n, S1 = S1n;
            if (k + 1 < kn) S0n = S0p[(size_t)(i + 1) * BLOCK_PTS + p], S1n = S1p[(size_t)(i + 1) * BLOCK_PTS + p];
            const int L = st.lq[k], row0 = st.row0[k];
            shell_components(L, px - st.ax[k], py - st.ay[k], pz - st.az[k], S0, S1, v, ax, ay, az);
#pragma unroll
            for (int c = 0; c < 5; ++c)
                if (c < 2 * L + 1) X[(size_t)(row0 + c) * BLOCK_PTS + p] = a * v[c] + cx * ax[c] + cy * ay[c] + cz * az[c];
        }
    }
    for (int r = m.nb; r < m.nbp; ++r) X[(size_t)r * BLOCK_PTS + p] = 0.0;
    // block sums in FP64 (deterministic order)
    __shared__ double red[2][BLOCK_PTS / 32];
    double se = warp_sum(e), sn = warp_sum(w * rho);
    if ((p & 31) == 0) red[0][p >> 5] = se, red[1][p >> 5] = sn;
    __syncthreads();
    if (p == 0) {
        double E = 0.0, N = 0.0;
        for (int q = 0; q < BLOCK_PTS / 32; ++q) E += red[0][q], N += red[1][q];
        blk_sum[2 * blk] = E;
        blk_sum[2 * blk + 1] = N;
    }
}

// The same build in three light kernels: rho and sum grad phi X per point (k_rho_rad, into
// rho_acc), the functional (launch_functional_points), then Z over X (k_z_rad). Each loop over
// the AO components holds few registers, so that enough warps hide the loads of X and of the
// radial sums; k_rho_functional_rad keeps all three in one kernel of 138 registers.
__global__ void __launch_bounds__(BLOCK_PTS, 6) k_rho_rad(BasisView bas, GridView g, int blk0, const char* ws,
                                                       double* rho_acc) {
    __shared__ ShellStage st;
    const int blk = blk0 + blockIdx.x;
    const BlockMeta m = g.meta[blk];
    const int p = threadIdx.x;
    const size_t plane = (size_t)m.nbp * BLOCK_PTS;
    const double* X = reinterpret_cast<const double*>(ws + m.ws) + plane;
    const double* S0p = X + plane;
    const double* S1p = S0p + (size_t)m.nsh * BLOCK_PTS;
    const size_t gp = (size_t)blk * BLOCK_PTS + p;
    const double px = g.px[gp], py = g.py[gp], pz = g.pz[gp];
    double rho = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
    for (int i0 = 0; i0 < m.nsh; i0 += 128) {
        __syncthreads();
        stage_shells(bas, g, m, i0, st);
        __syncthreads();
        const int kn = min(128, m.nsh - i0);
        for (int k = 0; k < kn; ++k) {
            const int i = i0 + k;
            const int L = st.lq[k], row0 = st.row0[k];
            double xv[5];
#pragma unroll
            for (int c = 0; c < 5; ++c) xv[c] = c < 2 * L + 1 ? X[(size_t)(row0 + c) * BLOCK_PTS + p] : 0.0;
            shell_rho<true>(L, px - st.ax[k], py - st.ay[k], pz - st.az[k], S0p[(size_t)i * BLOCK_PTS + p],
                            S1p[(size_t)i * BLOCK_PTS + p], xv, rho, gx, gy, gz);
        }
    }
    double* ra = rho_acc + gp * 4;
    ra[0] = rho, ra[1] = gx, ra[2] = gy, ra[3] = gz;
}

__global__ void __launch_bounds__(BLOCK_PTS, 6) k_z_rad(BasisView bas, GridView g, int blk0, const double* coef,
                                                     char* ws) {
    __shared__ ShellStage st;
    const int blk = blk0 + blockIdx.x;
    const BlockMeta m = g.meta[blk];
    const int p = threadIdx.x;
    const size_t plane = (size_t)m.nbp * BLOCK_PTS;
    double* Z = reinterpret_cast<double*>(ws + m.ws) + plane;
    const double* S0p = Z + plane;
    const double* S1p = S0p + (size_t)m.nsh * BLOCK_PTS;
    const size_t gp = (size_t)blk * BLOCK_PTS + p;
    const double px = g.px[gp], py = g.py[gp], pz = g.pz[gp];
    const double* cf = coef + gp * 4;
    const double a = cf[0], cx = cf[1], cy = cf[2], cz = cf[3];
    double zc[5];
    for (int i0 = 0; i0 < m.nsh; i0 += 128) {
        __syncthreads();
        stage_shells(bas, g, m, i0, st);
        __syncthreads();
        const int kn = min(128, m.nsh - i0);
        for (int k = 0; k < kn; ++k) {
            const int i = i0 + k;
            const int L = st.lq[k], row0 = st.row0[k];
            shell_z(L, px - st.ax[k], py - st.ay[k], pz - st.az[k], S0p[(size_t)i * BLOCK_PTS + p],
                    S1p[(size_t)i * BLOCK_PTS + p], a, cx, cy, cz, zc);
#pragma unroll
            for (int c = 0; c < 5; ++c)
                if (c < 2 * L + 1) Z[(size_t)(row0 + c) * BLOCK_PTS + p] = zc[c];
        }
    }
    for (int r = m.nb; r < m.nbp; ++r) Z[(size_t)r * BLOCK_PTS + p] = 0.0;
}

// Vacc[aos[m]][aos[n]] += sum_p phi[m][p] Z[n][p]: CTA tile 64 x 64 AOs, K = 128 points in
// steps of 16, 4 warps as 2 x 2 warp tiles of 32 x 32 (4 x 4 DMMA tiles). Z was formed by
// k_rho_functional in the place of X; both tiles are staged as [row][k] with 128-byte rows.
constexpr int GV_B = 64, GV_BK = 16, GV_AS = GV_BK + 2;
__global__ void __launch_bounds__(128, 3) k_gemm_v(GridView g, int blk0, char* ws, int zplane, double* Vacc, int nao,
                                                int tiles, int64_t t0) {
    int blk, tm, tn;
    if (g.vtiles) {  // one CTA per tile of the list
        const int2 it = g.vtiles[t0 + blockIdx.x];
        blk = it.x, tm = it.y >> 16, tn = it.y & 0xFFFF;
    } else {
        blk = blk0 + blockIdx.y, tm = blockIdx.x / tiles, tn = blockIdx.x % tiles;
    }
    const BlockMeta m = g.meta[blk];
    const int m0 = tm * GV_B, n0 = tn * GV_B;
    if (m0 >= m.nbp || n0 >= m.nbp) return;
    const double* phi = reinterpret_cast<const double*>(ws + m.ws);
    const double* Z = phi + (size_t)zplane * m.nbp * BLOCK_PTS;
    const int* aos = g.blk_aos + m.ao0;
    __shared__ double As[GV_B * GV_AS];  // [m][k]
    __shared__ double Bs[GV_B * GV_AS];  // [n][k]
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int wm = warp >> 1, wn = warp & 1, gq = lane >> 2, tq = lane & 3;
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    double ra[8], rb[8];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int e = t + q * 128, r = e >> 4, c = e & 15;  // row within tile, point within K step
            ra[q] = phi[(size_t)(m0 + r) * BLOCK_PTS + k0 + c];
            rb[q] = Z[(size_t)(n0 + r) * BLOCK_PTS + k0 + c];
        }
    };
    fetch(0);
    for (int k0 = 0; k0 < BLOCK_PTS; k0 += GV_BK) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int e = t + q * 128, r = e >> 4, c = e & 15;
            As[r * GV_AS + c] = ra[q];
            Bs[r * GV_AS + c] = rb[q];
        }
        __syncthreads();
        if (k0 + GV_BK < BLOCK_PTS) fetch(k0 + GV_BK);
#pragma unroll
        for (int kk = 0; kk < GV_BK; kk += 4) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[(wm * 32 + i * 8 + gq) * GV_AS + kk + tq];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[(wn * 32 + j * 8 + gq) * GV_AS + kk + tq];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = m0 + wm * 32 + i * 8 + gq;
        if (r >= m.nb) continue;
        const size_t rowoff = (size_t)aos[r] * nao;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = n0 + wn * 32 + j * 8 + 2 * tq;
            if (c < m.nb) atomicAdd(&Vacc[rowoff + aos[c]], acc[i][j][0]);
            if (c + 1 < m.nb) atomicAdd(&Vacc[rowoff + aos[c + 1]], acc[i][j][1]);
        }
    }
}

__global__ void k_symmetrize(const double* __restrict__ Vacc, double* V, int nao) {
    const int64_t n2 = (int64_t)nao * nao;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n2; e += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / nao), j = (int)(e % nao);
        V[e] = Vacc[e] + Vacc[(int64_t)j * nao + i];
    }
}

// Open shell (DfCalcGridX::calcRho_{LDA,GGA}_part(P_A, P_B, ...) :1891-1922, :1963-2016, and
// buildVxc(gridMatrix, functional, F_A, F_B) :2093-2135, :2195-2278). One CTA per block,
// one thread per point; X_A and X_B follow the phi planes. A point contributes when
// rho_A or rho_B exceeds the cut-off. Per spin s the Vxc coefficients are the reference's:
// 0.5 w vrho_s and c_s = w (2 vgamma_ss + vgamma_AB) grad rho_s (build_XC_Matrix,
// :2455-2500, is called once per spin with that spin's gradient). Z_s replaces X_s.
template <bool GGA>
__global__ void __launch_bounds__(BLOCK_PTS) k_rho_functional_uks(GridView g, int blk0, int fn, int incremental,
                                                                  double rho_cut, char* ws, double* rho_a,
                                                                  double* rho_b, double* blk_sum, double* blk_sum_b) {
    const int blk = blk0 + blockIdx.x;
    const BlockMeta m = g.meta[blk];
    const int p = threadIdx.x;
    const int nplanes = GGA ? 4 : 1;
    const size_t plane = (size_t)m.nbp * BLOCK_PTS;
    const double* phi = reinterpret_cast<const double*>(ws + m.ws);
    double* XA = const_cast<double*>(phi) + nplanes * plane;
    double* XB = XA + plane;
    double ra = 0.0, ax = 0.0, ay = 0.0, az = 0.0, rb = 0.0, bx = 0.0, by = 0.0, bz = 0.0;
    for (int r = 0; r < m.nb; ++r) {
        const size_t o = (size_t)r * BLOCK_PTS + p;
        const double xa = XA[o], xb = XB[o];
        ra = fma(phi[o], xa, ra);
        rb = fma(phi[o], xb, rb);
        if (GGA) {
            const double dx = phi[plane + o], dy = phi[2 * plane + o], dz = phi[3 * plane + o];
            ax = fma(dx, xa, ax), ay = fma(dy, xa, ay), az = fma(dz, xa, az);
            bx = fma(dx, xb, bx), by = fma(dy, xb, by), bz = fma(dz, xb, bz);
        }
    }
    ax *= 2.0, ay *= 2.0, az *= 2.0, bx *= 2.0, by *= 2.0, bz *= 2.0;
    const size_t gp = (size_t)blk * BLOCK_PTS + p;
    double* sa = rho_a + gp * 4;
    double* sb = rho_b + gp * 4;
    if (incremental) {
        ra += sa[0], ax += sa[1], ay += sa[2], az += sa[3];
        rb += sb[0], bx += sb[1], by += sb[2], bz += sb[3];
    }
    sa[0] = ra, sa[1] = ax, sa[2] = ay, sa[3] = az;
    sb[0] = rb, sb[1] = bx, sb[2] = by, sb[3] = bz;
    const double w = g.pw[gp];
    double e = 0.0, a_a = 0.0, a_b = 0.0, ca[3] = {0.0, 0.0, 0.0}, cb[3] = {0.0, 0.0, 0.0};
    if (w != 0.0 && (ra > rho_cut || rb > rho_cut)) {
        const double gaa = ax * ax + ay * ay + az * az, gbb = bx * bx + by * by + bz * bz;
        const double gab = ax * bx + ay * by + az * bz;
        const XcOut o = eval_functional(fn, ra, rb, gaa, gab, gbb);
        e = w * o.f;
        a_a = 0.5 * w * o.va, a_b = 0.5 * w * o.vb;
        if (GGA) {
            const double cca = w * (2.0 * o.vgaa + o.vgab), ccb = w * (2.0 * o.vgbb + o.vgab);
            ca[0] = cca * ax, ca[1] = cca * ay, ca[2] = cca * az;
            cb[0] = ccb * bx, cb[1] = ccb * by, cb[2] = ccb * bz;
        }
    }
    for (int r = 0; r < m.nbp; ++r) {
        const size_t o = (size_t)r * BLOCK_PTS + p;
        double za = a_a * phi[o], zb = a_b * phi[o];
        if (GGA) {
            const double dx = phi[plane + o], dy = phi[2 * plane + o], dz = phi[3 * plane + o];
            za += ca[0] * dx + ca[1] * dy + ca[2] * dz;
            zb += cb[0] * dx + cb[1] * dy + cb[2] * dz;
        }
        XA[o] = za, XB[o] = zb;
    }
    __shared__ double red[3][BLOCK_PTS / 32];
    const double se = warp_sum(e), sna = warp_sum(w * ra), snb = warp_sum(w * rb);
    if ((p & 31) == 0) red[0][p >> 5] = se, red[1][p >> 5] = sna, red[2][p >> 5] = snb;
    __syncthreads();
    if (p == 0) {
        double E = 0.0, NA = 0.0, NB = 0.0;
        for (int i = 0; i < BLOCK_PTS / 32; ++i) E += red[0][i], NA += red[1][i], NB += red[2][i];
        blk_sum[2 * blk] = E;
        blk_sum[2 * blk + 1] = NA;
        blk_sum_b[2 * blk] = NB;
        blk_sum_b[2 * blk + 1] = 0.0;
    }
}

// Deterministic FP64 sum of the per-block partials: one CTA, fixed order.
__global__ void k_block_sums(const double* __restrict__ blk_sum, int nblk, double* out) {
    __shared__ double se[256], sn[256];
    double e = 0.0, n = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) e += blk_sum[2 * b], n += blk_sum[2 * b + 1];
    se[threadIdx.x] = e, sn[threadIdx.x] = n;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) se[threadIdx.x] += se[threadIdx.x + s], sn[threadIdx.x] += sn[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = se[0], out[1] = sn[0];
}

// Per-segment (per-molecule of a batch) FP64 sums of the block partials: one CTA per
// segment, blocks [seg_blk[i], seg_blk[i+1]), the same fixed order as k_block_sums.
__global__ void k_segment_sums(const double* __restrict__ blk_sum, const int* __restrict__ seg_blk, double* out) {
    __shared__ double se[256], sn[256];
    const int b0 = seg_blk[blockIdx.x], b1 = seg_blk[blockIdx.x + 1];
    double e = 0.0, n = 0.0;
    for (int b = b0 + threadIdx.x; b < b1; b += blockDim.x) e += blk_sum[2 * b], n += blk_sum[2 * b + 1];
    se[threadIdx.x] = e, sn[threadIdx.x] = n;
    __syncthreads();
    for (int st = blockDim.x / 2; st > 0; st >>= 1) {
        if (threadIdx.x < st) se[threadIdx.x] += se[threadIdx.x + st], sn[threadIdx.x] += sn[threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[2 * blockIdx.x] = se[0], out[2 * blockIdx.x + 1] = sn[0];
}

}  // namespace

void launch_segment_sums(const double* blk_sum, const int* seg_blk, int nseg, double* out, cudaStream_t s) {
    k_segment_sums<<<nseg, 256, 0, s>>>(blk_sum, seg_blk, out);
}

void launch_ao_eval(const BasisView& b, const GridView& g, int blk0, int nblk, bool gga, char* ws,
                    int /*max_nsh*/, cudaStream_t s) {
    if (gga)
        k_ao_eval<true><<<nblk, 256, 0, s>>>(b, g, blk0, ws);
    else
        k_ao_eval<false><<<nblk, 256, 0, s>>>(b, g, blk0, ws);
}

void launch_gemm_x(const GridView& g, const double* P, int nao, int blk0, int nblk, int max_nbp,
                          int nplanes, char* ws, cudaStream_t s) {
    // X follows the phi planes (1 for LDA, 4 with gradients)
    launch_gemm_x_planes(g, P, nao, blk0, nblk, max_nbp, 0, nplanes, 1, ws, s);
}

void launch_gemm_x_planes(const GridView& g, const double* P, int nao, int blk0, int nblk, int max_nbp, int src0,
                          int dst0, int nz, char* ws, cudaStream_t s) {
    if (g.xtiles && g.h_xtile0) {
        const int64_t t0 = g.h_xtile0[blk0], n = g.h_xtile0[blk0 + nblk] - t0;
        if (n > 0) k_gemm_x<<<dim3((unsigned)n, 1, nz), 256, 0, s>>>(g, P, nao, blk0, ws, src0, dst0, t0);
        return;
    }
    dim3 grid((max_nbp + GX_BM - 1) / GX_BM, nblk, nz);
    k_gemm_x<<<grid, 256, 0, s>>>(g, P, nao, blk0, ws, src0, dst0, 0);
}

void launch_ao_eval_rad(const BasisView& b, const GridView& g, int blk0, int nblk, char* ws, cudaStream_t s) {
    k_ao_eval_rad<<<nblk, 256, 0, s>>>(b, g, blk0, ws);
}

void launch_rho_functional_rad(const BasisView& b, const GridView& g, int blk0, int nblk, int fn, bool incremental,
                               double rho_cut, char* ws, double* rho, double* coef, double* blk_sum, cudaStream_t s) {
    k_rho_functional_rad<<<nblk, BLOCK_PTS, 0, s>>>(b, g, blk0, fn, incremental, rho_cut, ws, rho, coef, blk_sum);
}

void launch_rho_rad(const BasisView& b, const GridView& g, int blk0, int nblk, const char* ws, double* rho_acc,
                    cudaStream_t s) {
    k_rho_rad<<<nblk, BLOCK_PTS, 0, s>>>(b, g, blk0, ws, rho_acc);
}

void launch_z_rad(const BasisView& b, const GridView& g, int blk0, int nblk, const double* coef, char* ws,
                  cudaStream_t s) {
    k_z_rad<<<nblk, BLOCK_PTS, 0, s>>>(b, g, blk0, coef, ws);
}

void launch_rho_functional(const GridView& g, int blk0, int nblk, int fn, bool incremental, double rho_cut,
                           char* ws, double* rho, double* coef, double* blk_sum, cudaStream_t s) {
    if (functional_is_gga(fn))
        k_rho_functional<true><<<nblk, BLOCK_PTS, 0, s>>>(g, blk0, fn, incremental, rho_cut, ws, rho, coef, blk_sum);
    else
        k_rho_functional<false><<<nblk, BLOCK_PTS, 0, s>>>(g, blk0, fn, incremental, rho_cut, ws, rho, coef, blk_sum);
}

void launch_gemm_v(const GridView& g, int blk0, int nblk, int max_nbp, bool gga, const double* coef, char* ws,
                   double* Vacc, int nao, cudaStream_t s) {
    (void)coef;
    launch_gemm_v_plane(g, blk0, nblk, max_nbp, gga ? 4 : 1, ws, Vacc, nao, s);
}

void launch_gemm_v_plane(const GridView& g, int blk0, int nblk, int max_nbp, int zplane, char* ws, double* Vacc,
                         int nao, cudaStream_t s) {
    const int tiles = (max_nbp + GV_B - 1) / GV_B;
    if (g.vtiles && g.h_vtile0) {
        const int64_t t0 = g.h_vtile0[blk0], n = g.h_vtile0[blk0 + nblk] - t0;
        if (n > 0) k_gemm_v<<<(unsigned)n, 128, 0, s>>>(g, blk0, ws, zplane, Vacc, nao, tiles, t0);
        return;
    }
    dim3 grid(tiles * tiles, nblk);
    k_gemm_v<<<grid, 128, 0, s>>>(g, blk0, ws, zplane, Vacc, nao, tiles, 0);
}

void launch_rho_functional_uks(const GridView& g, int blk0, int nblk, int fn, bool incremental, double rho_cut,
                               char* ws, double* rho_a, double* rho_b, double* blk_sum, double* blk_sum_b,
                               cudaStream_t s) {
    if (functional_is_gga(fn))
        k_rho_functional_uks<true><<<nblk, BLOCK_PTS, 0, s>>>(g, blk0, fn, incremental, rho_cut, ws, rho_a, rho_b,
                                                               blk_sum, blk_sum_b);
    else
        k_rho_functional_uks<false><<<nblk, BLOCK_PTS, 0, s>>>(g, blk0, fn, incremental, rho_cut, ws, rho_a, rho_b,
                                                                blk_sum, blk_sum_b);
}

void launch_block_sums(const double* blk_sum, int nblk, double* scalars, cudaStream_t s) {
    k_block_sums<<<1, 256, 0, s>>>(blk_sum, nblk, scalars);
}

// dV = V - Vprev (or V with no previous iteration), then Vprev = V: the XC part of
// DfFockMatrix::setXC_DIRECT (src/libpdf/DfFockMatrix.h:711-721) on the device.
__global__ void k_fock_delta(const double* __restrict__ V, double* Vprev, double* __restrict__ dV, size_t n,
                             int has_prev) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double v = V[i];
        dV[i] = has_prev ? v - Vprev[i] : v;
        Vprev[i] = v;
    }
}

void launch_fock_delta(const double* V, double* Vprev, double* dV, size_t n, bool has_prev, cudaStream_t s) {
    k_fock_delta<<<148 * 8, 256, 0, s>>>(V, Vprev, dV, n, has_prev ? 1 : 0);
}

// The upper triangle of a symmetric n x n matrix packed row by row: (i, j >= i) at
// i n - i (i - 1) / 2 + (j - i). One CTA per row; the reads and writes along j are coalesced.
__global__ void k_pack_upper(const double* __restrict__ V, int n, double* __restrict__ packed) {
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const int64_t o = (int64_t)i * n - (int64_t)i * (i - 1) / 2 - i;
        for (int j = i + threadIdx.x; j < n; j += blockDim.x) packed[o + j] = V[(int64_t)i * n + j];
    }
}

// Both triangles from the packed upper triangle, in 32 x 32 tiles: a tile on or above the
// diagonal copies packed rows; a tile below it reads its mirror tile's packed rows (coalesced)
// into shared memory and writes the transpose.
__global__ void k_unpack_upper(const double* __restrict__ packed, int n, double* __restrict__ V) {
    __shared__ double t[32][33];
    const int nt = (n + 31) / 32;
    for (int64_t tile = blockIdx.x; tile < (int64_t)nt * nt; tile += gridDim.x) {
        const int ti = (int)(tile / nt), tj = (int)(tile % nt);
        const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
        if (ti <= tj) {
            for (int r = ty; r < 32; r += 8) {
                const int i = ti * 32 + r, j = tj * 32 + tx;
                if (i < n && j < n) {
                    const int a = min(i, j), b = max(i, j);
                    V[(int64_t)i * n + j] = packed[(int64_t)a * n - (int64_t)a * (a - 1) / 2 + (b - a)];
                }
            }
        } else {
            // rows tj*32.. of the mirror tile (row index < column index: the packed upper part)
            for (int r = ty; r < 32; r += 8) {
                const int a = tj * 32 + r, b = ti * 32 + tx;
                if (a < n && b < n) t[r][tx] = packed[(int64_t)a * n - (int64_t)a * (a - 1) / 2 + (b - a)];
            }
            __syncthreads();
            for (int r = ty; r < 32; r += 8) {
                const int i = ti * 32 + r, j = tj * 32 + tx;
                if (i < n && j < n) V[(int64_t)i * n + j] = t[tx][r];
            }
            __syncthreads();
        }
    }
}

void launch_pack_upper(const double* V, int n, double* packed, cudaStream_t s) {
    k_pack_upper<<<148 * 8, 256, 0, s>>>(V, n, packed);
}

void launch_unpack_upper(const double* packed, int n, double* V, cudaStream_t s) {
    k_unpack_upper<<<148 * 8, 256, 0, s>>>(packed, n, V);
}

void launch_finish(const double* Vacc, double* V, int nao, const double* blk_sum, int nblk, double* scalars,
                   cudaStream_t s) {
    k_symmetrize<<<148 * 8, 256, 0, s>>>(Vacc, V, nao);
    k_block_sums<<<1, 256, 0, s>>>(blk_sum, nblk, scalars);
}

}  // namespace pdfxc
