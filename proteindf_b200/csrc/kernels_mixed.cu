// Mixed-precision XC build: the two contractions on tcgen05 tensor cores with
// split-BF16 operands (v = hi + mid [+ lo], each BF16) and FP32 accumulation in
// TMEM; AO values, weights, the functional, the per-block Exc / electron-count
// sums and the Vxc accumulation stay in FP64.
//
// Per block (128 points, nb screened AOs padded to nbp = 128k):
//   ao_mixed    phi, grad phi in FP64 -> FP32 copies (epilogue operands) and
//               split-BF16 packed operands phi^T (rows = points, K = AOs) and
//               phi (rows = AOs, K = points)
//   pack_p      P_sub = P_A[aos, aos] as split-BF16 packed (rows = mu, K = nu)
//   umma<RHO>   X^T = phi^T P_sub  (M = 128 points, N = 128 AOs per CTA, K = nbp);
//               epilogue: rho(p) += sum_mu phi[mu][p] X^T[p][mu] and the
//               gradient sums, FP64 atomics per point
//   functional  rho -> Exc partials, 0.5 w vrho, c = w (2 vgAA + vgAB) grad rho
//   pack_z      Z[nu][p] = 0.5 w vrho phi + c . grad phi, split-BF16 packed
//   umma<VXC>   W = phi Z^T (M = N = 128 AOs per CTA, K = 128 points);
//               epilogue: Vacc[aos, aos] += W in FP64
// The split product keeps the terms hi*hi + hi*mid + mid*hi (3 terms) or, with
// the three-way split, all terms of order <= 2^-24 (6 terms).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "ao.cuh"
#include "functional.cuh"
#include "pdfxc_internal.cuh"
#include "umma.cuh"

namespace pdfxc {

namespace {

using umma::packed_offset;

__device__ __forceinline__ void split3(double v, __nv_bfloat16& h, __nv_bfloat16& m, __nv_bfloat16& l) {
    h = __double2bfloat16(v);
    const double r1 = v - (double)__bfloat162float(h);
    m = __double2bfloat16(r1);
    const double r2 = r1 - (double)__bfloat162float(m);
    l = __double2bfloat16(r2);
}

__device__ __forceinline__ void ang_factor_m(int t, double x, double y, double z, double a2, double& v, double& dx,
                                             double& dy, double& dz) {
    const double s3 = 0.57735026918962576451;
    switch (t) {
        case 0: v = 1.0; dx = -a2 * x; dy = -a2 * y; dz = -a2 * z; break;
        case 1: v = x; dx = -a2 * x * x + 1.0; dy = -a2 * x * y; dz = -a2 * x * z; break;
        case 2: v = y; dx = -a2 * y * x; dy = -a2 * y * y + 1.0; dz = -a2 * y * z; break;
        case 3: v = z; dx = -a2 * z * x; dy = -a2 * z * y; dz = -a2 * z * z + 1.0; break;
        case 4: v = x * y; dx = -a2 * x * y * x + y; dy = -a2 * x * y * y + x; dz = -a2 * x * y * z; break;
        case 5: v = z * x; dx = -a2 * x * z * x + z; dy = -a2 * x * z * y; dz = -a2 * x * z * z + x; break;
        case 6: v = y * z; dx = -a2 * y * z * x; dy = -a2 * y * z * y + z; dz = -a2 * y * z * z + y; break;
        case 7:
            v = 0.5 * (x * x - y * y);
            dx = 0.5 * ((-a2 * x * x * x + 2.0 * x) - (-a2 * y * y * x));
            dy = 0.5 * ((-a2 * x * x * y) - (-a2 * y * y * y + 2.0 * y));
            dz = 0.5 * ((-a2 * x * x * z) - (-a2 * y * y * z));
            break;
        default: {
            v = s3 * (z * z - 0.5 * (x * x + y * y));
            const double xxX = -a2 * x * x * x + 2.0 * x, xxY = -a2 * x * x * y, xxZ = -a2 * x * x * z;
            const double yyX = -a2 * y * y * x, yyY = -a2 * y * y * y + 2.0 * y, yyZ = -a2 * y * y * z;
            const double zzX = -a2 * z * z * x, zzY = -a2 * z * z * y, zzZ = -a2 * z * z * z + 2.0 * z;
            dx = s3 * (zzX - 0.5 * (xxX + yyX));
            dy = s3 * (zzY - 0.5 * (xxY + yyY));
            dz = s3 * (zzZ - 0.5 * (xxZ + yyZ));
        }
    }
}

__device__ __forceinline__ void store_split(char* base, size_t plane, size_t off, double v) {
    __nv_bfloat16 h, m, l;
    split3(v, h, m, l);
    *reinterpret_cast<__nv_bfloat16*>(base + off) = h;
    *reinterpret_cast<__nv_bfloat16*>(base + plane + off) = m;
    *reinterpret_cast<__nv_bfloat16*>(base + 2 * plane + off) = l;
}

// AO values for one block. 256 threads: point = tid % 128, halves take alternate shells.
template <bool GGA>
__global__ void __launch_bounds__(256) k_ao_mixed(BasisView bas, GridView g, int blk0, char* ws) {
    const int blk = blk0 + blockIdx.x;
    const BlockMeta m = g.meta[blk];
    const MixedLayout L = mixed_layout(m.nbp);
    char* base = ws + m.ws;
    float* phi32 = reinterpret_cast<float*>(base + L.phi32);
    char* phi1 = base + L.phi1;
    char* phi2 = base + L.phi2;
    const size_t plane32 = (size_t)m.nbp * BLOCK_PTS;
    const int p = threadIdx.x & (BLOCK_PTS - 1);
    const int half = threadIdx.x >> 7;
    const int gp = blk * BLOCK_PTS + p;
    const double rx = g.px[gp], ry = g.py[gp], rz = g.pz[gp];
    for (int i = half; i < m.nsh; i += 2) {
        const int s = g.blk_shells[m.sh0 + i];
        const int row0 = g.blk_shell_row[m.sh0 + i];
        const int a = bas.sh_atom[s];
        const double x = rx - bas.atom_xyz[3 * a], y = ry - bas.atom_xyz[3 * a + 1], z = rz - bas.atom_xyz[3 * a + 2];
        const double d2 = x * x + y * y + z * z;
        const int Lq = bas.sh_l[s], n = 2 * Lq + 1, np = bas.sh_nprim[s], p0 = bas.sh_p0[s];
        for (int c = 0; c < n; ++c) {
            double v = 0, gx = 0, gy = 0, gz = 0;
            for (int k = 0; k < np; ++k) {
                const double al = bas.p_exp[p0 + k];
                if (al * d2 <= 30.0) {
                    const double e = bas.p_coef[p0 + k] * exp(-al * d2);
                    double av, ax, ay, az;
                    ang_factor_m(Lq * Lq + c, x, y, z, 2.0 * al, av, ax, ay, az);
                    v += av * e;
                    if (GGA) gx += ax * e, gy += ay * e, gz += az * e;
                }
            }
            const int mu = row0 + c;
            const size_t o = (size_t)mu * BLOCK_PTS + p;
            phi32[o] = (float)v;
            if (GGA) {
                phi32[plane32 + o] = (float)gx;
                phi32[2 * plane32 + o] = (float)gy;
                phi32[3 * plane32 + o] = (float)gz;
            }
            store_split(phi1, L.phi1_plane, packed_offset(p, mu, m.nbp), v);
            store_split(phi2, L.phi2_plane, packed_offset(mu, p, BLOCK_PTS), v);
        }
    }
    for (int mu = m.nb + half; mu < m.nbp; mu += 2) {
        const size_t o = (size_t)mu * BLOCK_PTS + p;
        phi32[o] = 0.f;
        if (GGA) phi32[plane32 + o] = phi32[2 * plane32 + o] = phi32[3 * plane32 + o] = 0.f;
        store_split(phi1, L.phi1_plane, packed_offset(p, mu, m.nbp), 0.0);
        store_split(phi2, L.phi2_plane, packed_offset(mu, p, BLOCK_PTS), 0.0);
    }
}

// P_sub of one block, split and packed; thread = (row mu, 8 consecutive nu) -> 16-byte stores.
__global__ void __launch_bounds__(256) k_pack_p(GridView g, const double* __restrict__ P, int nao, int blk0, char* ws) {
    const int blk = blk0 + blockIdx.x;
    const BlockMeta m = g.meta[blk];
    const MixedLayout L = mixed_layout(m.nbp);
    char* pp = ws + m.ws + L.ppack;
    const int* aos = g.blk_aos + m.ao0;
    const int groups = m.nbp / 8;
    for (int e = threadIdx.x; e < m.nbp * groups; e += blockDim.x) {
        const int mu = e / groups, nu0 = (e % groups) * 8;
        __align__(16) __nv_bfloat16 h[8], md[8], lo[8];
        const size_t row = mu < m.nb ? (size_t)aos[mu] * nao : 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int nu = nu0 + j;
            const double v = (mu < m.nb && nu < m.nb) ? P[row + aos[nu]] : 0.0;
            split3(v, h[j], md[j], lo[j]);
        }
        const size_t off = packed_offset(mu, nu0, m.nbp);
        *reinterpret_cast<uint4*>(pp + off) = *reinterpret_cast<uint4*>(h);
        *reinterpret_cast<uint4*>(pp + L.ppack_plane + off) = *reinterpret_cast<uint4*>(md);
        *reinterpret_cast<uint4*>(pp + 2 * L.ppack_plane + off) = *reinterpret_cast<uint4*>(lo);
    }
}

__device__ __forceinline__ double warp_sum_m(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// rho accumulators -> functional -> Vxc coefficients, per point (128 threads per block).
template <bool GGA>
__global__ void __launch_bounds__(BLOCK_PTS) k_functional_mixed(GridView g, int blk0, int fn, int incremental,
                                                                double rho_cut, const double* rho_acc,
                                                                double* rho_store, double* coef, double* blk_sum) {
    const int blk = blk0 + blockIdx.x;
    const int p = threadIdx.x;
    const size_t gp = (size_t)blk * BLOCK_PTS + p;
    const double* ra = rho_acc + gp * 4;
    double rho = ra[0], gx = 2.0 * ra[1], gy = 2.0 * ra[2], gz = 2.0 * ra[3];
    double* rs = rho_store + gp * 4;
    if (incremental) rho += rs[0], gx += rs[1], gy += rs[2], gz += rs[3];
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
    __shared__ double red[2][BLOCK_PTS / 32];
    const double se = warp_sum_m(e), sn = warp_sum_m(w * rho);
    if ((p & 31) == 0) red[0][p >> 5] = se, red[1][p >> 5] = sn;
    __syncthreads();
    if (p == 0) {
        double E = 0.0, N = 0.0;
        for (int i = 0; i < BLOCK_PTS / 32; ++i) E += red[0][i], N += red[1][i];
        blk_sum[2 * blk] = E, blk_sum[2 * blk + 1] = N;
    }
}

// The open shell (DfCalcGridX::calcRho_*_part(P_A, P_B, ...) and buildVxc(gridMatrix, functional,
// F_A, F_B), src/libpdf/DfCalcGridX.cpp:1891-1922, :1963-2016, :2093-2135, :2195-2278): both
// spins' rho accumulators -> the open-shell functional -> each spin's Vxc coefficients
// (0.5 w vrho_s and c_s = w (2 vgamma_ss + vgamma_AB) grad rho_s, as the FP64 open-shell
// kernel); a point contributes when rho_A or rho_B exceeds the cut-off.
template <bool GGA>
__global__ void __launch_bounds__(BLOCK_PTS) k_functional_mixed_uks(GridView g, int blk0, int fn, int incremental,
                                                                    double rho_cut, const double* rho_acc_a,
                                                                    const double* rho_acc_b, double* rho_store_a,
                                                                    double* rho_store_b, double* coef_a, double* coef_b,
                                                                    double* blk_sum, double* blk_sum_b) {
    const int blk = blk0 + blockIdx.x;
    const int p = threadIdx.x;
    const size_t gp = (size_t)blk * BLOCK_PTS + p;
    double d[2][4];
    const double* acc[2] = {rho_acc_a + gp * 4, rho_acc_b + gp * 4};
    double* st[2] = {rho_store_a + gp * 4, rho_store_b + gp * 4};
#pragma unroll
    for (int sp = 0; sp < 2; ++sp) {
        d[sp][0] = acc[sp][0], d[sp][1] = 2.0 * acc[sp][1], d[sp][2] = 2.0 * acc[sp][2], d[sp][3] = 2.0 * acc[sp][3];
        if (incremental)
            for (int k = 0; k < 4; ++k) d[sp][k] += st[sp][k];
        for (int k = 0; k < 4; ++k) st[sp][k] = d[sp][k];
    }
    const double w = g.pw[gp];
    const double ra = d[0][0], rb = d[1][0];
    double e = 0.0, a_a = 0.0, a_b = 0.0, ca[3] = {0.0, 0.0, 0.0}, cb[3] = {0.0, 0.0, 0.0};
    if (w != 0.0 && (ra > rho_cut || rb > rho_cut)) {
        const double gaa = d[0][1] * d[0][1] + d[0][2] * d[0][2] + d[0][3] * d[0][3];
        const double gbb = d[1][1] * d[1][1] + d[1][2] * d[1][2] + d[1][3] * d[1][3];
        const double gab = d[0][1] * d[1][1] + d[0][2] * d[1][2] + d[0][3] * d[1][3];
        const XcOut o = eval_functional(fn, ra, rb, gaa, gab, gbb);
        e = w * o.f;
        a_a = 0.5 * w * o.va, a_b = 0.5 * w * o.vb;
        if (GGA) {
            const double cca = w * (2.0 * o.vgaa + o.vgab), ccb = w * (2.0 * o.vgbb + o.vgab);
            for (int k = 0; k < 3; ++k) ca[k] = cca * d[0][1 + k], cb[k] = ccb * d[1][1 + k];
        }
    }
    double* fa = coef_a + gp * 4;
    double* fb = coef_b + gp * 4;
    fa[0] = a_a, fa[1] = ca[0], fa[2] = ca[1], fa[3] = ca[2];
    fb[0] = a_b, fb[1] = cb[0], fb[2] = cb[1], fb[3] = cb[2];
    __shared__ double red[3][BLOCK_PTS / 32];
    const double se = warp_sum_m(e), sna = warp_sum_m(w * ra), snb = warp_sum_m(w * rb);
    if ((p & 31) == 0) red[0][p >> 5] = se, red[1][p >> 5] = sna, red[2][p >> 5] = snb;
    __syncthreads();
    if (p == 0) {
        double E = 0.0, NA = 0.0, NB = 0.0;
        for (int i = 0; i < BLOCK_PTS / 32; ++i) E += red[0][i], NA += red[1][i], NB += red[2][i];
        blk_sum[2 * blk] = E, blk_sum[2 * blk + 1] = NA;
        blk_sum_b[2 * blk] = NB, blk_sum_b[2 * blk + 1] = 0.0;
    }
}

// Z[nu][p] = 0.5 w vrho phi + c . grad phi, split and packed (rows = AOs, K = points).
template <bool GGA>
__global__ void __launch_bounds__(256) k_pack_z(GridView g, int blk0, const double* __restrict__ coef, char* ws) {
    const int blk = blk0 + blockIdx.x;
    const BlockMeta m = g.meta[blk];
    const MixedLayout L = mixed_layout(m.nbp);
    const float* phi32 = reinterpret_cast<const float*>(ws + m.ws + L.phi32);
    char* zp = ws + m.ws + L.zpack;
    const size_t plane32 = (size_t)m.nbp * BLOCK_PTS;
    __shared__ double cf[4][BLOCK_PTS];
    for (int e = threadIdx.x; e < 4 * BLOCK_PTS; e += blockDim.x)
        cf[e & 3][e >> 2] = coef[((size_t)blk * BLOCK_PTS + (e >> 2)) * 4 + (e & 3)];
    __syncthreads();
    const int groups = BLOCK_PTS / 8;
    for (int e = threadIdx.x; e < m.nbp * groups; e += blockDim.x) {
        const int nu = e / groups, p0 = (e % groups) * 8;
        __align__(16) __nv_bfloat16 h[8], md[8], lo[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int p = p0 + j;
            const size_t o = (size_t)nu * BLOCK_PTS + p;
            double z = cf[0][p] * (double)phi32[o];
            if (GGA)
                z += cf[1][p] * (double)phi32[plane32 + o] + cf[2][p] * (double)phi32[2 * plane32 + o] +
                     cf[3][p] * (double)phi32[3 * plane32 + o];
            split3(z, h[j], md[j], lo[j]);
        }
        const size_t off = packed_offset(nu, p0, BLOCK_PTS);
        *reinterpret_cast<uint4*>(zp + off) = *reinterpret_cast<uint4*>(h);
        *reinterpret_cast<uint4*>(zp + L.zpack_plane + off) = *reinterpret_cast<uint4*>(md);
        *reinterpret_cast<uint4*>(zp + 2 * L.zpack_plane + off) = *reinterpret_cast<uint4*>(lo);
    }
}

// ---------------------------------------------------------------------------
// The tcgen05 contraction. One CTA (4 warps) computes one 128 x 128 FP32 tile
// D = sum_terms A_i B_j^T over K in 64-wide slabs: warp 0 / lane 0 streams the
// slabs of the needed split planes into a ring of shared-memory stages with
// cp.async.bulk, warp 1 / lane 0 issues tcgen05.mma (M = 128, N = 128, K = 16)
// into a 128-column TMEM accumulator, and all four warps run the epilogue on
// their 32 TMEM lanes. Every wait is bounded; on expiry an error code is
// recorded in *err and the CTA winds down (waiting, bounded, for its issued
// MMAs) before freeing TMEM.
enum { MODE_RHO = 0, MODE_VXC = 1 };

struct UmmaParams {
    int nterms;    // 3 or 6
    int stages;    // ring depth
    int* err;      // device error word
    const double* dummy;
};

__constant__ int kTermA[6] = {0, 0, 1, 0, 1, 2};
__constant__ int kTermB[6] = {0, 1, 0, 2, 1, 0};

template <int MODE, bool GGA>
__global__ void __launch_bounds__(128, 1)
    k_umma(GridView g, int blk0, char* ws, UmmaParams prm, int tiles_max, double* rho_acc, double* Vacc, int nao) {
    extern __shared__ __align__(1024) uint8_t smem[];
    const int blk = blk0 + blockIdx.y;
    const BlockMeta m = g.meta[blk];
    const MixedLayout L = mixed_layout(m.nbp);
    const int ntiles = m.nbp / umma::TILE_ROWS;
    int mt, nt;
    if (MODE == MODE_RHO) {
        mt = 0, nt = blockIdx.x;
        if (nt >= ntiles) return;
    } else {
        mt = blockIdx.x / tiles_max, nt = blockIdx.x % tiles_max;
        if (mt >= ntiles || nt >= ntiles) return;
    }
    // once any CTA has recorded an expired wait, the rest of the grid exits at once
    __shared__ int s_abort;
    if (threadIdx.x == 0) s_abort = *reinterpret_cast<const volatile int*>(prm.err);
    __syncthreads();
    if (s_abort) return;
    const int nA = prm.nterms == 3 ? 2 : 3, nB = nA;
    const int S = prm.stages;
    const uint32_t stage_bytes = (uint32_t)(nA + nB) * umma::SLAB_BYTES;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * stage_bytes);
    uint64_t* empty = full + S;
    uint64_t* done = empty + S;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);

    // operands of this tile
    const char* base = ws + m.ws;
    const char *Ab, *Bb;
    size_t Aplane, Bplane;
    int nslabs;
    if (MODE == MODE_RHO) {
        Ab = base + L.phi1;  // rows = 128 points, K = nbp
        Aplane = L.phi1_plane;
        Bb = base + L.ppack + (size_t)nt * umma::TILE_ROWS * m.nbp * 2;  // rows = mu tile, K = nbp
        Bplane = L.ppack_plane;
        nslabs = m.nbp / umma::SLAB_K;
    } else {
        Ab = base + L.phi2 + (size_t)mt * umma::TILE_ROWS * BLOCK_PTS * 2;  // rows = mu tile, K = 128 points
        Aplane = L.phi2_plane;
        Bb = base + L.zpack + (size_t)nt * umma::TILE_ROWS * BLOCK_PTS * 2;
        Bplane = L.zpack_plane;
        nslabs = BLOCK_PTS / umma::SLAB_K;
    }

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) umma::tmem_alloc(tslot, 128);
    if (threadIdx.x == 32) {
        for (int s = 0; s < S; ++s) umma::mbar_init(&full[s], 1), umma::mbar_init(&empty[s], 1);
        umma::mbar_init(done, 1);
        umma::mbar_init_fence();
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tslot;
    bool ok = true;

    if (warp == 0 && lane == 0) {  // producer
        for (int j = 0; j < nslabs && ok; ++j) {
            const int s = j % S;
            if (j >= S && !umma::mbar_wait(&empty[s], ((j / S) - 1) & 1, prm.err)) {
                ok = false;
                atomicExch(prm.err, 1);
                break;
            }
            uint8_t* st = smem + s * stage_bytes;
            umma::mbar_expect_tx(&full[s], stage_bytes);
            for (int a = 0; a < nA; ++a)
                umma::bulk_g2s(st + a * umma::SLAB_BYTES, Ab + a * Aplane + (size_t)j * umma::SLAB_BYTES,
                               umma::SLAB_BYTES, &full[s]);
            for (int b = 0; b < nB; ++b)
                umma::bulk_g2s(st + (nA + b) * umma::SLAB_BYTES, Bb + b * Bplane + (size_t)j * umma::SLAB_BYTES,
                               umma::SLAB_BYTES, &full[s]);
        }
    } else if (warp == 1 && lane == 0) {  // MMA issuer
        const uint32_t idesc = umma::instr_desc_bf16(128, 128);
        bool issued = false;
        for (int j = 0; j < nslabs; ++j) {
            const int s = j % S;
            if (!umma::mbar_wait(&full[s], (j / S) & 1, prm.err)) {
                ok = false;
                atomicExch(prm.err, 2);
                break;
            }
            umma::fence_after_sync();
            const uint32_t st = umma::smem_u32(smem + s * stage_bytes);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                for (int t = 0; t < prm.nterms; ++t) {
                    const uint64_t ad = umma::smem_desc(st + kTermA[t] * umma::SLAB_BYTES + kk * 4096, umma::LBO, umma::SBO);
                    const uint64_t bd =
                        umma::smem_desc(st + (nA + kTermB[t]) * umma::SLAB_BYTES + kk * 4096, umma::LBO, umma::SBO);
                    umma::mma_bf16(tmem, ad, bd, idesc, (j > 0 || kk > 0 || t > 0) ? 1u : 0u);
                }
            }
            issued = true;
            umma::mma_commit(&empty[s]);
        }
        if (issued) umma::mma_commit(done);
        else umma::mbar_expect_tx(done, 0);  // nothing issued: complete the phase ourselves
    }
    __syncwarp();
    bool waited = umma::mbar_wait(done, 0, prm.err);
    if (!waited) atomicExch(prm.err, 3);
    // one decision for the whole CTA: the epilogue below has CTA-wide barriers
    const bool ready = __syncthreads_and(waited) != 0;
    umma::fence_after_sync();

    if (ready) {
        const int row = warp * 32 + lane;
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
        if (MODE == MODE_RHO) {
            const float* phi32 = reinterpret_cast<const float*>(base + L.phi32);
            const size_t plane32 = (size_t)m.nbp * BLOCK_PTS;
            double r = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
            for (int c0 = 0; c0 < 128; c0 += 16) {
                float v[16];
                umma::tmem_ld16(taddr + c0, v);
#pragma unroll
                for (int c = 0; c < 16; ++c) {
                    const int mu = nt * 128 + c0 + c;
                    if (mu >= m.nb) break;
                    const size_t o = (size_t)mu * BLOCK_PTS + row;
                    const double x = v[c];
                    r += (double)phi32[o] * x;
                    if (GGA) {
                        gx += (double)phi32[plane32 + o] * x;
                        gy += (double)phi32[2 * plane32 + o] * x;
                        gz += (double)phi32[3 * plane32 + o] * x;
                    }
                }
            }
            double* acc = rho_acc + ((size_t)blk * BLOCK_PTS + row) * 4;
            atomicAdd(acc, r);
            if (GGA) atomicAdd(acc + 1, gx), atomicAdd(acc + 2, gy), atomicAdd(acc + 3, gz);
        } else {
            // stage 16 columns of all 128 rows in shared memory, then let each warp
            // add two rows x 16 consecutive columns per instruction
            float* tile = reinterpret_cast<float*>(smem);  // [128][17]
            const int* aos = g.blk_aos + m.ao0;
            for (int c0 = 0; c0 < 128; c0 += 16) {
                float v[16];
                umma::tmem_ld16(taddr + c0, v);
#pragma unroll
                for (int c = 0; c < 16; ++c) tile[row * 17 + c] = v[c];
                __syncthreads();
                const int c = threadIdx.x & 15;
                const int nu = nt * 128 + c0 + c;
                if (nu < m.nb) {
                    const int anu = aos[nu];
                    for (int rr = threadIdx.x >> 4; rr < 128; rr += 8) {
                        const int mu = mt * 128 + rr;
                        if (mu < m.nb) atomicAdd(&Vacc[(size_t)aos[mu] * nao + anu], (double)tile[rr * 17 + c]);
                    }
                }
                __syncthreads();
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, 128);
}

// ===========================================================================
// Fixed-point slices on the INT8 tensor cores (the split-integer product of
// Ozaki, Ogita, Oishi and Rump, 2012, on an integer unit). Each operand row
// gets a power-of-two scale 2^e with |v| < 2^e and four signed digits in [-128, 127]:
// v = 2^e (s_1 + s_2 / 256 + s_3 / 256^2 + s_4 / 256^3) / 127, the balanced base-256
// expansion of v rounded to 127 256^3 units of 2^e: about 31 bits per operand. The
// digits of q = rint(v 127 256^3 2^-e) are the bytes of q + 0x80808080 with their top
// bits flipped, two integer operations per value. Their mean is -1/2, so the dropped
// low-order products carry a bias, but it is about 1e-3 of their random part (a CPU
// emulation of the chain12 quadrature: mean / rms of the error of X 0.002, the same as
// for the symmetric base-255 digit set, which costs three divisions per value).
// A_i B_j^T is an exact integer product (|s_i s_j| <= 128^2), accumulated exactly in
// int32 TMEM; the products with i + j <= 5 are kept, one accumulator per order
// k = i + j, and the epilogue forms 2^(eA + eB) sum_k D_k / (127^2 256^(k-2)) in FP64
// (exact while K <= OZ_MAX_K). The operands are sliced from FP64 AO values (an FP32 copy
// of phi would cost ~3e-9 of Exc, the slices cost ~1e-11), and the rho epilogue
// multiplies by FP64 AO values. FP32 accumulation, whose rounding on the tensor cores is
// toward zero, never occurs.
//
// AO values are never stored: the AO kernel keeps each shell's radial sums S0, S1
// per point (16 bytes per shell and point instead of 32 per AO and point for phi
// and its gradient) and every consumer forms the components from them.
constexpr double kOzD1 = 127.0, kOzD = 256.0;
__device__ __forceinline__ double oz_weight(int k) {  // weight of order k = i + j
    double w = 1.0 / (kOzD1 * kOzD1);
    for (int i = 2; i < k; ++i) w /= kOzD;
    return w;
}

// exponent e with |v| < 2^e for every |v| <= m; an all-zero row gets kOzZeroExp, below every
// double's exponent, so that a group maximum over row exponents ignores it (its digits are 0
// and ldexp of a zero sum stays 0)
constexpr int kOzZeroExp = -1100;
__device__ __forceinline__ int oz_exponent(double m) {
    int e = kOzZeroExp;
    if (m > 0.0) frexp(m, &e);
    return e;
}

// 2^e (0 below the normal range, where only kOzZeroExp sums lie, and those sums are 0)
__device__ __forceinline__ double oz_pow2(int e) {
    return e < -1022 ? 0.0 : __longlong_as_double((long long)(e + 1023) << 52);
}

// The digits of one value at row scale 2^e as one word (byte i = digit s_{4-i}):
// q = rint(v 127 256^3 2^-e), |q| <= 127 2^24, is sum_i s_i 256^(4-i) with s_i in [-128, 127];
// u = q + 0x80808080 (no carry out of 32 bits for that range) has the bytes s_i + 128, and
// flipping every byte's top bit gives s_i in two's complement. sc = 0 for an all-zero row.
constexpr double kOzFull = 127.0 * 256.0 * 256.0 * 256.0;
__device__ __forceinline__ double oz_digit_scale(int e) { return e <= kOzZeroExp ? 0.0 : ldexp(kOzFull, -e); }
// rint(t) for |t| < 2^31 is the low word of t + 1.5 2^52 (one FP64 add, round to nearest even, the
// rounding of cvt.rni), so the cut needs no conversion instruction; the product is rounded
// first, as in rint(v sc).
constexpr double kOzRound = 6755399441055744.0;  // 1.5 2^52
__device__ __forceinline__ uint32_t oz_word(double v, double sc) {
    const int q = __double2loint(__dadd_rn(__dmul_rn(v, sc), kOzRound));
    return ((uint32_t)q + 0x80808080u) ^ 0x80808080u;
}
// Digit-plane layouts in HBM, in the order the contraction stages need them, so that a stage is
// two bulk copies. Within a 64-K slab the canonical no-swizzle K-major core-matrix order of a
// 128-row tile, [k16 group][8-row group][8 rows x 16 bytes].
// * A operands (128-row tiles: phi^T for rho, phi for Vxc): per (tile, slab) the four planes'
//   8 KiB slabs one after another (32 KiB); plane i at + 8192 i.
// * B operands (64-row tiles: P_sub for rho, Z for Vxc): per (64-row tile, slab) two 8 KiB pairs
//   [B_1; B_2], [B_3; B_4] in the layout of a 128-row slab, plane i at rows 64 (i % 2) of pair
//   i / 2 (16 KiB); plane i at + 8192 (i / 2) + 1024 (i % 2).
struct OzPlanes {
    uint32_t pair, half;  // plane i lies (i / 2) pair + (i % 2) half bytes after plane 0
};
constexpr OzPlanes kOzPlanesA{16384, 8192}, kOzPlanesB{8192, 1024};
__host__ __device__ inline size_t oz_off_a(int r, int k, int K) {
    return ((size_t)(r / 128) * (K / 64) + k / 64) * 32768 + (size_t)((((k % 64) / 16) * 16 + (r % 128) / 8) * 128) +
           (r % 8) * 16 + (k % 16);
}
__host__ __device__ inline size_t oz_off_b(int r, int k, int K) {
    return ((size_t)(r / 64) * (K / 64) + k / 64) * 16384 + (size_t)(((k % 64) / 16) * 2048 + ((r % 64) / 8) * 128) +
           (r % 8) * 16 + (k % 16);
}

// 16 values' digit words (byte i of a word = digit s_{4-i}) to the four digit planes
__device__ __forceinline__ void oz_store16_words(char* base, OzPlanes pl, size_t off, const uint32_t* wd) {
    uint4 d[OZ_SLICES];
    uint32_t* dw = reinterpret_cast<uint32_t*>(d);
#pragma unroll
    for (int g = 0; g < 4; ++g) {
        const uint32_t a = wd[4 * g], b = wd[4 * g + 1], c = wd[4 * g + 2], w = wd[4 * g + 3];
        const uint32_t t0 = __byte_perm(a, b, 0x5140), t1 = __byte_perm(a, b, 0x7362);
        const uint32_t t2 = __byte_perm(c, w, 0x5140), t3 = __byte_perm(c, w, 0x7362);
        dw[3 * 4 + g] = __byte_perm(t0, t2, 0x5410);  // byte 0: s_4
        dw[2 * 4 + g] = __byte_perm(t0, t2, 0x7632);  // byte 1: s_3
        dw[1 * 4 + g] = __byte_perm(t1, t3, 0x5410);  // byte 2: s_2
        dw[0 * 4 + g] = __byte_perm(t1, t3, 0x7632);  // byte 3: s_1
    }
#pragma unroll
    for (int i = 0; i < OZ_SLICES; ++i)
        *reinterpret_cast<uint4*>(base + off + (i >> 1) * pl.pair + (i & 1) * pl.half) = d[i];
}
__device__ __forceinline__ void oz_store16(char* base, OzPlanes pl, size_t off, const double* v, int e) {
    const double sc = oz_digit_scale(e);
    uint32_t w[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) w[j] = oz_word(v[j], sc);
    oz_store16_words(base, pl, off, w);
}

__device__ __forceinline__ double warp_max_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}


// AO stage and phi digits of a whole group in one CTA (512 threads, one per point of its up
// to four blocks). Pass 1: the radial sums S0, S1 of every shell of the group's basis at the
// thread's point (stored for the later stages) and the point's exponent of phi^T rows (the
// max over the AOs: max_c |A_c S0| = |S0| max_c |A_c|, the rounding being monotone). Pass 2,
// per tile of 16 AO rows: every thread forms phi of its point row by row from S0 and cuts its
// 16 digits with the point's scale (one 16-byte store per digit plane). These are the only
// phi digits: the Vxc contraction reads them as an MN-major operand and takes the point scale
// into Z' = 2^e_pt Z.
constexpr int kGroupPts = 4 * BLOCK_PTS;

// Prefetch into L1 of the line holding p (no wait, no register).
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// L1 prefetches of this thread's radial sums (S0, and S1 for a GGA) of the shells of 16 rows.
template <bool S1>
__device__ __forceinline__ void oz_prefetch_rows(const RowGeom* rg, int r0, const BlockMeta& m, const double* rad,
                                                 int q) {
    int prev = -1;
#pragma unroll 4
    for (int r = 0; r < 16; ++r) {
        if (r0 + r >= m.nb) break;
        const int slot = rg[r].info >> 4;
        if (slot != prev) {
            prefetch_l1(rad + (size_t)slot * BLOCK_PTS + q);
            if (S1) prefetch_l1(rad + (size_t)(m.nsh + slot) * BLOCK_PTS + q);
            prev = slot;
        }
    }
}

// Row geometry of rows r0 .. r0 + 15 into rg by the CTA's last 16 threads (zero past the last row).
__device__ __forceinline__ void oz_stage_rows(const GridView& g, const BlockMeta& m, int r0, RowGeom* rg) {
    const int k = (int)threadIdx.x - ((int)blockDim.x - 16);
    if (k >= 0) rg[k] = r0 + k < m.nb ? g.blk_row_geom[m.ao0 + r0 + k] : RowGeom{0.0, 0.0, 0.0, 0, 0};
}

// max_c |A_c| over a shell's components (the expressions of ang_poly1, without its branch per component)
__device__ __forceinline__ double ang_max_abs(int L, double x, double y, double z) {
    if (L == 0) return 1.0;
    if (L == 1) return fmax(fabs(x), fmax(fabs(y), fabs(z)));
    const double s3 = 0.57735026918962576451;  // 1/sqrt(3)
    const double a = fmax(fabs(x * y), fmax(fabs(z * x), fabs(y * z)));
    return fmax(a, fmax(fabs(0.5 * (x * x - y * y)), fabs(s3 * (z * z - 0.5 * (x * x + y * y)))));
}

// Shared memory of k_phi_group: the group's shell table (pass 1), then its rows' geometry
// (pass 2); a group whose table or rows do not fit reads them from global.
constexpr size_t kPhiGroupBytes = 64 * 1024;
constexpr int kPhiRowsCap = (int)(kPhiGroupBytes / sizeof(RowGeom));

template <bool GGA>
__global__ void __launch_bounds__(kGroupPts, 2) k_phi_group(BasisView bas, GridView g, const int* __restrict__ grp,
                                                              char* ws) {
    extern __shared__ __align__(16) uint8_t psm[];
    const int lead = grp[blockIdx.x];
    const BlockMeta m = g.meta[lead];
    const OzLayout L = oz_layout(m.nbp, m.nsh);
    const int tid = threadIdx.x, b = tid / BLOCK_PTS, q = tid % BLOCK_PTS;
    const bool live = b < m.gn;
    char* base = ws + g.meta[lead + (live ? b : 0)].ws;
    double* rad = reinterpret_cast<double*>(base + L.rad);
    ShellRec* recs = reinterpret_cast<ShellRec*>(psm);
    RowGeom* rows = reinterpret_cast<RowGeom*>(psm);
    const bool staged = (size_t)m.nsh * sizeof(ShellRec) <= kPhiGroupBytes;  // uniform over the CTA
    if (staged)
        for (int i = tid; i < m.nsh; i += blockDim.x) stage_shell(bas, g.blk_shells[m.sh0 + i], 0, recs[i]);
    __syncthreads();
    int ept = kOzZeroExp;
    double rx = 0.0, ry = 0.0, rz = 0.0;
    if (live) {
        const size_t gp = (size_t)(lead + b) * BLOCK_PTS + q;
        rx = g.px[gp], ry = g.py[gp], rz = g.pz[gp];
        double pm = 0.0;
        for (int i = 0; i < m.nsh; ++i) {
            double x, y, z, S0, S1;
            int Lq;
            if (staged) {
                const ShellRec& r = recs[i];
                x = rx - r.ax, y = ry - r.ay, z = rz - r.az;
                Lq = r.lq;
                shell_radial_staged<GGA>(bas, r, x * x + y * y + z * z, S0, S1);
            } else {
                const int sh = g.blk_shells[m.sh0 + i];
                const int a = bas.sh_atom[sh];
                x = rx - bas.atom_xyz[3 * a], y = ry - bas.atom_xyz[3 * a + 1], z = rz - bas.atom_xyz[3 * a + 2];
                Lq = bas.sh_l[sh];
                shell_radial<GGA>(bas, sh, x * x + y * y + z * z, S0, S1);
            }
            rad[(size_t)i * BLOCK_PTS + q] = S0;
            if (GGA) rad[(size_t)(m.nsh + i) * BLOCK_PTS + q] = S1;
            pm = fmax(pm, ang_max_abs(Lq, x, y, z) * fabs(S0));
        }
        ept = oz_exponent(pm);
        reinterpret_cast<int*>(base + L.e_pt)[q] = ept;
    }
    __syncthreads();  // the shell table is no longer read
    const bool rows_staged = m.nb <= kPhiRowsCap;
    if (rows_staged)
        for (int i = tid; i < m.nb; i += blockDim.x) rows[i] = g.blk_row_geom[m.ao0 + i];
    __syncthreads();
    if (!live) return;
    const RowGeom* rg = rows_staged ? rows : g.blk_row_geom + m.ao0;
    const double sc = oz_digit_scale(ept);
    oz_prefetch_rows<false>(rg, 0, m, rad, q);
    for (int mu0 = 0; mu0 < m.nbp; mu0 += 16) {
        if (mu0 + 16 < m.nb) oz_prefetch_rows<false>(rg + mu0 + 16, mu0 + 16, m, rad, q);  // the next tile's S0
        // row by row (uniform over the CTA; the rows of one shell read the same S0 from L1), phi = A S0,
        // cut at once: the tile's 16 values stay in registers
        uint32_t w[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            double v = 0.0;
            if (mu0 + r < m.nb) {
                const RowGeom gq = rg[mu0 + r];
                double A, Ax, Ay, Az;
                ang_poly1(gq.info & 15, rx - gq.ax, ry - gq.ay, rz - gq.az, A, Ax, Ay, Az);
                v = A * rad[(size_t)(gq.info >> 4) * BLOCK_PTS + q];
            }
            w[r] = oz_word(v, sc);
        }
        oz_store16_words(base + L.phi1, kOzPlanesA, oz_off_a(q, mu0, m.nbp), w);
    }
}

// The digits of P, once per build (a warp per row): the row's exponent (the scale of that row in
// every group's P_sub; the maximum over the whole row bounds the maximum over a group's
// columns, so the digits stay in range, and a row's largest elements, near its diagonal, lie in
// every group that holds the row, so the scale is almost always the sub-row's own), then each
// element's four digits as one word. The groups' P_sub packing then gathers 4-byte words
// instead of 8-byte values and cuts nothing.
__global__ void __launch_bounds__(256) k_p_digits(const double* __restrict__ P, int nao, const int* __restrict__ row_cols,
                                                  int* __restrict__ e, uint32_t* __restrict__ words) {
    const int row = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (row >= nao) return;
    const int c0 = row_cols ? row_cols[2 * row] : 0, c1 = row_cols ? row_cols[2 * row + 1] : nao;
    const double* r = P + (size_t)row * nao;
    double mx = 0.0;
    for (int c = c0 + lane; c < c1; c += 32) mx = fmax(mx, fabs(__ldg(r + c)));
    mx = warp_max_d(mx);
    const int er = oz_exponent(mx);
    if (lane == 0) e[row] = er;
    const double sc = oz_digit_scale(er);
    uint32_t* w = words + (size_t)row * nao;
    for (int c = c0 + lane; c < c1; c += 32) w[c] = oz_word(__ldg(r + c), sc);
}

// P_sub digits of a group: a gather of the words of P[aos[mu]][aos[nu]] (the digit words of a
// zero are 0). A warp takes tiles of 8 rows x 64 columns. It loads them along the rows (lane = a
// column, 32 consecutive screened AOs per load instruction: runs of neighbouring addresses), writes
// them to a shared-memory tile, and reads them back across (lane = row r, K group kg: 16 columns)
// for the digit-plane stores, each of which writes four whole 128-byte core matrices. The shared
// tile's columns are XOR-swizzled by row (a read touches each bank at most twice).
__global__ void __launch_bounds__(256) k_pack_p_oz(GridView g, const uint32_t* __restrict__ words, int nao,
                                                   const int* __restrict__ grp, const int* __restrict__ p_rowexp,
                                                   char* ws) {
    const int blk = grp[blockIdx.x];  // one CTA per group: P_sub lives in the first block's region
    const BlockMeta m = g.meta[blk];
    const OzLayout L = oz_layout(m.nbp, m.nsh);
    char* base = ws + m.ws;
    int* e_p = reinterpret_cast<int*>(base + L.e_p);
    // the group's AO list in shared memory (a group with more screened AOs reads it from global)
    constexpr int kAosCap = 1024;
    __shared__ int s_aos[kAosCap];
    __shared__ uint32_t s_tile[8][8][64];  // per warp: 8 rows x 64 columns
    const bool staged = m.nb <= kAosCap;
    if (staged)
        for (int i = threadIdx.x; i < m.nb; i += blockDim.x) s_aos[i] = g.blk_aos[m.ao0 + i];
    __syncthreads();
    const int* aos = staged ? s_aos : g.blk_aos + m.ao0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = lane & 7, kg = lane >> 3;
    const int nk = m.nbp / 64, ntile = (m.nbp / 8) * nk;
    constexpr int kWarps = 8;  // 256 threads
    uint32_t(*tile)[64] = s_tile[warp];
    for (int t = warp; t < ntile; t += kWarps) {
        const int mu0 = (t / nk) * 8, k0 = (t % nk) * 64;
        // the tile's column AOs (two per lane) and, row by row, the words
        const int nu0 = k0 + lane, nu1 = k0 + 32 + lane;
        const int anu0 = nu0 < m.nb ? aos[nu0] : -1, anu1 = nu1 < m.nb ? aos[nu1] : -1;
        uint32_t v[8][2];
#pragma unroll
        for (int rr = 0; rr < 8; ++rr) {
            const int mu = mu0 + rr;
            const bool live = mu < m.nb;
            const uint32_t* row = words + (size_t)(live ? aos[mu] : 0) * nao;
            v[rr][0] = (live && anu0 >= 0) ? __ldg(row + anu0) : 0u;
            v[rr][1] = (live && anu1 >= 0) ? __ldg(row + anu1) : 0u;
        }
        if (k0 == 0 && lane < 8) {
            const int mu = mu0 + lane;
            e_p[mu] = mu < m.nb ? __ldg(p_rowexp + aos[mu]) : kOzZeroExp;
        }
#pragma unroll
        for (int rr = 0; rr < 8; ++rr) {
            tile[rr][lane ^ rr] = v[rr][0];
            tile[rr][(32 + lane) ^ rr] = v[rr][1];
        }
        __syncwarp();
        uint32_t w[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) w[j] = tile[r][(kg * 16 + j) ^ r];
        __syncwarp();  // the tile is read before the next one is written
        oz_store16_words(base + L.ppack, kOzPlanesB, oz_off_b(mu0 + r, k0 + kg * 16, m.nbp), w);
    }
}

// Z' digits of a whole group in one CTA (512 threads, one per point of its up to four blocks):
// Z' = 2^e_pt Z takes the point scale of the phi^T digits, which the Vxc contraction reads as
// its other operand (W_mu_nu = sum_p phi_p_mu Z_p_nu = sum_p (2^-e_pt phi_p_mu) Z'_p_nu). Per tile
// of 16 rows the CTA forms Z' once in shared memory, takes each row's maximum over the group's
// points (the group's row scale, stored by the first block for the Vxc epilogue), and cuts the
// digits of every block from the same tile into 128-row A-operand tiles.
struct OzGroupTile {
    double x[kGroupPts], y[kGroupPts], z[kGroupPts];
    double c[4][kGroupPts];
    double vt[16][kGroupPts + 1];
    RowGeom rg[2][16];  // row geometry of this tile and the next (staged during this tile's row maxima)
    int eg[16];
};
constexpr size_t kGroupTileBytes = sizeof(OzGroupTile);

template <bool GGA>
__global__ void __launch_bounds__(kGroupPts, 2) k_pack_z_group(GridView g, const int* __restrict__ grp,
                                                                 const double* __restrict__ coef, char* ws) {
    extern __shared__ __align__(16) uint8_t zsm[];
    OzGroupTile& T = *reinterpret_cast<OzGroupTile*>(zsm);
    const int lead = grp[blockIdx.x];
    const BlockMeta m = g.meta[lead];
    const OzLayout L = oz_layout(m.nbp, m.nsh);
    const int tid = threadIdx.x, b = tid / BLOCK_PTS, q = tid % BLOCK_PTS;
    const bool live = b < m.gn;
    const int blk = lead + (live ? b : 0);
    char* base = ws + g.meta[blk].ws;
    const double* rad = reinterpret_cast<const double*>(base + L.rad);
    if (live) {
        const size_t gp = (size_t)blk * BLOCK_PTS + q;
        T.x[tid] = g.px[gp], T.y[tid] = g.py[gp], T.z[tid] = g.pz[gp];
        const double s = oz_pow2(reinterpret_cast<const int*>(base + L.e_pt)[q]);  // the point's phi scale
#pragma unroll
        for (int k = 0; k < 4; ++k) T.c[k][tid] = coef[gp * 4 + k] * s;
    }
    const int warp = tid >> 5, lane = tid & 31;
    oz_stage_rows(g, m, 0, T.rg[0]);
    for (int nu0 = 0; nu0 < m.nbp; nu0 += 16) {
        const int cur = (nu0 >> 4) & 1;
        __syncthreads();  // the previous tile's digits are cut (and the points and rows are loaded)
        if (live) {
            // Shell by shell over the tile's rows (a run of rows of one shell is uniform over the
            // CTA), with the shell's Z from shell_z: a few FMAs per component.
            const double c0 = T.c[0][tid], c1 = GGA ? T.c[1][tid] : 0.0, c2 = GGA ? T.c[2][tid] : 0.0,
                         c3 = GGA ? T.c[3][tid] : 0.0;
            int r = 0;
            while (r < 16) {
                if (nu0 + r >= m.nb) {
                    T.vt[r][tid] = 0.0;
                    ++r;
                    continue;
                }
                const RowGeom& gq = T.rg[cur][r];
                const int t = gq.info & 15, slot = gq.info >> 4;
                const int Lq = t == 0 ? 0 : (t < 4 ? 1 : 2);
                const int u0 = t - Lq * Lq;                 // the component of row r
                const int n = min(2 * Lq + 1 - u0, 16 - r);  // the shell's rows in this tile from r
                const double S0 = rad[(size_t)slot * BLOCK_PTS + q];
                const double S1 = GGA ? rad[(size_t)(m.nsh + slot) * BLOCK_PTS + q] : 0.0;
                double zc[5];
                shell_z(Lq, T.x[tid] - gq.ax, T.y[tid] - gq.ay, T.z[tid] - gq.az, S0, S1, c0, c1, c2, c3, zc);
#pragma unroll
                for (int k = 0; k < 5; ++k)
                    if (k >= u0 && k < u0 + n) T.vt[r + k - u0][tid] = zc[k];
                r += n;
            }
        } else {
            for (int r = 0; r < 16; ++r) T.vt[r][tid] = 0.0;
        }
        __syncthreads();
        {  // warp r: the row's maximum over the group's points
            const int r = warp;  // 16 warps, 16 rows
            double mx = 0.0;
            for (int p = lane; p < kGroupPts; p += 32) mx = fmax(mx, fabs(T.vt[r][p]));
            mx = warp_max_d(mx);
            if (lane == 0) {
                const int e = oz_exponent(mx);
                T.eg[r] = e;
                reinterpret_cast<int*>(ws + m.ws + L.e_z_g)[nu0 + r] = e;
            }
        }
        oz_stage_rows(g, m, nu0 + 16, T.rg[cur ^ 1]);  // every thread has formed this tile's values
        __syncthreads();
        if (live) oz_prefetch_rows<GGA>(T.rg[cur ^ 1], nu0 + 16, m, rad, q);  // the next tile's sums, under the cut
        if (live) {  // thread = (block b, row r, 16 points kg) of the tile
            const int r = (q & 7) + 8 * (q >> 6), kg = (q >> 3) & 7;
            double v[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) v[j] = T.vt[r][b * BLOCK_PTS + kg * 16 + j];
            oz_store16(base + L.zpack, kOzPlanesA, oz_off_a(nu0 + r, kg * 16, BLOCK_PTS), v, T.eg[r]);
        }
    }
}

// RHO items: (block, 64-row N tile): X^T = phi^T P_sub (M = 128 points, N = 64 AOs mu,
// K = nbp AOs nu, P_sub of the block's group) with the rho / grad rho epilogue. VXC items:
// (group, 128-row M tile, 64-row N tile): W = phi Z^T (M = 128 AOs mu, N = 64 AOs nu, K = all
// points of the group's blocks, 128 per block) with the FP64 atomic epilogue.
//
// One persistent CTA per SM takes items from the device-side scheduler below, with three
// roles: warp 0 claims the items and copies their operand slabs into a ring of S stages
// (mbarriers full / empty), warp 1 issues the MMAs of an item into one of two TMEM accumulator
// sets (each four int32 accumulators of 64 columns, one per order i + j = 2..5; 512 columns in
// all) and commits it to tfull[set], and two epilogue groups of eight warps take alternate
// items: group h reads set h and releases it through tempty[h]. So one item's epilogue runs
// under the next items' copies and MMAs. A stage holds the A tile's four digit planes (128 rows
// x 64 K, canonical no-swizzle K-major layout, 8 KiB each) and the B operand's four planes of
// 64 rows as two stacked pairs [B_1; B_2], [B_3; B_4] of 128 rows (8 KiB each). RHO: A = the
// block's phi^T digits, B = the N tile of P_sub, both K-major, one bulk copy each. VXC: A = the
// M tile of Z', B = the phi^T digits of the N tile's 64 AOs over the slab's 64 points, read
// MN-major (1 KiB per plane and 16-AO group, one 4-D tensor copy per stage).
constexpr int OZ_NT = 64;
// operand ring stages: three in flight for both contractions (the Vxc contraction: K = a group's
// 512 points, eight slabs per item, three stages unless the autotuner picks two; the rho contraction:
// K = nbp, three stages beside its radial-sum staging of kOzRsCap = 8 shells per column half, 1 %
// faster on the 2000-atom chain than two stages beside 12 shells)
template <int MODE>
constexpr int oz_stages() {
    return 3;
}
constexpr uint32_t OZ_A_BYTES = OZ_SLICES * umma::I8_SLAB_BYTES;   // 32 KiB
constexpr uint32_t OZ_B_SLICE = OZ_NT * umma::I8_SLAB_K;          // 4 KiB
constexpr uint32_t OZ_STAGE_BYTES = OZ_A_BYTES + OZ_SLICES * OZ_B_SLICE;  // 48 KiB
constexpr uint32_t OZ_TMEM_COLS = 4 * OZ_NT;                      // one accumulator set
constexpr int OZ_EPI_WARPS = 16;  // two groups of 4 lane quarters x 2 column halves
constexpr int OZ_THREADS = 64 + 32 * OZ_EPI_WARPS;  // copies, MMAs, epilogue
// Epilogue region after the ring, a quarter per (group, column half). RHO: the radial sums of
// up to kOzRsCap shells of the half's columns, staged per thread. VXC: the half's [128][17]
// FP64 transpose tile.
constexpr int kOzRsCap = 8;
template <int MODE>
constexpr uint32_t oz_epi_bytes() {  // rho: 64 KiB of staged radial sums; Vxc: four 17 KiB tiles
    return MODE == MODE_RHO ? 4u * kOzRsCap * 2 * BLOCK_PTS * 8 : 4u * 128 * 17 * 8;
}
template <int MODE, int S>
constexpr uint32_t oz_bar_off() {
    return S * OZ_STAGE_BYTES + oz_epi_bytes<MODE>();
}

// An item's int32 accumulators of orders 2..5 as one exact integer: with weights
// w_k = 256^(5-k) w_5, sum_k d_k w_k = n w_5 with n = ((d2 256 + d3) 256 + d4) 256 + d5, whose
// partial sums are integers below 2^53 for K <= OZ_MAX_K: exact in 64-bit integers, and exactly
// representable in FP64.
__device__ __forceinline__ double oz_combine(uint32_t d2, uint32_t d3, uint32_t d4, uint32_t d5) {
    // n in 64-bit integer arithmetic (three wide multiply-adds), then one exact conversion
    long long n = (long long)(int)d5;
    n += (long long)(int)d4 * 256;
    n += (long long)(int)d3 * 65536;
    n += (long long)(int)d2 * 16777216;
    return (double)n;
}

// Work items of the persistent contraction kernels, one int2 each, in a list sorted by
// decreasing cost (built with the grid, per chunk): RHO {block, N tile of 64 AOs}; VXC {the
// group's first block, (M tile of 128 AOs) << 16 | N tile of 64 AOs}. x < 0 ends the list.
__device__ __forceinline__ void oz_decode(int MODE_, int2 item, int& blk, int& mt, int& nt) {
    blk = item.x;
    mt = MODE_ == MODE_RHO ? 0 : item.y >> 16;
    nt = item.y & 0xFFFF;
}

// The device-side scheduler: the copy warp claims the next item of the cost-sorted list with an
// atomic counter (skipping items outside the launch's block range) and hands it to the MMA
// warp and the epilogue groups through a ring of kOzRing shared-memory slots: ifull[slot]
// (one arrival, the copy warp) and iempty[slot] (two arrivals: the MMA warp and the epilogue
// group that takes the item). Entry q of the ring goes to epilogue group q % 2 and TMEM set
// q % 2; the end of the list is written twice, so that both epilogue groups see it.
constexpr int kOzRing = 4;

// The 10 slice products A_i B_j^T with i + j <= 5 as six MMAs per K step. Product (i, j) goes to
// the accumulator of order i + j, at TMEM columns 64 (i + j - 2); for one A plane the products
// with consecutive j land in adjacent 64-column ranges, so the stage stores the B planes as two
// stacked pairs [B_1; B_2] and [B_3; B_4] (128 rows each, the layout of a 128-row A tile) and
// one N = 128 MMA computes two products:
//   t  A plane  B pair  N    columns  orders
//   0  1        0       128  0..127   2, 3
//   1  1        1       128  128..255 4, 5
//   2  2        0       128  64..191  3, 4
//   3  2        1 (B_3) 64   192..255 5
//   4  3        0       128  128..255 4, 5
//   5  4        0 (B_1) 64   192..255 5
// (nibble t of each constant; unrolled loops fold them). The per-instruction cost of the
// tensor core is nearly the same for N = 64 and N = 128, so six MMAs take about 60 % of the time
// of ten.
__device__ __forceinline__ constexpr int oz_mma_a(int t) { return (int)((0x432211u >> (4 * t)) & 15); }
__device__ __forceinline__ constexpr int oz_mma_pair(int t) { return (int)((0x001010u >> (4 * t)) & 15); }
__device__ __forceinline__ constexpr int oz_mma_wide(int t) { return (int)((0x010111u >> (4 * t)) & 15); }
__device__ __forceinline__ constexpr int oz_mma_col(int t) { return (int)((0x323120u >> (4 * t)) & 15); }

template <int MODE, bool GGA, int S>
__global__ void __launch_bounds__(OZ_THREADS, 1)
    k_oz(BasisView bas, GridView g, int blk0, int nblk, const int2* __restrict__ items, int nitems, int* counter,
         char* ws, int* err, double* rho_acc, double* Vacc, int nao, const __grid_constant__ CUtensorMap phi_map,
         int use_map) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ int2 s_item[kOzRing];
    // per epilogue group and alternate item of the group (a group writes one buffer while its
    // slower warps may still read the other): RHO the item's columns (row geometry, scale); VXC
    // the AO indices of the item's columns and rows and the columns' Z exponents
    __shared__ RowGeom s_geom[MODE == MODE_RHO ? 4 : 1][OZ_NT];
    __shared__ double s_cs[MODE == MODE_RHO ? 4 : 1][OZ_NT];
    __shared__ int s_acol[MODE == MODE_VXC ? 4 : 1][OZ_NT], s_ez[MODE == MODE_VXC ? 4 : 1][OZ_NT];
    __shared__ int s_arow[MODE == MODE_VXC ? 4 : 1][128];
    __shared__ int s_abort;
    if (threadIdx.x == 0) s_abort = *reinterpret_cast<const volatile int*>(err);
    __syncthreads();
    if (s_abort) return;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + oz_bar_off<MODE, S>());
    uint64_t* empty = full + S;
    uint64_t* tfull = empty + S;
    uint64_t* tempty = tfull + 2;
    uint64_t* ifull = tempty + 2;
    uint64_t* iempty = ifull + kOzRing;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(iempty + kOzRing);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) umma::tmem_alloc(tslot, 2 * OZ_TMEM_COLS);
    if (threadIdx.x == 32) {
        for (int st = 0; st < S; ++st) umma::mbar_init(&full[st], 1), umma::mbar_init(&empty[st], 1);
        for (int k = 0; k < 2; ++k) umma::mbar_init(&tfull[k], 1), umma::mbar_init(&tempty[k], OZ_EPI_WARPS / 2);
        for (int k = 0; k < kOzRing; ++k) umma::mbar_init(&ifull[k], 1), umma::mbar_init(&iempty[k], 2);
        umma::mbar_init_fence();
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tslot;
    constexpr int kBlockSlabs = BLOCK_PTS / (int)umma::I8_SLAB_K;  // VXC: K slabs per block

    if (warp == 0) {
        // the scheduler (lane 0), then the item's copies: lane 0 issues the A copy (and the rho B
        // copy), and for the Vxc contraction lanes 0..15 issue the 16 pieces of its B operand at once
        constexpr unsigned kAll = 0xffffffffu;
        uint32_t gj = 0;
        bool ok = true;
        // entry q of the ring into its slot, once the slot's entry q - kOzRing is consumed (lane 0)
        auto push = [&](int q, int2 item) {
            const int slot = q % kOzRing;
            if (q >= kOzRing && !umma::mbar_wait(&iempty[slot], ((q / kOzRing) - 1) & 1, err)) {
                atomicExch(err, 5);
                return false;
            }
            s_item[slot] = item;
            umma::mbar_arrive(&ifull[slot]);  // release: the slot's item is visible to the consumers
            return true;
        };
        for (int q = 0; ok; ++q) {
            int2 item = make_int2(-1, 0);
            int pushed = 1;
            if (lane == 0) {
                for (;;) {  // the next item of the launch's block range
                    const int it = atomicAdd(counter, 1);
                    if (it >= nitems) break;
                    item = __ldg(items + it);
                    if (item.x >= blk0 && item.x < blk0 + nblk) break;
                    item = make_int2(-1, 0);
                }
                pushed = push(q, item) ? 1 : 0;
                if (pushed && item.x < 0) push(q + 1, item);
            }
            item.x = __shfl_sync(kAll, item.x, 0);
            item.y = __shfl_sync(kAll, item.y, 0);
            pushed = __shfl_sync(kAll, pushed, 0);
            if (!pushed || item.x < 0) break;
            int blk, mt, nt;
            oz_decode(MODE, item, blk, mt, nt);
            const BlockMeta m = g.meta[blk];
            const OzLayout L = oz_layout(m.nbp, m.nsh);
            const char* base = ws + m.ws;
            const char* lead = ws + g.meta[m.lead].ws;
            size_t Ao, Bo;
            int nslabs, kslabs;  // slabs of the item; slabs per block of the K extent
            if (MODE == MODE_RHO) {  // per slab one 32 KiB A copy and one 16 KiB B copy
                nslabs = kslabs = m.nbp / (int)umma::I8_SLAB_K;
                Ao = L.phi1;
                Bo = L.ppack + (size_t)nt * kslabs * 16384;
            } else {  // A: Z' rows of tile mt; B: the phi^T digits of AO slab nt, read MN-major
                kslabs = kBlockSlabs;
                nslabs = m.gn * kBlockSlabs;
                Ao = L.zpack + (size_t)mt * kslabs * 32768;
                Bo = L.phi1 + (size_t)nt * 32768;
            }
            for (int j = 0; j < nslabs; ++j, ++gj) {
                const int st = gj % S;
                int w = 1;
                if (lane == 0) {
                    if (gj >= S && !umma::mbar_wait(&empty[st], ((gj / S) - 1) & 1, err)) {
                        atomicExch(err, 1);
                        w = 0;
                    } else {
                        umma::mbar_expect_tx(&full[st], OZ_STAGE_BYTES);
                    }
                }
                if (!__shfl_sync(kAll, w, 0)) {
                    ok = false;
                    break;
                }
                uint8_t* sp = smem + st * OZ_STAGE_BYTES;
                const char *As = base + Ao, *Bs = lead + Bo;
                int js = j;
                if (MODE == MODE_VXC) {  // slab j: block lead + j / kBlockSlabs, its slab j % kBlockSlabs
                    const char* bj = ws + g.meta[m.lead + j / kBlockSlabs].ws;
                    As = bj + Ao, Bs = bj + Bo;
                    js = j % kBlockSlabs;
                }
                if (lane == 0) umma::bulk_g2s(sp, As + (size_t)js * 32768, OZ_A_BYTES, &full[st]);
                if (MODE == MODE_RHO) {
                    if (lane == 0)
                        umma::bulk_g2s(sp + OZ_A_BYTES, Bs + (size_t)js * 16384, OZ_STAGE_BYTES - OZ_A_BYTES,
                                       &full[st]);
                } else if (use_map) {
                    // the 64 points js of the slab: per plane i and 16-AO group kg the 8 core matrices of
                    // those points (1 KiB), in the stage plane i at 4 KiB i, group kg at 1 KiB kg: one
                    // tensor copy of the box {1 KiB, 4 groups, 4 planes} at the slab's 256-byte offset
                    if (lane == 0)
                        umma::tensor4_g2s(sp + OZ_A_BYTES, &phi_map, 0, 0, 0,
                                          (int)((Bs + (size_t)js * 1024 - ws) >> 8), &full[st]);
                } else if (lane < 16) {  // the same 16 pieces as bulk copies
                    const int i = lane >> 2, kg = lane & 3;
                    umma::bulk_g2s(sp + OZ_A_BYTES + i * 4096 + kg * 1024,
                                   Bs + (size_t)i * 8192 + kg * 2048 + (size_t)js * 1024, 1024, &full[st]);
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {  // MMAs
            // Vxc: B (the phi^T digits) is MN-major (bit 16 of the instruction descriptor)
            constexpr uint32_t bmaj = MODE == MODE_VXC ? (1u << 16) : 0u;
            const uint32_t idesc128 = umma::instr_desc_s8(128, 2 * OZ_NT) | bmaj,
                           idesc64 = umma::instr_desc_s8(128, OZ_NT) | bmaj;
            uint32_t gj = 0;
            int li = 0;
            bool ok = true;
            for (int q = 0; ok; ++q) {
                const int slot = q % kOzRing;
                if (!umma::mbar_wait(&ifull[slot], (q / kOzRing) & 1, err)) {
                    atomicExch(err, 6);
                    break;
                }
                const int2 item = s_item[slot];
                umma::mbar_arrive(&iempty[slot]);
                if (item.x < 0) break;
                int blk, mt, nt;
                oz_decode(MODE, item, blk, mt, nt);
                const BlockMeta m = g.meta[blk];
                const int nslabs = MODE == MODE_RHO ? m.nbp / (int)umma::I8_SLAB_K : m.gn * kBlockSlabs;
                const int set = li & 1;
                if (li >= 2 && !umma::mbar_wait(&tempty[set], ((li >> 1) - 1) & 1, err)) {
                    atomicExch(err, 4);
                    break;
                }
                umma::fence_after_sync();
                const uint32_t tacc = tmem + (uint32_t)set * OZ_TMEM_COLS;
                for (int j = 0; j < nslabs; ++j, ++gj) {
                    const int st = gj % S;
                    if (!umma::mbar_wait(&full[st], (gj / S) & 1, err)) {
                        atomicExch(err, 2);
                        ok = false;
                        break;
                    }
                    umma::fence_after_sync();
                    // the stage's base descriptors; an operand's descriptor adds its byte offset / 16
                    // to the start-address field (addresses stay below 256 KiB, so it cannot carry)
                    const uint32_t sp = umma::smem_u32(smem + st * OZ_STAGE_BYTES);
                    const uint64_t ad0 = umma::smem_desc(sp, umma::LBO, umma::SBO);
                    // B: K-major stacked pairs (rho), or MN-major planes of 64 AOs x 64 points (Vxc: in
                    // the no-swizzle MN-major layout LBO steps K, the next 8 points 128 B on, and SBO
                    // steps MN, the next 16 AOs 1 KiB on)
                    const uint64_t bd0 = MODE == MODE_RHO ? umma::smem_desc(sp + OZ_A_BYTES, umma::LBO, umma::SBO)
                                                          : umma::smem_desc(sp + OZ_A_BYTES, 128, 1024);
                    constexpr uint32_t bk = MODE == MODE_RHO ? 4096 : 512;  // B offset of the second K step
#pragma unroll
                    for (int kk = 0; kk < 2; ++kk) {
#pragma unroll
                        for (int t = 0; t < 6; ++t) {
                            const int i = oz_mma_a(t);
                            const uint64_t ad = ad0 + (uint64_t)(((i - 1) * umma::I8_SLAB_BYTES + kk * 4096) >> 4);
                            const uint64_t bd = bd0 + (uint64_t)((oz_mma_pair(t) * 8192 + kk * bk) >> 4);
                            // the two MMAs of A_1 start all four accumulators
                            const bool first = (j == 0 && kk == 0 && t < 2);
                            umma::mma_s8(tacc + (uint32_t)oz_mma_col(t) * OZ_NT, ad, bd,
                                         oz_mma_wide(t) ? idesc128 : idesc64, first ? 0u : 1u);
                        }
                    }
                    umma::mma_commit(&empty[st]);
                }
                if (!ok) break;
                umma::mma_commit(&tfull[set]);
                ++li;
            }
        }
        __syncwarp();
    } else {  // epilogue: two groups of 8 warps (2..9 and 10..17) take alternate items
        // Group h takes the items with li % 2 == h and so always reads TMEM set h; while one
        // group waits on its loads the other computes. Warp w reads TMEM lanes 32 (w % 4) .. + 31.
        const int h = (warp - 2) >> 3;
        const int quarter = warp & 3, chalf = ((warp - 2) >> 2) & 1;  // lane quarter, column half
        const int gt = (threadIdx.x - 64) & 255;                        // thread index in the group
        const int gbar = 1 + h;                                          // the group's named barrier
        const int ca = chalf * 32;                                       // this thread's columns [ca, ca + 32)
        const double w5 = oz_weight(5);
        uint8_t* epi = smem + S * OZ_STAGE_BYTES;
        const uint32_t tq = tmem + (uint32_t)h * OZ_TMEM_COLS + ((uint32_t)(quarter * 32) << 16);
        for (int q = h;; q += 2) {  // ring entries q = h, h + 2, ...: TMEM set h
            const int slot = q % kOzRing;
            bool got = umma::mbar_wait(&ifull[slot], (q / kOzRing) & 1, err);
            got = umma::named_and(gbar, 256, got);
            if (!got) {
                if (gt == 0) atomicExch(err, 7);
                break;
            }
            const int2 item = s_item[slot];
            umma::named_sync(gbar, 256);  // every thread of the group has read the slot
            if (gt == 0) umma::mbar_arrive(&iempty[slot]);
            if (item.x < 0) break;
            int blk, mt, nt;
            oz_decode(MODE, item, blk, mt, nt);
            const int ph = (q >> 1) & 1;  // tfull[h] parity of this item
            const int sb = 2 * h + ph;    // the item's shared-memory buffer
            const BlockMeta m = g.meta[blk];
            const OzLayout L = oz_layout(m.nbp, m.nsh);
            const char* base = ws + m.ws;
            const char* lead = ws + g.meta[m.lead].ws;
            if (MODE == MODE_RHO) {
                // Per item: the columns' row geometry and scales w5 2^e_p in shared memory; each
                // thread (point = its lane, 32 columns) stages the radial sums of its columns'
                // shells (independent loads) while the MMAs run; then, shell by shell, it reads the
                // shell's accumulator columns from TMEM, forms X and phi, grad phi of the shell's
                // components at its point and accumulates rho and grad rho.
                const int col0 = nt * OZ_NT;
                if (gt < OZ_NT) {
                    const bool live = col0 + gt < m.nb;
                    s_geom[sb][gt] = live ? g.blk_row_geom[m.ao0 + col0 + gt] : RowGeom{0.0, 0.0, 0.0, 0, 0};
                    s_cs[sb][gt] = live ? w5 * oz_pow2(reinterpret_cast<const int*>(lead + L.e_p)[col0 + gt]) : 0.0;
                }
                umma::named_sync(gbar, 256);
                const int pt = quarter * 32 + lane;
                const double* rad = reinterpret_cast<const double*>(base + L.rad);
                const int cb = min(ca + 32, m.nb - col0);
                double* rs = reinterpret_cast<double*>(epi) + (size_t)(2 * h + chalf) * kOzRsCap * 2 * BLOCK_PTS;
                int slot0 = 0, ns = 0;
                if (ca < cb) {
                    slot0 = s_geom[sb][ca].info >> 4;
                    ns = min((s_geom[sb][cb - 1].info >> 4) - slot0 + 1, kOzRsCap);
                    for (int k = 0; k < ns; ++k) {
                        rs[(2 * k) * BLOCK_PTS + pt] = rad[(size_t)(slot0 + k) * BLOCK_PTS + pt];
                        if (GGA) rs[(2 * k + 1) * BLOCK_PTS + pt] = rad[(size_t)(m.nsh + slot0 + k) * BLOCK_PTS + pt];
                    }
                }
                const int ep = reinterpret_cast<const int*>(base + L.e_pt)[pt];
                const size_t gp = (size_t)blk * BLOCK_PTS + pt;
                const double px = g.px[gp], py = g.py[gp], pz = g.pz[gp];
                bool ok = umma::mbar_wait(&tfull[h], ph, err);
                __syncwarp();
                ok = umma::named_and(gbar, 256, ok);
                if (!ok) {
                    if (gt == 0) atomicExch(err, 3);
                    break;
                }
                umma::fence_after_sync();
                double r = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
                for (int c = ca; c < cb;) {
                    const RowGeom q = s_geom[sb][c];
                    const int t = q.info & 15, slot = q.info >> 4, k = slot - slot0;
                    const int Lq = t == 0 ? 0 : (t < 4 ? 1 : 2);
                    const int cs0 = c - (t - Lq * Lq);  // column of the shell's first component
                    const int ce = cs0 + 2 * Lq + 1;
                    // the shell's accumulator columns in [ca, cb) (a uniform branch per column)
                    uint32_t d[5][4];
#pragma unroll
                    for (int u = 0; u < 5; ++u) {
                        const int cc = cs0 + u;
                        if (cc < ce && cc >= ca && cc < cb) {
#pragma unroll
                            for (int o = 0; o < 4; ++o) umma::tmem_ld1_raw(tq + o * OZ_NT + cc, d[u][o]);
                        }
                    }
                    const bool staged = (unsigned)k < (unsigned)ns;
                    const double S0 = staged ? rs[(2 * k) * BLOCK_PTS + pt] : rad[(size_t)slot * BLOCK_PTS + pt];
                    double S1 = 0.0;
                    if (GGA)
                        S1 = staged ? rs[(2 * k + 1) * BLOCK_PTS + pt] : rad[(size_t)(m.nsh + slot) * BLOCK_PTS + pt];
                    const double x = px - q.ax, y = py - q.ay, z = pz - q.az;
                    umma::tmem_wait_ld();
                    // the shell's X (zero for its components outside [ca, cb)), then its rho terms
                    double xv[5];
#pragma unroll
                    for (int u = 0; u < 5; ++u) {
                        const int cc = cs0 + u;
                        xv[u] = (cc < ce && cc >= ca && cc < cb)
                                    ? oz_combine(d[u][0], d[u][1], d[u][2], d[u][3]) * s_cs[sb][cc]
                                    : 0.0;
                    }
                    shell_rho<GGA>(Lq, x, y, z, S0, S1, xv, r, gx, gy, gz);
                    c = ce;
                }
                umma::fence_before_sync();
                __syncwarp();
                if (lane == 0) umma::mbar_arrive(&tempty[h]);
                if (ca < cb) {
                    const double sc = oz_pow2(ep);
                    double* acc = rho_acc + ((size_t)blk * BLOCK_PTS + pt) * 4;
                    atomicAdd(acc, r * sc);
                    if (GGA) atomicAdd(acc + 1, gx * sc), atomicAdd(acc + 2, gy * sc), atomicAdd(acc + 3, gz * sc);
                }
            } else {
                // Per item: the columns' AO indices and Z exponents and the rows' AO indices in
                // shared memory; per 16 columns each thread converts its row's accumulators to FP64
                // W in its column half's transpose tile, then the half's 128 threads add the tile
                // to Vacc (16 consecutive columns of two rows per warp instruction).
                // rows: the Z' AOs nu of tile mt (scale 2^e_z_g); columns: the phi AOs mu of tile nt,
                // whose point scales went into Z'. The item adds W_mu_nu at Vacc[nu][mu] (the build
                // symmetrises Vacc).
                const int* aos = g.blk_aos + m.ao0;
                if (gt < OZ_NT) {
                    const int nu = nt * OZ_NT + gt;
                    s_acol[sb][gt] = nu < m.nb ? aos[nu] : -1;
                    s_ez[sb][gt] = 0;
                }
                if (gt < 128) {
                    const int mu = mt * 128 + gt;
                    s_arow[sb][gt] = mu < m.nb ? aos[mu] : -1;
                }
                const int row = quarter * 32 + lane;
                const int em = reinterpret_cast<const int*>(base + L.e_z_g)[mt * 128 + row];
                umma::named_sync(gbar, 256);
                bool ok = umma::mbar_wait(&tfull[h], ph, err);
                __syncwarp();
                ok = umma::named_and(gbar, 256, ok);
                if (!ok) {
                    if (gt == 0) atomicExch(err, 3);
                    break;
                }
                umma::fence_after_sync();
                double* tile = reinterpret_cast<double*>(epi) + (size_t)(2 * h + chalf) * 128 * 17;
                const int tbar = 3 + 2 * h + chalf;  // the column half's named barrier
                for (int c0 = ca; c0 < ca + 32; c0 += 16) {
                    uint32_t d2[16], d3[16], d4[16], d5[16];
                    umma::tmem_ld16_raw(tq + c0, d2);
                    umma::tmem_ld16_raw(tq + OZ_NT + c0, d3);
                    umma::tmem_ld16_raw(tq + 2 * OZ_NT + c0, d4);
                    umma::tmem_ld16_raw(tq + 3 * OZ_NT + c0, d5);
                    umma::tmem_wait_ld();
                    if (c0 == ca + 16) {  // the set is read: hand it back to the MMAs
                        umma::fence_before_sync();
                        __syncwarp();
                        if (lane == 0) umma::mbar_arrive(&tempty[h]);
                    }
#pragma unroll
                    for (int c = 0; c < 16; ++c)
                        tile[row * 17 + c] =
                            oz_combine(d2[c], d3[c], d4[c], d5[c]) * (w5 * oz_pow2(em + s_ez[sb][c0 + c]));
                    umma::named_sync(tbar, 128);
                    const int c = row & 15;
                    const int anu = s_acol[sb][c0 + c];
                    if (anu >= 0) {
                        for (int rr = row >> 4; rr < 128; rr += 8) {
                            const int amu = s_arow[sb][rr];
                            if (amu >= 0) atomicAdd(&Vacc[(size_t)amu * nao + anu], tile[rr * 17 + c]);
                        }
                    }
                    umma::named_sync(tbar, 128);
                }
            }
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) umma::tmem_dealloc(tmem, 2 * OZ_TMEM_COLS);
}

}  // namespace

template <int MODE, int S>
size_t oz_smem_bytes() {
    return (size_t)oz_bar_off<MODE, S>() + (2 * S + 4 + 2 * kOzRing) * 8 + 16;
}

void launch_functional_points(const GridView& g, int blk0, int nblk, int fn, bool incremental, double rho_cut,
                              const double* rho_acc, double* rho_store, double* coef, double* blk_sum,
                              cudaStream_t s) {
    if (functional_is_gga(fn))
        k_functional_mixed<true><<<nblk, BLOCK_PTS, 0, s>>>(g, blk0, fn, incremental, rho_cut, rho_acc, rho_store,
                                                            coef, blk_sum);
    else
        k_functional_mixed<false><<<nblk, BLOCK_PTS, 0, s>>>(g, blk0, fn, incremental, rho_cut, rho_acc, rho_store,
                                                             coef, blk_sum);
}

// The failure path of the bounded waits, exercised without a fault: one thread waits on an
// mbarrier that nothing arrives on, through the same mbar_wait as the contraction kernels,
// gives up after limit_ns and records code 8 in the device error word.
__global__ void k_wait_selftest(int* err, uint64_t limit_ns) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        umma::mbar_init(&bar, 1);
        umma::mbar_init_fence();
        if (!umma::mbar_wait(&bar, 0, err, limit_ns)) atomicExch(err, 8);
    }
}

void launch_wait_selftest(int* err, uint64_t limit_ns, cudaStream_t s) { k_wait_selftest<<<1, 32, 0, s>>>(err, limit_ns); }

void oz_p_digits(const double* P, int nao, const int* row_cols, int* e, uint32_t* words, cudaStream_t s) {
    k_p_digits<<<(nao + 7) / 8, 256, 0, s>>>(P, nao, row_cols, e, words);
}

void oz_prepare(const MixedArgs& a, cudaStream_t s) {
    // per group: radial sums, row scales and the phi digits of both layouts; then P_sub
    if (functional_is_gga(a.fn)) {
        cudaFuncSetAttribute(k_phi_group<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPhiGroupBytes);
        k_phi_group<true><<<a.ngrp, kGroupPts, kPhiGroupBytes, s>>>(a.b, a.g, a.grp, a.ws);
    } else {
        cudaFuncSetAttribute(k_phi_group<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPhiGroupBytes);
        k_phi_group<false><<<a.ngrp, kGroupPts, kPhiGroupBytes, s>>>(a.b, a.g, a.grp, a.ws);
    }
    k_pack_p_oz<<<a.ngrp, 256, 0, s>>>(a.g, a.p_words, a.nao, a.grp, a.p_rowexp, a.ws);
}

// Persistent contraction grid: one CTA per SM (its shared memory and all 512 TMEM columns
// keep a second CTA off the SM), no more than there are items.
static int oz_grid(int nitems) {
    int dev = 0, nsm = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    return std::max(1, std::min(nitems, nsm));
}

template <int MODE, bool GGA, int S>
static void launch_oz(const MixedArgs& a, const int2* items, int nitems, int* counter, cudaStream_t s) {
    const size_t smem = oz_smem_bytes<MODE, S>();
    cudaFuncSetAttribute(k_oz<MODE, GGA, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    CUtensorMap map{};
    if (a.phi_map) map = *a.phi_map;
    k_oz<MODE, GGA, S><<<oz_grid(nitems), OZ_THREADS, smem, s>>>(a.b, a.g, a.blk0, a.nblk, items, nitems, counter,
                                                                 a.ws, a.err, a.rho_acc, a.Vacc, a.nao, map,
                                                                 a.phi_map ? 1 : 0);
}

// The tensor map of the Vxc contraction's phi operand: the workspace as a 4-D tensor of 8-byte
// elements, {128 elements = 1 KiB; 4 16-AO groups, 2 KiB apart; 4 digit planes, 8 KiB apart; the
// offset in 256-byte units} (every region of the workspace starts on 256 bytes), box
// {128, 4, 4, 1}: 16 KiB, landing in shared memory as [plane][group][1 KiB]. The copies it
// serves stay inside a block's phi digits (its slab of 32 KiB).
bool make_phi_map(const void* ws, size_t ws_bytes, CUtensorMap* map) {
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static Encode encode = nullptr;
    static bool looked = false;
    if (!looked) {
        looked = true;
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = reinterpret_cast<Encode>(fn);
        else
            cudaGetLastError();
    }
    if (!encode || !ws || ws_bytes < 32768 || (reinterpret_cast<uintptr_t>(ws) & 255)) return false;
    const cuuint64_t dims[4] = {128, 4, 4, (cuuint64_t)(ws_bytes / 256)};
    const cuuint64_t strides[3] = {2048, 8192, 256};  // bytes, dimensions 1..3
    const cuuint32_t box[4] = {128, 4, 4, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT64, 4, const_cast<void*>(ws), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

void oz_rho(const MixedArgs& a, cudaStream_t s) {
    constexpr int S = oz_stages<MODE_RHO>();
    if (functional_is_gga(a.fn))
        launch_oz<MODE_RHO, true, S>(a, a.items_rho, a.n_rho, a.counters, s);
    else
        launch_oz<MODE_RHO, false, S>(a, a.items_rho, a.n_rho, a.counters, s);
}

void oz_functional(const MixedArgs& a, cudaStream_t s) {
    if (functional_is_gga(a.fn))
        k_functional_mixed<true><<<a.nblk, BLOCK_PTS, 0, s>>>(a.g, a.blk0, a.fn, a.incremental, a.rho_cut, a.rho_acc,
                                                              a.rho_store, a.coef, a.blk_sum);
    else
        k_functional_mixed<false><<<a.nblk, BLOCK_PTS, 0, s>>>(a.g, a.blk0, a.fn, a.incremental, a.rho_cut, a.rho_acc,
                                                               a.rho_store, a.coef, a.blk_sum);
    oz_pack_z(a, s);
}

void oz_pack_p(const MixedArgs& a, cudaStream_t s) {
    k_pack_p_oz<<<a.ngrp, 256, 0, s>>>(a.g, a.p_words, a.nao, a.grp, a.p_rowexp, a.ws);
}

void oz_functional_uks(const MixedArgs& a, const double* rho_acc_b, double* rho_store_b, double* coef_b,
                       double* blk_sum_b, cudaStream_t s) {
    if (functional_is_gga(a.fn))
        k_functional_mixed_uks<true><<<a.nblk, BLOCK_PTS, 0, s>>>(a.g, a.blk0, a.fn, a.incremental, a.rho_cut,
                                                                  a.rho_acc, rho_acc_b, a.rho_store, rho_store_b,
                                                                  a.coef, coef_b, a.blk_sum, blk_sum_b);
    else
        k_functional_mixed_uks<false><<<a.nblk, BLOCK_PTS, 0, s>>>(a.g, a.blk0, a.fn, a.incremental, a.rho_cut,
                                                                   a.rho_acc, rho_acc_b, a.rho_store, rho_store_b,
                                                                   a.coef, coef_b, a.blk_sum, blk_sum_b);
}

void oz_pack_z(const MixedArgs& a, cudaStream_t s) {
    if (functional_is_gga(a.fn)) {
        cudaFuncSetAttribute(k_pack_z_group<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGroupTileBytes);
        k_pack_z_group<true><<<a.ngrp, kGroupPts, kGroupTileBytes, s>>>(a.g, a.grp, a.coef, a.ws);
    } else {
        cudaFuncSetAttribute(k_pack_z_group<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGroupTileBytes);
        k_pack_z_group<false><<<a.ngrp, kGroupPts, kGroupTileBytes, s>>>(a.g, a.grp, a.coef, a.ws);
    }
}

// the Vxc contraction with 2 or 3 operand stages (MixedArgs::vxc_stages; 0 = 3)
void oz_vxc(const MixedArgs& a, cudaStream_t s) {
    if (a.vxc_stages == 2)
        launch_oz<MODE_VXC, false, 2>(a, a.items_vxc, a.n_vxc, a.counters + 1, s);
    else
        launch_oz<MODE_VXC, false, 3>(a, a.items_vxc, a.n_vxc, a.counters + 1, s);
}

size_t umma_smem_bytes(int nterms) {
    const int nA = nterms == 3 ? 2 : 3;
    const int S = nterms == 3 ? 3 : 2;
    return (size_t)S * 2 * nA * umma::SLAB_BYTES + (2 * S + 1) * 8 + 16;
}

static UmmaParams umma_params(const MixedArgs& a) { return UmmaParams{a.nterms, a.nterms == 3 ? 3 : 2, a.err, nullptr}; }

void mixed_prepare(const MixedArgs& a, cudaStream_t s) {
    if (functional_is_gga(a.fn))
        k_ao_mixed<true><<<a.nblk, 256, 0, s>>>(a.b, a.g, a.blk0, a.ws);
    else
        k_ao_mixed<false><<<a.nblk, 256, 0, s>>>(a.b, a.g, a.blk0, a.ws);
    k_pack_p<<<a.nblk, 256, 0, s>>>(a.g, a.P, a.nao, a.blk0, a.ws);
}

void mixed_rho(const MixedArgs& a, cudaStream_t s) {
    const int tiles = a.max_nbp / umma::TILE_ROWS;
    const size_t smem = umma_smem_bytes(a.nterms);
    if (functional_is_gga(a.fn)) {
        cudaFuncSetAttribute(k_umma<MODE_RHO, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_umma<MODE_RHO, true><<<dim3(tiles, a.nblk), 128, smem, s>>>(a.g, a.blk0, a.ws, umma_params(a), tiles,
                                                                     a.rho_acc, a.Vacc, a.nao);
    } else {
        cudaFuncSetAttribute(k_umma<MODE_RHO, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        k_umma<MODE_RHO, false><<<dim3(tiles, a.nblk), 128, smem, s>>>(a.g, a.blk0, a.ws, umma_params(a), tiles,
                                                                      a.rho_acc, a.Vacc, a.nao);
    }
}

void mixed_functional(const MixedArgs& a, cudaStream_t s) {
    if (functional_is_gga(a.fn)) {
        k_functional_mixed<true><<<a.nblk, BLOCK_PTS, 0, s>>>(a.g, a.blk0, a.fn, a.incremental, a.rho_cut, a.rho_acc,
                                                              a.rho_store, a.coef, a.blk_sum);
        k_pack_z<true><<<a.nblk, 256, 0, s>>>(a.g, a.blk0, a.coef, a.ws);
    } else {
        k_functional_mixed<false><<<a.nblk, BLOCK_PTS, 0, s>>>(a.g, a.blk0, a.fn, a.incremental, a.rho_cut, a.rho_acc,
                                                               a.rho_store, a.coef, a.blk_sum);
        k_pack_z<false><<<a.nblk, 256, 0, s>>>(a.g, a.blk0, a.coef, a.ws);
    }
}

void mixed_vxc(const MixedArgs& a, cudaStream_t s) {
    const int tiles = a.max_nbp / umma::TILE_ROWS;
    const size_t smem = umma_smem_bytes(a.nterms);
    cudaFuncSetAttribute(k_umma<MODE_VXC, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_umma<MODE_VXC, false><<<dim3(tiles * tiles, a.nblk), 128, smem, s>>>(a.g, a.blk0, a.ws, umma_params(a), tiles,
                                                                          a.rho_acc, a.Vacc, a.nao);
}

}  // namespace pdfxc
