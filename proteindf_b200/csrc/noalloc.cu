// pdfxc_build_vxc_noalloc: the FP64 XC build for callers that cannot allocate
// device memory.
//
// Some callers cannot call cudaMalloc at all: a host program whose device memory
// is owned by a pool or arena it does not control, code that runs inside a
// region where allocation is forbidden (a memory-capped sandbox, a real-time
// loop that must not block in the allocator), or a plugin whose host process
// has already reserved the whole device. They hold their inputs and outputs in
// device memory already and only need the kernels to run. For them this entry
// point takes every operand as a device pointer and keeps all of its
// intermediates in one file-scope __device__ array (g_noalloc_scratch below,
// PDFXC_NOALLOC_SCRATCH_BYTES = 32 MiB). It calls no cudaMalloc, cudaFree or
// allocating library routine.
//
// Costs and rules of the shared array:
//  * every GPU that loads this library holds the 32 MiB until the process exits;
//  * every call on a device uses the same array, and it keeps the contents of
//    the last call: the accumulators are cleared at the start of each call;
//  * calls whose work overlaps on the GPU race on the array: the entry point
//    synchronises its stream before returning, and two host threads must not
//    call it concurrently on the same device;
//  * the first call on a device looks up the array's device address (once per
//    device, with that device current); that first call should come before any
//    stream capture the caller does.
//
// Limits: n_ao <= 256 and nshell <= 256 (the intermediates of one 128-point
// block of the basis must fit the array several times over); larger inputs
// are rejected with PDFXC_ERR_ARG. Every block uses the whole basis (no
// screening), the density is recomputed from PA (no incremental update).
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "functional.cuh"
#include "pdfxc_internal.cuh"

#define PDFXC_NOALLOC_SCRATCH_BYTES (32u << 20)
#define PDFXC_NOALLOC_MAX_AO 256
#define PDFXC_NOALLOC_MAX_SHELL 256
#define PDFXC_NOALLOC_MAX_DEVICES 64

// The scratch of pdfxc_build_vxc_noalloc. In host code this name is only a
// host-side stand-in for the symbol: its device address comes from
// cudaGetSymbolAddress (see scratch_address below).
static __device__ __align__(256) unsigned char g_noalloc_scratch[PDFXC_NOALLOC_SCRATCH_BYTES];

namespace {

using pdfxc::BLOCK_PTS;
using pdfxc::BlockMeta;

std::mutex g_addr_mutex;
void* g_addr[PDFXC_NOALLOC_MAX_DEVICES] = {nullptr};

// Device address of the scratch array on the current device (looked up once per device).
cudaError_t scratch_address(int device, unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_addr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_addr[device]);
    return cudaSuccess;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Shell prefix sums and the block-independent index lists (every block uses
// all shells, local AO row = global AO index).
__global__ void k_noalloc_basis(int nshell, const int* sh_l, const int* sh_nprim, int* sh_p0, int* sh_ao0,
                                int* blk_shells, int* blk_shell_row, int* blk_aos, int nao) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        int p = 0, a = 0;
        for (int s = 0; s < nshell; ++s) {
            sh_p0[s] = p, sh_ao0[s] = a;
            blk_shells[s] = s, blk_shell_row[s] = a;
            p += sh_nprim[s];
            a += 2 * sh_l[s] + 1;
        }
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nao; i += gridDim.x * blockDim.x) blk_aos[i] = i;
}

// Block metadata and the padded structure-of-arrays points of one chunk.
__global__ void k_noalloc_chunk(const double* xyzw, int64_t npts, int64_t p0, int nblk, int nshell, int nao, int nbp,
                                int64_t ws_block, BlockMeta* meta, double* px, double* py, double* pz, double* pw) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)nblk * BLOCK_PTS;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int b = (int)(e / BLOCK_PTS), j = (int)(e % BLOCK_PTS);
        const int64_t i = p0 + e;
        const int64_t first = p0 + (int64_t)b * BLOCK_PTS;
        const int64_t src = i < npts ? i : first;  // padding slots reuse the block's first point, weight 0
        px[e] = xyzw[4 * src], py[e] = xyzw[4 * src + 1], pz[e] = xyzw[4 * src + 2];
        pw[e] = i < npts ? xyzw[4 * src + 3] : 0.0;
        if (j == 0) {
            const int64_t left = npts - first;
            meta[b] = BlockMeta{0, nshell, 0, nao, nbp, (int)(left < BLOCK_PTS ? left : BLOCK_PTS), (int)b, 1,
                                (int64_t)b * ws_block};
        }
    }
}

// Adds this chunk's block sums (Exc, electron count) to the running totals, in block order.
__global__ void k_noalloc_sums(const double* blk_sum, int nblk, double* totals) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double e = 0.0, n = 0.0;
        for (int b = 0; b < nblk; ++b) e += blk_sum[2 * b], n += blk_sum[2 * b + 1];
        totals[0] += e, totals[1] += n;
    }
}

__global__ void k_noalloc_symmetrize(const double* Vacc, double* V, int nao) {
    const int64_t n2 = (int64_t)nao * nao;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n2; e += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(e / nao), j = (int)(e % nao);
        V[e] = Vacc[e] + Vacc[(int64_t)j * nao + i];
    }
}

}  // namespace

extern "C" pdfxc_status pdfxc_build_vxc_noalloc(int device, int functional, int natom, const double* d_atom_xyz,
                                                int nshell, const int* d_shell_atom, const int* d_shell_l,
                                                const int* d_shell_nprim, const double* d_prim_exp,
                                                const double* d_prim_coef, int nao, int64_t npts,
                                                const double* d_xyzw, const double* d_PA, double* d_V,
                                                double* d_exc_nelec, void* stream) {
    if (functional < PDFXC_SVWN || functional > PDFXC_PBE || natom <= 0 || nshell <= 0 || nao <= 0 || npts <= 0)
        return PDFXC_ERR_ARG;
    if (nao > PDFXC_NOALLOC_MAX_AO || nshell > PDFXC_NOALLOC_MAX_SHELL) return PDFXC_ERR_ARG;
    if (!d_atom_xyz || !d_shell_atom || !d_shell_l || !d_shell_nprim || !d_prim_exp || !d_prim_coef || !d_xyzw ||
        !d_PA || !d_V || !d_exc_nelec)
        return PDFXC_ERR_ARG;
    if (device < 0 || device >= PDFXC_NOALLOC_MAX_DEVICES) return PDFXC_ERR_ARG;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return PDFXC_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return PDFXC_ERR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    pdfxc_status st = PDFXC_OK;
    do {
        // the AO count implied by the shells must match n_ao: a small device -> host copy (no
        // allocation) ordered on the caller's stream, after the caller's writes of the shell table
        int h_l[PDFXC_NOALLOC_MAX_SHELL];
        if (cudaMemcpyAsync(h_l, d_shell_l, sizeof(int) * nshell, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            st = PDFXC_ERR_CUDA;
            break;
        }
        int count = 0;
        for (int i = 0; i < nshell; ++i) {
            if (h_l[i] < 0 || h_l[i] > 2) count = -1000000;
            count += 2 * h_l[i] + 1;
        }
        if (count != nao) {
            st = PDFXC_ERR_ARG;
            break;
        }
        unsigned char* base = nullptr;
        if (scratch_address(device, &base) != cudaSuccess) {
            st = PDFXC_ERR_CUDA;
            break;
        }
        const bool gga = pdfxc::functional_is_gga(functional);
        const int nbp = nao > 64 ? (nao + 63) / 64 * 64 : 64;
        const size_t ws_block = pdfxc::block_ws_doubles(nbp, true) * sizeof(double);
        // the carve-outs of the array for `chunk` blocks per pass; each starts on a 256-byte boundary
        struct Layout {
            double *Vacc, *totals, *px, *py, *pz, *pw, *rho, *coef, *blk_sum;
            int *sh_p0, *sh_ao0, *blk_shells, *blk_shell_row, *blk_aos;
            BlockMeta* meta;
            char* ws;
            size_t end;
        };
        auto layout = [&](int chunk) {
            Layout L;
            size_t off = 0;
            auto take = [&](size_t bytes) {
                unsigned char* p = base + off;
                off = align256(off + bytes);
                return p;
            };
            L.Vacc = reinterpret_cast<double*>(take(sizeof(double) * nao * nao));
            L.totals = reinterpret_cast<double*>(take(sizeof(double) * 2));
            L.sh_p0 = reinterpret_cast<int*>(take(sizeof(int) * nshell));
            L.sh_ao0 = reinterpret_cast<int*>(take(sizeof(int) * nshell));
            L.blk_shells = reinterpret_cast<int*>(take(sizeof(int) * nshell));
            L.blk_shell_row = reinterpret_cast<int*>(take(sizeof(int) * nshell));
            L.blk_aos = reinterpret_cast<int*>(take(sizeof(int) * nao));
            L.meta = reinterpret_cast<BlockMeta*>(take(sizeof(BlockMeta) * chunk));
            L.px = reinterpret_cast<double*>(take(sizeof(double) * BLOCK_PTS * chunk));
            L.py = reinterpret_cast<double*>(take(sizeof(double) * BLOCK_PTS * chunk));
            L.pz = reinterpret_cast<double*>(take(sizeof(double) * BLOCK_PTS * chunk));
            L.pw = reinterpret_cast<double*>(take(sizeof(double) * BLOCK_PTS * chunk));
            L.rho = reinterpret_cast<double*>(take(sizeof(double) * BLOCK_PTS * 4 * chunk));
            L.coef = reinterpret_cast<double*>(take(sizeof(double) * BLOCK_PTS * 4 * chunk));
            L.blk_sum = reinterpret_cast<double*>(take(sizeof(double) * 2 * chunk));
            L.ws = reinterpret_cast<char*>(take(ws_block * chunk));
            L.end = off;
            return L;
        };
        // the largest block count per pass whose layout fits the array (padding included)
        const size_t per_block = ws_block + sizeof(BlockMeta) + sizeof(double) * BLOCK_PTS * (4 + 4 + 4) +
                                 2 * sizeof(double);
        int chunk = (int)(PDFXC_NOALLOC_SCRATCH_BYTES / per_block);
        while (chunk > 0 && layout(chunk).end > PDFXC_NOALLOC_SCRATCH_BYTES) --chunk;
        if (chunk < 1) {
            st = PDFXC_ERR_ARG;
            break;
        }
        const Layout L = layout(chunk);
        double* Vacc = L.Vacc;
        double* totals = L.totals;
        int *sh_p0 = L.sh_p0, *sh_ao0 = L.sh_ao0, *blk_shells = L.blk_shells, *blk_shell_row = L.blk_shell_row;
        int* blk_aos = L.blk_aos;
        BlockMeta* meta = L.meta;
        double *px = L.px, *py = L.py, *pz = L.pz, *pw = L.pw, *rho = L.rho, *coef = L.coef, *blk_sum = L.blk_sum;
        char* ws = L.ws;
        // clear what must start at zero: the Vxc accumulator and the totals
        if (cudaMemsetAsync(Vacc, 0, sizeof(double) * nao * nao, s) != cudaSuccess ||
            cudaMemsetAsync(totals, 0, sizeof(double) * 2, s) != cudaSuccess) {
            st = PDFXC_ERR_CUDA;
            break;
        }
        k_noalloc_basis<<<1, 256, 0, s>>>(nshell, d_shell_l, d_shell_nprim, sh_p0, sh_ao0, blk_shells, blk_shell_row,
                                          blk_aos, nao);
        if (cudaPeekAtLastError() != cudaSuccess) {
            st = PDFXC_ERR_CUDA;
            break;
        }
        const pdfxc::BasisView bv{d_atom_xyz, d_shell_atom, d_shell_l, d_shell_nprim, sh_p0, sh_ao0, d_prim_exp,
                                  d_prim_coef};
        const pdfxc::GridView gv{px, py, pz, pw, meta, blk_shells, blk_shell_row, blk_aos};
        const int64_t nblk_total = (npts + BLOCK_PTS - 1) / BLOCK_PTS;
        for (int64_t b0 = 0; b0 < nblk_total; b0 += chunk) {
            const int nb = (int)((nblk_total - b0) < chunk ? (nblk_total - b0) : chunk);
            k_noalloc_chunk<<<(nb * BLOCK_PTS + 255) / 256, 256, 0, s>>>(d_xyzw, npts, b0 * BLOCK_PTS, nb, nshell, nao,
                                                                         nbp, (int64_t)ws_block, meta, px, py, pz, pw);
            pdfxc::launch_ao_eval(bv, gv, 0, nb, gga, ws, 0, s);
            pdfxc::launch_gemm_x(gv, d_PA, nao, 0, nb, nbp, gga ? 4 : 1, ws, s);
            pdfxc::launch_rho_functional(gv, 0, nb, functional, false, 1e-16, ws, rho, coef, blk_sum, s);
            pdfxc::launch_gemm_v(gv, 0, nb, nbp, gga, coef, ws, Vacc, nao, s);
            k_noalloc_sums<<<1, 32, 0, s>>>(blk_sum, nb, totals);
            if (cudaPeekAtLastError() != cudaSuccess) {  // this pass's launches (configuration, resources)
                st = PDFXC_ERR_CUDA;
                break;
            }
        }
        if (st != PDFXC_OK) break;
        k_noalloc_symmetrize<<<148 * 4, 256, 0, s>>>(Vacc, d_V, nao);
        if (cudaPeekAtLastError() != cudaSuccess ||
            cudaMemcpyAsync(d_exc_nelec, totals, 2 * sizeof(double), cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            st = PDFXC_ERR_CUDA;
            break;
        }
    } while (false);
    cudaSetDevice(prev);
    return st;
}
