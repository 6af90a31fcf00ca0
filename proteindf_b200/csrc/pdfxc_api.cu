// libpdfxc C ABI: context, system and grid set-up (spatial blocking and
// per-block basis screening, once per geometry) and the per-iteration build
// orchestration. Every entry point catches C++ exceptions and reports a status.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <map>
#include <mutex>
#include <new>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "functional.cuh"
#include "pdfxc_internal.cuh"

using pdfxc::BLOCK_PTS;
using pdfxc::BlockMeta;
using pdfxc::Chunk;

namespace {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// An input the library cannot take (status PDFXC_ERR_UNSUPPORTED).
struct Unsupported : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// After a kernel launch: a launch that failed (configuration, resources) names itself in the
// error, also while a graph is being captured. No synchronisation.
#define PDFXC_LAUNCHED(what)                                                                        \
    do {                                                                                            \
        cudaError_t e_ = cudaPeekAtLastError();                                                     \
        if (e_ != cudaSuccess) throw CudaError(std::string("launch of ") + (what) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define PDFXC_CUDA(call)                                                                            \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            throw CudaError(std::string(#call) + ": " + cudaGetErrorString(e_));                    \
    } while (0)

template <class T>
void dev_alloc(T** p, size_t n) {
    if (*p) cudaFree(*p);
    *p = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        throw std::bad_alloc();
    }
}

template <class T>
void upload(T** p, const std::vector<T>& v, cudaStream_t s) {
    dev_alloc(p, v.size());
    if (!v.empty()) PDFXC_CUDA(cudaMemcpyAsync(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

// cudaMemsetAsync in pieces of at most 1 GiB (the 18,600-AO matrices are 2.8 GB)
void memset_async(void* p, size_t bytes, cudaStream_t s) {
    constexpr size_t piece = size_t(1) << 30;
    char* c = static_cast<char*>(p);
    for (size_t off = 0; off < bytes; off += piece)
        PDFXC_CUDA(cudaMemsetAsync(c + off, 0, std::min(piece, bytes - off), s));
}

template <class T>
void dev_free(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

template <class F>
pdfxc_status guarded(pdfxc_ctx* ctx, F&& f) {
    if (!ctx) return PDFXC_ERR_ARG;
    try {
        cudaSetDevice(ctx->device);
        return f();
    } catch (const std::bad_alloc&) {
        ctx->err = "device or host allocation failed";
        return PDFXC_ERR_NOMEM;
    } catch (const CudaError& e) {
        ctx->err = e.what();
        return PDFXC_ERR_CUDA;
    } catch (const Unsupported& e) {
        ctx->err = e.what();
        return PDFXC_ERR_UNSUPPORTED;
    } catch (const std::exception& e) {
        ctx->err = e.what();
        return PDFXC_ERR_ARG;
    }
}

// Distance beyond which a shell's value and gradient bounds both stay below
// `cutoff`: bound(r) = sum_k |c_k| e^{-a_k r^2} max(r^L, L r^(L-1) + 2 a_k r^(L+1)).
double shell_cutoff_radius(int L, const double* e, const double* c, int np, double cutoff) {
    double R = 0.0;
    for (double r = 60.0; r > 0.0; r -= 0.01) {
        double b = 0.0;
        for (int k = 0; k < np; ++k) {
            const double rl = std::pow(r, L);
            const double g = std::max(rl, (L > 0 ? L * std::pow(r, L - 1) : 0.0) + 2.0 * e[k] * rl * r);
            b += std::fabs(c[k]) * std::exp(-e[k] * r * r) * g;
        }
        if (b >= cutoff) {
            R = r + 0.01;
            break;
        }
    }
    return R;
}

uint64_t spread3(uint64_t v) {
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffULL;
    v = (v | v << 16) & 0x1f0000ff0000ffULL;
    v = (v | v << 8) & 0x100f00f00f00f00fULL;
    v = (v | v << 4) & 0x10c30c30c30c30c3ULL;
    v = (v | v << 2) & 0x1249249249249249ULL;
    return v;
}

// Host threads for the grid planner: fn(lo, hi, t) over [0, n) in contiguous ranges, one per
// thread (t = the range's index); small ranges run on the calling thread.
unsigned host_threads() { return std::min(16u, std::max(1u, std::thread::hardware_concurrency())); }

template <class F>
void parallel_ranges(int64_t n, int64_t min_per_thread, F&& fn) {
    const int64_t nt = std::max<int64_t>(1, std::min<int64_t>(host_threads(), n / std::max<int64_t>(1, min_per_thread)));
    if (nt == 1) {
        fn((int64_t)0, n, 0);
        return;
    }
    std::vector<std::thread> th;
    std::vector<std::exception_ptr> err(nt);  // an exception of a range is rethrown on the calling thread
    for (int64_t t = 0; t < nt; ++t)
        th.emplace_back([&, t]() {
            try {
                fn(n * t / nt, n * (t + 1) / nt, (int)t);
            } catch (...) {
                err[t] = std::current_exception();
            }
        });
    for (auto& x : th) x.join();
    for (auto& e : err)
        if (e) std::rethrow_exception(e);
}

// std::sort's result (a total order: the keys are distinct) from sorted ranges merged pairwise,
// each range and each merge on its own thread.
template <class T>
void parallel_sort(T* a, int64_t n) {
    const int64_t nt = std::min<int64_t>(host_threads(), std::max<int64_t>(1, n / (1 << 18)));
    if (nt <= 1) {
        std::sort(a, a + n);
        return;
    }
    std::vector<int64_t> cut(nt + 1);
    for (int64_t t = 0; t <= nt; ++t) cut[t] = n * t / nt;
    parallel_ranges(nt, 1, [&](int64_t lo, int64_t hi, int) {
        for (int64_t t = lo; t < hi; ++t) std::sort(a + cut[t], a + cut[t + 1]);
    });
    std::vector<T> tmp(n);
    T *src = a, *dst = tmp.data();
    for (int64_t w = 1; w < nt; w *= 2) {
        std::vector<std::thread> th;
        for (int64_t t = 0; t < nt; t += 2 * w) {
            const int64_t l = cut[t], m = cut[std::min(nt, t + w)], r = cut[std::min(nt, t + 2 * w)];
            th.emplace_back([=]() { std::merge(src + l, src + m, src + m, src + r, dst + l); });
        }
        for (auto& x : th) x.join();
        std::swap(src, dst);
    }
    if (src != a) std::copy(src, src + n, a);
}

pdfxc::BasisView basis_view(const pdfxc_ctx* c) {
    return {c->d_atom_xyz, c->d_sh_atom, c->d_sh_l, c->d_sh_nprim, c->d_sh_p0, c->d_sh_ao0, c->d_p_exp, c->d_p_coef};
}

pdfxc::GridView grid_view(const pdfxc_ctx* c) {
    return {c->d_px,         c->d_py,         c->d_pz,          c->d_pw,         c->d_meta,
            c->d_blk_shells, c->d_blk_shell_row, c->d_blk_aos, c->d_blk_row_info, c->d_blk_row_geom,
            c->d_xtiles,     c->d_vtiles,        c->h_xtile0.empty() ? nullptr : c->h_xtile0.data(),
            c->h_vtile0.empty() ? nullptr : c->h_vtile0.data()};
}

void drop_graph(pdfxc_ctx* c) {
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    c->graph_exec = nullptr;
    c->graph_fn = c->graph_inc = -1;
    c->graph_P = nullptr;
}

void free_plan(pdfxc::Plan& p) {
    dev_free(p.d_meta);
    if (p.d_ws) cudaFree(p.d_ws);
    p.d_ws = nullptr;
    p.ws_bytes = 0;
    p.planes = -1;
    p.chunks.clear();
}

// Per-block workspace offsets and chunks for `planes` FP64 planes of nbp x BLOCK_PTS per
// block, within the workspace budget; recomputed only when the plane count changes.
void ensure_plan(pdfxc_ctx* ctx, pdfxc::Plan& p, int planes) {
    if (p.planes == planes) return;
    std::vector<BlockMeta> gm = ctx->h_meta;
    const size_t per_plane = sizeof(double) * BLOCK_PTS;
    p.chunks.clear();
    size_t off = 0, max_ws = 0;
    Chunk cur{0, 0, 0, 0};
    for (int b = 0; b < ctx->nblk; ++b) {
        const size_t need = per_plane * (size_t)gm[b].nbp * planes;
        if (off + need > ctx->opt.workspace_bytes && b > cur.b0) {
            cur.b1 = b;
            cur.ws_bytes = off;
            p.chunks.push_back(cur);
            max_ws = std::max(max_ws, off);
            cur = Chunk{b, b, 0, 0};
            off = 0;
        }
        gm[b].ws = (int64_t)off;
        off += need;
        cur.max_nbp = std::max(cur.max_nbp, gm[b].nbp);
    }
    cur.b1 = ctx->nblk;
    cur.ws_bytes = off;
    p.chunks.push_back(cur);
    max_ws = std::max(max_ws, off);
    upload(&p.d_meta, gm, ctx->stream);
    if (max_ws > p.ws_bytes) {
        if (p.d_ws) cudaFree(p.d_ws);
        p.d_ws = nullptr;
        p.ws_bytes = 0;
        if (cudaMalloc(&p.d_ws, max_ws) != cudaSuccess) {
            p.d_ws = nullptr;
            p.planes = -1;
            throw std::bad_alloc();
        }
        p.ws_bytes = max_ws;
    }
    p.planes = planes;
}

void free_grid(pdfxc_ctx* c) {
    drop_graph(c);
    dev_free(c->d_px), dev_free(c->d_py), dev_free(c->d_pz), dev_free(c->d_pw);
    dev_free(c->d_meta), dev_free(c->d_blk_shells), dev_free(c->d_blk_shell_row), dev_free(c->d_blk_aos);
    dev_free(c->d_blk_row_info), dev_free(c->d_blk_row_geom);
    dev_free(c->d_seg_blk), dev_free(c->d_mol_sums), dev_free(c->d_grp);
    dev_free(c->d_items), dev_free(c->d_counters);
    c->seg_blk.clear();
    c->h_grp.clear();
    dev_free(c->d_rho), dev_free(c->d_coef), dev_free(c->d_blk_sum), dev_free(c->d_rho_acc);
    if (c->d_ws) cudaFree(c->d_ws);
    c->d_ws = nullptr;
    c->h_owner.clear();
    dev_free(c->d_owner), dev_free(c->d_ao_atom), dev_free(c->d_grad);
    dev_free(c->d_fdens), dev_free(c->d_wslot), dev_free(c->d_brad), dev_free(c->d_pair);
    dev_free(c->d_wscratch);
    dev_free(c->d_xtiles), dev_free(c->d_vtiles);
    c->h_xtile0.clear(), c->h_vtile0.clear();
    free_plan(c->gplan);
    free_plan(c->uplan);
    dev_free(c->d_rho_b), dev_free(c->d_blk_sum_b);
    c->rho_spin = 0;
    c->nblk = 0;
    c->npts = 0;
    c->rho_valid = false;
}

}  // namespace

extern "C" {

void pdfxc_default_options(pdfxc_options* opt) {
    if (!opt) return;
    opt->precision = PDFXC_PRECISION_FP64;
    opt->block_points = BLOCK_PTS;
    opt->ao_cutoff = 1e-14;
    opt->rho_cutoff = 1e-16;
    opt->workspace_bytes = 0;
    opt->split_terms = 10;
    opt->group_blocks = 0;
    opt->vxc_stages = 0;
}

pdfxc_status pdfxc_create(pdfxc_ctx** out, int device, const pdfxc_options* opt) {
    if (!out) return PDFXC_ERR_ARG;
    *out = nullptr;
    pdfxc_ctx* c = new (std::nothrow) pdfxc_ctx();
    if (!c) return PDFXC_ERR_NOMEM;
    pdfxc_default_options(&c->opt);
    if (opt) c->opt = *opt;
    if (c->opt.block_points <= 0 || c->opt.block_points > BLOCK_PTS) c->opt.block_points = BLOCK_PTS;
    if (c->opt.workspace_bytes == 0) c->opt.workspace_bytes = size_t(4) << 30;
    if (c->opt.split_terms != 3 && c->opt.split_terms != 6 && c->opt.split_terms != 10) c->opt.split_terms = 10;
    if (c->opt.precision != PDFXC_PRECISION_FP64 && c->opt.precision != PDFXC_PRECISION_MIXED) {
        delete c;
        return PDFXC_ERR_ARG;
    }
    c->device = device;
    if (const char* g = std::getenv("PDFXC_GRAPH")) c->use_graph = std::atoi(g) != 0;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        delete c;
        return PDFXC_ERR_CUDA;
    }
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return PDFXC_ERR_CUDA;
    }
    for (auto& e : c->ev) cudaEventCreate(&e);
    if (cudaMalloc(&c->d_scalars, 2 * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&c->d_err, sizeof(int)) != cudaSuccess || cudaMemset(c->d_err, 0, sizeof(int)) != cudaSuccess) {
        pdfxc_destroy(c);
        return PDFXC_ERR_NOMEM;
    }
    *out = c;
    return PDFXC_OK;
}

}  // extern "C"

namespace {

// The host copy of a system (atoms, shells, primitives) with its AO offsets; no device work.
pdfxc_status set_host_system(pdfxc_ctx* ctx, int natom, const double* atom_xyz, const int* atom_z, int nshell,
                             const int* shell_atom, const int* shell_l, const int* shell_nprim,
                             const double* prim_exp, const double* prim_coef) {
    if (natom <= 0 || nshell <= 0 || !atom_xyz || !shell_atom || !shell_l || !shell_nprim || !prim_exp || !prim_coef) {
        ctx->err = "pdfxc_set_system: empty system or null pointer";
        return PDFXC_ERR_ARG;
    }
    for (int s = 0; s < nshell; ++s)
        if (shell_l[s] < 0 || shell_l[s] > 2 || shell_nprim[s] <= 0 || shell_atom[s] < 0 || shell_atom[s] >= natom) {
            ctx->err = "pdfxc_set_system: shell " + std::to_string(s) + " out of range (only s, p, d shells)";
            return PDFXC_ERR_ARG;
        }
    ctx->natom = natom;
    ctx->nshell = nshell;
    ctx->h_atom_xyz.assign(atom_xyz, atom_xyz + 3 * natom);
    ctx->h_atom_z.assign(natom, 0);
    if (atom_z) ctx->h_atom_z.assign(atom_z, atom_z + natom);
    ctx->h_sh_atom.assign(shell_atom, shell_atom + nshell);
    ctx->h_sh_l.assign(shell_l, shell_l + nshell);
    ctx->h_sh_nprim.assign(shell_nprim, shell_nprim + nshell);
    ctx->h_sh_p0.resize(nshell);
    ctx->h_sh_ao0.resize(nshell);
    int np = 0, ao = 0;
    for (int s = 0; s < nshell; ++s) {
        ctx->h_sh_p0[s] = np;
        ctx->h_sh_ao0[s] = ao;
        np += shell_nprim[s];
        ao += 2 * shell_l[s] + 1;
    }
    ctx->nao = ao;
    ctx->h_p_exp.assign(prim_exp, prim_exp + np);
    ctx->h_p_coef.assign(prim_coef, prim_coef + np);
    // primitives by ascending exponent within each shell, the order the reference sums them in
    // (TlOrbitalInfoObject::setCGTO, src/libpdf/TlOrbitalInfoObject.cpp:95); the kernels stop at
    // the first primitive past the cut alpha r^2 > 30
    for (int s = 0; s < nshell; ++s) {
        const int p0 = ctx->h_sh_p0[s], n = shell_nprim[s];
        std::vector<std::pair<double, double>> pr(n);
        for (int k = 0; k < n; ++k) pr[k] = {ctx->h_p_exp[p0 + k], ctx->h_p_coef[p0 + k]};
        std::stable_sort(pr.begin(), pr.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (int k = 0; k < n; ++k) ctx->h_p_exp[p0 + k] = pr[k].first, ctx->h_p_coef[p0 + k] = pr[k].second;
    }
    return PDFXC_OK;
}

}  // namespace

extern "C" {

pdfxc_status pdfxc_set_system(pdfxc_ctx* ctx, int natom, const double* atom_xyz, const int* atom_z, int nshell,
                              const int* shell_atom, const int* shell_l, const int* shell_nprim,
                              const double* prim_exp, const double* prim_coef) {
    return guarded(ctx, [&]() -> pdfxc_status {
        if (const pdfxc_status st = set_host_system(ctx, natom, atom_xyz, atom_z, nshell, shell_atom, shell_l,
                                                    shell_nprim, prim_exp, prim_coef))
            return st;
        dev_free(ctx->d_nbr_idx), dev_free(ctx->d_nbr_dist);  // neighbour lists of the old geometry
        const int ao = ctx->nao;
        // dummy atoms (atomic number <= 0; only when atomic numbers are given): the Becke partition
        // leaves them out as partners (DfGenerateGrid::Ps_uij, src/libpdf/DfGenerateGrid.cpp:2056)
        dev_free(ctx->d_ghost);
        if (atom_z && std::any_of(atom_z, atom_z + natom, [](int z) { return z <= 0; })) {
            std::vector<int> ghost(natom);
            for (int a = 0; a < natom; ++a) ghost[a] = atom_z[a] <= 0 ? 1 : 0;
            upload(&ctx->d_ghost, ghost, ctx->stream);
        }
        cudaStream_t s = ctx->stream;
        upload(&ctx->d_atom_xyz, ctx->h_atom_xyz, s);
        upload(&ctx->d_sh_atom, ctx->h_sh_atom, s);
        upload(&ctx->d_sh_l, ctx->h_sh_l, s);
        upload(&ctx->d_sh_nprim, ctx->h_sh_nprim, s);
        upload(&ctx->d_sh_p0, ctx->h_sh_p0, s);
        upload(&ctx->d_sh_ao0, ctx->h_sh_ao0, s);
        upload(&ctx->d_p_exp, ctx->h_p_exp, s);
        upload(&ctx->d_p_coef, ctx->h_p_coef, s);
        const size_t n2 = (size_t)ao * ao;
        dev_alloc(&ctx->d_P, n2);
        dev_alloc(&ctx->d_V, n2);
        dev_alloc(&ctx->d_Vacc, n2);
        dev_free(ctx->d_Vprev);  // the delta history belongs to the old system
        ctx->vprev_iter = 0;
        dev_alloc(&ctx->d_p_rowexp, (size_t)ao);
        dev_free(ctx->d_p_words);
        dev_free(ctx->d_row_cols);  // a batch sets it after this call
        if (ctx->opt.precision == PDFXC_PRECISION_MIXED && ctx->opt.split_terms == 10) dev_alloc(&ctx->d_p_words, n2);
        dev_free(ctx->d_P_b), dev_free(ctx->d_V_b), dev_free(ctx->d_Vacc_b);  // open shell: sized on first use
        PDFXC_CUDA(cudaStreamSynchronize(s));
        free_grid(ctx);
        return PDFXC_OK;
    });
}

}  // extern "C"

namespace {

// Points [p0, p1) of the grid whose blocks are screened against shells [sh0, sh1):
// the whole grid for one molecule, one segment per molecule for a batch.
struct GridSegment {
    int64_t p0, p1;
    int sh0, sh1;
};

// Blocks of one group on the INT8 path: the Vxc contraction of a group runs over all its
// points before one epilogue, and the group's blocks share one screened basis. Shell
// screening radii, not the point count, set a block's basis, so a group of four blocks
// screens in about as many AOs as one block: on a 100-atom chain (cc-pVDZ, 99 x 590 grid)
// groups of 4 x 128 points raise the contraction work by 18 % and cut the per-block
// epilogue work (sum of nb^2) by 3.4x.
int group_blocks(const pdfxc_ctx* ctx) {
    if (!(ctx->opt.precision == PDFXC_PRECISION_MIXED && ctx->opt.split_terms == 10)) return 1;
    return ctx->tuned_group > 0 ? ctx->tuned_group : 4;
}

// Tile and group shapes chosen by pdfxc_autotune, kept for the process under the workload's class
// (precision, operand split, batch or single molecule, and the AO and point counts to a factor of
// two), so that later contexts of the same class start from them.
struct TuneChoice {
    int group_blocks, vxc_stages;
};
std::mutex g_tune_mutex;
std::map<std::string, TuneChoice> g_tune_cache;

std::string tune_class(const pdfxc_ctx* ctx, int64_t npts, size_t nseg) {
    auto lg = [](double v) { return v > 1.0 ? (int)std::floor(std::log2(v)) : 0; };
    return std::to_string(ctx->opt.precision) + "/" + std::to_string(ctx->opt.split_terms) + "/" +
           std::to_string(nseg > 1) + "/" + std::to_string(lg(ctx->nao)) + "/" + std::to_string(lg((double)npts));
}

// The group size and Vxc stage count of a new grid: the options' explicit values, else the tuned
// ones of the workload's class, else 4 and 3.
void resolve_shapes(pdfxc_ctx* ctx, int64_t npts, size_t nseg) {
    int g = ctx->opt.group_blocks, st = ctx->opt.vxc_stages;
    if (g < 1 || g > 4 || (st != 2 && st != 3)) {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        const auto it = g_tune_cache.find(tune_class(ctx, npts, nseg));
        if (it != g_tune_cache.end()) {
            if (g < 1 || g > 4) g = it->second.group_blocks;
            if (st != 2 && st != 3) st = it->second.vxc_stages;
        }
    }
    ctx->tuned_group = (g >= 1 && g <= 4) ? g : 4;
    ctx->tuned_stages = (st == 2 || st == 3) ? st : 3;
}

// Spatial blocks and basis screening, once per geometry: within each segment the points
// are put in Morton order over the segment's bounding box and cut into groups of up to
// group_blocks x block_points consecutive points, each group into blocks of block_points;
// every group keeps the shells of its segment whose value/gradient envelope reaches
// ao_cutoff at the group's nearest point.
// The host side of a blocked grid (plan_grid), before it is uploaded.
struct HostGrid {
    std::vector<double> px, py, pz, pw;
    std::vector<int> shells, rows, aos, row_info, grp_blk;
    int nblk = 0, ngrp = 0, max_nb = 0;
    double flops = 0.0, sum_nb = 0.0;
    size_t max_ws = 0;
    bool mixed = false;
};

void plan_grid(pdfxc_ctx* ctx, int64_t npts, const double* xyzw, const int* atom,
               const std::vector<GridSegment>& segs, HostGrid& G) {
    ctx->h_owner.clear();
    const int bp = ctx->opt.block_points;
    const int gb = group_blocks(ctx);
    // 1. spatial order: Morton code over each segment's bounding box; a group takes up to
    // gb * block_points consecutive points and is closed early when its bounding-box diagonal
    // would pass kMaxBlockExtent, so that it never straddles two distant regions (on sparse outer
    // grid shells a 128-point run of the Z curve can span 100 bohr and screen in thousands of AOs)
    constexpr double kMaxBlockExtent = 12.0;  // bohr
    std::vector<std::pair<uint64_t, int64_t>> key(npts);
    std::vector<std::pair<int64_t, int64_t>> runs;  // [i0, i1) of key per block
    std::vector<int> blk_seg;
    std::vector<int>& grp_blk = G.grp_blk;  // blocks of group k: [grp_blk[k], grp_blk[k+1])
    grp_blk.assign(1, 0);
    ctx->seg_blk.assign(1, 0);
    for (size_t si = 0; si < segs.size(); ++si) {
        const GridSegment& sg = segs[si];
        const int64_t np = sg.p1 - sg.p0;
        std::vector<std::array<double, 6>> box(host_threads());
        parallel_ranges(np, 1 << 16, [&](int64_t a, int64_t b, int t) {
            std::array<double, 6> bx = {1e300, 1e300, 1e300, -1e300, -1e300, -1e300};
            for (int64_t i = sg.p0 + a; i < sg.p0 + b; ++i)
                for (int k = 0; k < 3; ++k)
                    bx[k] = std::min(bx[k], xyzw[4 * i + k]), bx[3 + k] = std::max(bx[3 + k], xyzw[4 * i + k]);
            box[t] = bx;
        });
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (const auto& bx : box)
            for (int k = 0; k < 3; ++k) lo[k] = std::min(lo[k], bx[k]), hi[k] = std::max(hi[k], bx[3 + k]);
        const double span = std::max({hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2], 1e-12});
        parallel_ranges(np, 1 << 16, [&](int64_t a, int64_t b, int) {
            for (int64_t i = sg.p0 + a; i < sg.p0 + b; ++i) {
                const double* r = xyzw + 4 * i;
                uint64_t q[3];
                for (int k = 0; k < 3; ++k)
                    q[k] = (uint64_t)std::min(2097151.0, std::floor((r[k] - lo[k]) / span * 2097151.0));
                key[i] = {spread3(q[0]) | spread3(q[1]) << 1 | spread3(q[2]) << 2, i};
            }
        });
        parallel_sort(key.data() + sg.p0, np);
        // the points in that order, contiguous, for the sequential cut below
        std::vector<double> sxyz(3 * (size_t)np);
        parallel_ranges(np, 1 << 16, [&](int64_t a, int64_t b, int) {
            for (int64_t i = a; i < b; ++i)
                for (int k = 0; k < 3; ++k) sxyz[3 * i + k] = xyzw[4 * key[sg.p0 + i].second + k];
        });
        for (int64_t i0 = sg.p0; i0 < sg.p1;) {
            const double* r0 = &sxyz[3 * (i0 - sg.p0)];
            double blo[3] = {r0[0], r0[1], r0[2]}, bhi[3] = {r0[0], r0[1], r0[2]};
            int64_t i1 = i0 + 1;
            for (; i1 < sg.p1 && i1 - i0 < (int64_t)gb * bp; ++i1) {
                const double* r = &sxyz[3 * (i1 - sg.p0)];
                double d2 = 0.0;
                for (int k = 0; k < 3; ++k) {
                    const double l = std::min(blo[k], r[k]), h = std::max(bhi[k], r[k]);
                    d2 += (h - l) * (h - l);
                }
                if (d2 > kMaxBlockExtent * kMaxBlockExtent) break;
                for (int k = 0; k < 3; ++k) blo[k] = std::min(blo[k], r[k]), bhi[k] = std::max(bhi[k], r[k]);
            }
            for (int64_t j0 = i0; j0 < i1; j0 += bp) {
                runs.push_back({j0, std::min(i1, j0 + bp)});
                blk_seg.push_back((int)si);
            }
            grp_blk.push_back((int)runs.size());
            i0 = i1;
        }
        ctx->seg_blk.push_back((int)runs.size());
    }
    const int nblk = (int)runs.size();
    const int ngrp = (int)grp_blk.size() - 1;
    std::vector<double>&px = G.px, &py = G.py, &pz = G.pz, &pw = G.pw;
    px.assign((size_t)nblk * BLOCK_PTS, 0.0), py.assign(px.size(), 0.0), pz.assign(px.size(), 0.0),
        pw.assign(px.size(), 0.0);
    ctx->h_src.assign(px.size(), -1);
    if (atom) ctx->h_owner.assign(px.size(), 0);
    std::vector<double> cen(3 * (size_t)ngrp), rad(ngrp);
    ctx->h_meta.assign(nblk, BlockMeta{});
    parallel_ranges(ngrp, 256, [&](int64_t glo, int64_t ghi, int) {
        for (int64_t gi = glo; gi < ghi; ++gi) {
            // the group's centre and radius (screening)
            const int64_t g0 = runs[grp_blk[gi]].first, g1 = runs[grp_blk[gi + 1] - 1].second;
            double gc[3] = {0, 0, 0};
            for (int64_t i = g0; i < g1; ++i)
                for (int k = 0; k < 3; ++k) gc[k] += xyzw[4 * key[i].second + k];
            for (int k = 0; k < 3; ++k) gc[k] /= double(g1 - g0);
            double gr2 = 0.0;
            for (int64_t i = g0; i < g1; ++i) {
                const double* r = xyzw + 4 * key[i].second;
                gr2 = std::max(gr2, (r[0] - gc[0]) * (r[0] - gc[0]) + (r[1] - gc[1]) * (r[1] - gc[1]) +
                                        (r[2] - gc[2]) * (r[2] - gc[2]));
            }
            for (int k = 0; k < 3; ++k) cen[3 * gi + k] = gc[k];
            rad[gi] = std::sqrt(gr2);
            for (int b = grp_blk[gi]; b < grp_blk[gi + 1]; ++b) {
                const int64_t i0 = runs[b].first, i1 = runs[b].second;
                double c[3] = {0, 0, 0};
                for (int64_t i = i0; i < i1; ++i)
                    for (int k = 0; k < 3; ++k) c[k] += xyzw[4 * key[i].second + k];
                for (int k = 0; k < 3; ++k) c[k] /= double(i1 - i0);
                for (int j = 0; j < BLOCK_PTS; ++j) {
                    const size_t slot = (size_t)b * BLOCK_PTS + j;
                    const int64_t i = i0 + j;
                    if (i < i1) {
                        const double* r = xyzw + 4 * key[i].second;
                        px[slot] = r[0], py[slot] = r[1], pz[slot] = r[2], pw[slot] = r[3];
                        ctx->h_src[slot] = key[i].second;
                        if (atom) ctx->h_owner[slot] = atom[key[i].second];
                    } else {
                        px[slot] = c[0], py[slot] = c[1], pz[slot] = c[2], pw[slot] = 0.0;
                        if (atom) ctx->h_owner[slot] = atom[key[i0].second];  // padding: weight 0
                    }
                }
                ctx->h_meta[b].npts = (int)(i1 - i0);
                ctx->h_meta[b].lead = grp_blk[gi];
                ctx->h_meta[b].gn = grp_blk[gi + 1] - grp_blk[gi];
            }
        }
    });
    // 2. per-shell screening radius, then the per-block shell lists
    // (once per distinct shell: the shells of one element's basis repeat on every such atom)
    std::vector<double> Rs(ctx->nshell);
    std::map<std::vector<double>, double> radius_of;
    for (int sh = 0; sh < ctx->nshell; ++sh) {
        const int p0 = ctx->h_sh_p0[sh], np = ctx->h_sh_nprim[sh];
        std::vector<double> k = {(double)ctx->h_sh_l[sh]};
        k.insert(k.end(), ctx->h_p_exp.begin() + p0, ctx->h_p_exp.begin() + p0 + np);
        k.insert(k.end(), ctx->h_p_coef.begin() + p0, ctx->h_p_coef.begin() + p0 + np);
        auto it = radius_of.find(k);
        if (it == radius_of.end())
            it = radius_of.emplace(k, shell_cutoff_radius(ctx->h_sh_l[sh], &ctx->h_p_exp[p0], &ctx->h_p_coef[p0], np,
                                                          ctx->opt.ao_cutoff)).first;
        Rs[sh] = it->second;
    }
    std::vector<int>&shells = G.shells, &rows = G.rows, &aos = G.aos, &row_info = G.row_info;
    shells.clear(), rows.clear(), aos.clear(), row_info.clear();
    const bool mixed = ctx->opt.precision == PDFXC_PRECISION_MIXED;
    double flops = 0.0, sum_nb = 0.0;
    // Candidate shells of a group from a uniform grid of the segment's atoms (cell edge = the
    // largest screening radius): only atoms whose cell overlaps the cube of half-edge
    // rad + max Rs around the group's centre can pass the test below, and walking the candidates
    // in atom order visits their shells in shell order when each atom's shells are contiguous and
    // atoms ascend with the shell index (otherwise every shell of the segment is tested).
    struct AtomCells {
        bool ok = false;
        double lo[3], edge, reach;
        int dim[3];
        std::vector<int> start, atoms;    // CSR: the atoms of each cell, ascending
        std::vector<int> sh_first, sh_end;  // per atom of the segment: its shells
        int a0 = 0;
    };
    std::vector<AtomCells> cells(segs.size());
    auto build_cells = [&](size_t si) {
        AtomCells& C = cells[si];
        const GridSegment& sg = segs[si];
        if (sg.sh1 <= sg.sh0) return;
        const int a0 = ctx->h_sh_atom[sg.sh0], a1 = ctx->h_sh_atom[sg.sh1 - 1] + 1;
        for (int sh = sg.sh0 + 1; sh < sg.sh1; ++sh)
            if (ctx->h_sh_atom[sh] < ctx->h_sh_atom[sh - 1]) return;  // not in atom order
        C.a0 = a0;
        C.sh_first.assign(a1 - a0, 0), C.sh_end.assign(a1 - a0, 0);
        for (int sh = sg.sh1 - 1; sh >= sg.sh0; --sh) C.sh_first[ctx->h_sh_atom[sh] - a0] = sh;
        for (int sh = sg.sh0; sh < sg.sh1; ++sh) C.sh_end[ctx->h_sh_atom[sh] - a0] = sh + 1;
        double rmax = 0.0, hi[3];
        for (int sh = sg.sh0; sh < sg.sh1; ++sh) rmax = std::max(rmax, Rs[sh]);
        C.edge = std::max(rmax, 1.0), C.reach = rmax;
        for (int k = 0; k < 3; ++k) C.lo[k] = 1e300, hi[k] = -1e300;
        for (int a = a0; a < a1; ++a)
            for (int k = 0; k < 3; ++k)
                C.lo[k] = std::min(C.lo[k], ctx->h_atom_xyz[3 * a + k]), hi[k] = std::max(hi[k], ctx->h_atom_xyz[3 * a + k]);
        size_t ncell = 1;
        for (int k = 0; k < 3; ++k) C.dim[k] = (int)((hi[k] - C.lo[k]) / C.edge) + 1, ncell *= (size_t)C.dim[k];
        if (ncell > (size_t)1 << 22) return;  // too fine a grid: test every shell
        auto cell_of = [&](int a) {
            size_t c = 0;
            for (int k = 0; k < 3; ++k)
                c = c * C.dim[k] + std::min(C.dim[k] - 1, (int)((ctx->h_atom_xyz[3 * a + k] - C.lo[k]) / C.edge));
            return c;
        };
        C.start.assign(ncell + 1, 0);
        for (int a = a0; a < a1; ++a) ++C.start[cell_of(a) + 1];
        for (size_t c = 0; c < ncell; ++c) C.start[c + 1] += C.start[c];
        C.atoms.resize(a1 - a0);
        std::vector<int> fill(C.start.begin(), C.start.end() - 1);
        for (int a = a0; a < a1; ++a) C.atoms[fill[cell_of(a)]++] = a;  // ascending within a cell
        C.ok = true;
    };
    for (size_t si = 0; si < segs.size(); ++si) build_cells(si);
    // the shells to test for group gi, in shell order
    auto candidates = [&](size_t si, int gi, std::vector<int>& cand_sh, std::vector<int>& ats) {
        const AtomCells& C = cells[si];
        const GridSegment& sg = segs[si];
        cand_sh.clear();
        if (!C.ok) {
            for (int sh = sg.sh0; sh < sg.sh1; ++sh) cand_sh.push_back(sh);
            return;
        }
        const double r = rad[gi] + C.reach;
        int c0[3], c1[3];
        for (int k = 0; k < 3; ++k) {
            c0[k] = std::max(0, (int)std::floor((cen[3 * gi + k] - r - C.lo[k]) / C.edge));
            c1[k] = std::min(C.dim[k] - 1, (int)std::floor((cen[3 * gi + k] + r - C.lo[k]) / C.edge));
        }
        ats.clear();
        for (int x = c0[0]; x <= c1[0]; ++x)
            for (int y = c0[1]; y <= c1[1]; ++y)
                for (int z = c0[2]; z <= c1[2]; ++z) {
                    const size_t c = ((size_t)x * C.dim[1] + y) * C.dim[2] + z;
                    ats.insert(ats.end(), C.atoms.begin() + C.start[c], C.atoms.begin() + C.start[c + 1]);
                }
        std::sort(ats.begin(), ats.end());
        for (int a : ats)
            for (int sh = C.sh_first[a - C.a0]; sh < C.sh_end[a - C.a0]; ++sh) cand_sh.push_back(sh);
    };
    // Groups screened on host threads, each range of groups into its own lists (offsets local to
    // the range), then the lists joined in group order and the offsets moved by the ranges' bases.
    struct Part {
        int64_t g0 = 0, g1 = 0;
        std::vector<int> shells, rows, aos, row_info;
    };
    std::vector<Part> parts(host_threads());
    std::vector<double> blk_flops(nblk, 0.0);
    parallel_ranges(ngrp, 256, [&](int64_t glo, int64_t ghi, int t) {
        Part& P = parts[t];
        P.g0 = glo, P.g1 = ghi;
        std::vector<int> cand_sh, ats;
        for (int64_t gi = glo; gi < ghi; ++gi) {
            const size_t si = blk_seg[grp_blk[gi]];
            const int sh0 = (int)P.shells.size(), ao0 = (int)P.aos.size();
            int row = 0;
            candidates(si, (int)gi, cand_sh, ats);
            for (int sh : cand_sh) {
                const double* A = &ctx->h_atom_xyz[3 * ctx->h_sh_atom[sh]];
                const double d = std::sqrt((A[0] - cen[3 * gi]) * (A[0] - cen[3 * gi]) +
                                           (A[1] - cen[3 * gi + 1]) * (A[1] - cen[3 * gi + 1]) +
                                           (A[2] - cen[3 * gi + 2]) * (A[2] - cen[3 * gi + 2]));
                if (d - rad[gi] > Rs[sh]) continue;
                P.shells.push_back(sh);
                P.rows.push_back(row);
                const int L = ctx->h_sh_l[sh], nc = 2 * L + 1;
                for (int c = 0; c < nc; ++c) {
                    P.aos.push_back(ctx->h_sh_ao0[sh] + c);
                    P.row_info.push_back(16 * ((int)P.shells.size() - 1 - sh0) + L * L + c);
                }
                row += nc;
            }
            for (int bb = grp_blk[gi]; bb < grp_blk[gi + 1]; ++bb) {
                BlockMeta& m = ctx->h_meta[bb];
                m.sh0 = sh0, m.ao0 = ao0;
                m.nsh = (int)P.shells.size() - sh0;
                m.nb = row;
                m.nbp = mixed ? std::max(128, (row + 127) / 128 * 128) : std::max(64, (row + 63) / 64 * 64);
                blk_flops[bb] = 4.0 * double(m.nb) * m.nb * m.npts;
            }
        }
    });
    for (const Part& P : parts) {
        if (P.g1 <= P.g0) continue;
        const int bsh = (int)shells.size(), bao = (int)aos.size();
        for (int bb = grp_blk[P.g0]; bb < grp_blk[P.g1]; ++bb) ctx->h_meta[bb].sh0 += bsh, ctx->h_meta[bb].ao0 += bao;
        shells.insert(shells.end(), P.shells.begin(), P.shells.end());
        rows.insert(rows.end(), P.rows.begin(), P.rows.end());
        aos.insert(aos.end(), P.aos.begin(), P.aos.end());
        row_info.insert(row_info.end(), P.row_info.begin(), P.row_info.end());
    }
    for (int bb = 0; bb < nblk; ++bb) {  // in block order, as one sequential sum
        flops += blk_flops[bb];
        sum_nb += ctx->h_meta[bb].nb;
        G.max_nb = std::max(G.max_nb, ctx->h_meta[bb].nb);
    }
    // The INT8 rho contraction runs over K = nbp screened AOs and is exact up to OZ_MAX_K: its
    // order-5 int32 accumulator sums four digit products of at most 128^2 per K index, and the
    // FP64 combination of the four orders must stay below 2^53 (pdfxc_internal.cuh).
    if (mixed && ctx->opt.split_terms == 10) {
        for (int bb = 0; bb < nblk; ++bb)
            if (ctx->h_meta[bb].nbp > pdfxc::OZ_MAX_K)
                throw Unsupported("grid: a group of points screens in " + std::to_string(ctx->h_meta[bb].nb) +
                                  " AOs; the INT8 tensor-core contraction is exact up to " +
                                  std::to_string(pdfxc::OZ_MAX_K) +
                                  " AOs per group (use the FP64 path or a larger ao_cutoff)");
    }
    // 3. chunks of whole groups whose intermediates fit the workspace budget
    ctx->chunks.clear();
    size_t off = 0, max_ws = 0;
    Chunk cur{0, 0, 0, 0};
    auto block_need = [&](int bb) -> size_t {
        const BlockMeta& m = ctx->h_meta[bb];
        if (!mixed) return pdfxc::block_ws_doubles_rad(m.nbp, m.nsh) * sizeof(double);
        if (ctx->opt.split_terms != 10) return pdfxc::mixed_layout(m.nbp).total;
        const pdfxc::OzLayout L = pdfxc::oz_layout(m.nbp, m.nsh);
        return m.lead == bb ? L.total_lead : L.total;
    };
    for (int gi = 0; gi < ngrp; ++gi) {
        size_t need = 0;
        for (int bb = grp_blk[gi]; bb < grp_blk[gi + 1]; ++bb) need += block_need(bb);
        if (off + need > ctx->opt.workspace_bytes && grp_blk[gi] > cur.b0) {
            cur.b1 = grp_blk[gi];
            cur.ws_bytes = off;
            ctx->chunks.push_back(cur);
            max_ws = std::max(max_ws, off);
            cur = Chunk{grp_blk[gi], grp_blk[gi], 0, 0};
            off = 0;
        }
        for (int bb = grp_blk[gi]; bb < grp_blk[gi + 1]; ++bb) {
            ctx->h_meta[bb].ws = (int64_t)off;
            off += block_need(bb);
            cur.max_nbp = std::max(cur.max_nbp, ctx->h_meta[bb].nbp);
        }
    }
    cur.b1 = nblk;
    cur.ws_bytes = off;
    ctx->chunks.push_back(cur);
    max_ws = std::max(max_ws, off);

    G.nblk = nblk, G.ngrp = ngrp, G.flops = flops, G.sum_nb = sum_nb, G.max_ws = max_ws, G.mixed = mixed;
}

void build_grid(pdfxc_ctx* ctx, int64_t npts, const double* xyzw, const int* atom,
                const std::vector<GridSegment>& segs) {
    free_grid(ctx);
    resolve_shapes(ctx, npts, segs.size());
    ctx->seg_pts.clear(), ctx->seg_sh.clear();
    for (const GridSegment& sg : segs) ctx->seg_pts.push_back({sg.p0, sg.p1}), ctx->seg_sh.push_back({sg.sh0, sg.sh1});
    HostGrid G;
    plan_grid(ctx, npts, xyzw, atom, segs, G);
    const int nblk = G.nblk, ngrp = G.ngrp;
    const size_t max_ws = G.max_ws;
    const bool mixed = G.mixed;
    const std::vector<double>&px = G.px, &py = G.py, &pz = G.pz, &pw = G.pw;
    const std::vector<int>&shells = G.shells, &rows = G.rows, &aos = G.aos, &row_info = G.row_info;
    const std::vector<int>& grp_blk = G.grp_blk;
    const double flops = G.flops, sum_nb = G.sum_nb;
    cudaStream_t s = ctx->stream;
    upload(&ctx->d_px, px, s);
    upload(&ctx->d_py, py, s);
    upload(&ctx->d_pz, pz, s);
    upload(&ctx->d_pw, pw, s);
    upload(&ctx->d_meta, ctx->h_meta, s);
    upload(&ctx->d_blk_shells, shells, s);
    upload(&ctx->d_blk_shell_row, rows, s);
    upload(&ctx->d_blk_aos, aos, s);
    upload(&ctx->d_blk_row_info, row_info, s);
    if (mixed) {
        std::vector<pdfxc::RowGeom> geom(row_info.size());
        for (int gi = 0; gi < ngrp; ++gi) {
            const BlockMeta& m = ctx->h_meta[grp_blk[gi]];
            for (int r = 0; r < m.nb; ++r) {
                const int info = row_info[m.ao0 + r];
                const double* A = &ctx->h_atom_xyz[3 * ctx->h_sh_atom[shells[m.sh0 + (info >> 4)]]];
                geom[m.ao0 + r] = pdfxc::RowGeom{A[0], A[1], A[2], info, 0};
            }
        }
        upload(&ctx->d_blk_row_geom, geom, s);
    }
    upload(&ctx->d_seg_blk, ctx->seg_blk, s);
    {  // the FP64 contractions' tile lists (64-AO tiles of each block's nbp rows)
        std::vector<int2> xt, vt;
        ctx->h_xtile0.assign(1, 0), ctx->h_vtile0.assign(1, 0);
        for (int b = 0; b < nblk; ++b) {
            const int nt = (ctx->h_meta[b].nbp + 63) / 64;
            for (int i = 0; i < nt; ++i) xt.push_back(make_int2(b, i));
            for (int i = 0; i < nt; ++i)
                for (int j = 0; j < nt; ++j) vt.push_back(make_int2(b, (i << 16) | j));
            ctx->h_xtile0.push_back((int64_t)xt.size());
            ctx->h_vtile0.push_back((int64_t)vt.size());
        }
        upload(&ctx->d_xtiles, xt, s);
        upload(&ctx->d_vtiles, vt, s);
    }
    ctx->h_grp.assign(grp_blk.begin(), grp_blk.end() - 1);
    upload(&ctx->d_grp, ctx->h_grp, s);
    if (mixed && ctx->opt.split_terms == 10) {
        // the contraction work items of every chunk, largest first (longest-processing-time order
        // for the device scheduler; a stable sort keeps a block's or group's items together)
        std::vector<int2> items;
        ctx->items_off_rho.clear(), ctx->items_n_rho.clear(), ctx->items_off_vxc.clear(), ctx->items_n_vxc.clear();
        for (const Chunk& c : ctx->chunks) {
            std::vector<std::pair<int, int2>> it;
            for (int b = c.b0; b < c.b1; ++b)  // rho: (block, 64-AO output tile); cost ~ K = nbp
                for (int nt = 0; nt < ctx->h_meta[b].nbp / 64; ++nt) it.push_back({ctx->h_meta[b].nbp, make_int2(b, nt)});
            std::stable_sort(it.begin(), it.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
            ctx->items_off_rho.push_back((int)items.size());
            ctx->items_n_rho.push_back((int)it.size());
            for (const auto& x : it) items.push_back(x.second);
            it.clear();
            for (int b = c.b0; b < c.b1; ++b) {  // Vxc: (group, 128-AO row tile, 64-AO column tile); cost ~ K = points
                const BlockMeta& m = ctx->h_meta[b];
                if (m.lead != b) continue;
                for (int mt = 0; mt < m.nbp / 128; ++mt)
                    for (int nt = 0; nt < m.nbp / 64; ++nt) it.push_back({m.gn, make_int2(b, (mt << 16) | nt)});
            }
            std::stable_sort(it.begin(), it.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
            ctx->items_off_vxc.push_back((int)items.size());
            ctx->items_n_vxc.push_back((int)it.size());
            for (const auto& x : it) items.push_back(x.second);
        }
        upload(&ctx->d_items, items, s);
        dev_alloc(&ctx->d_counters, 2 * ctx->chunks.size());
    }
    dev_alloc(&ctx->d_rho, (size_t)nblk * BLOCK_PTS * 4);
    dev_alloc(&ctx->d_coef, (size_t)nblk * BLOCK_PTS * 4);
    dev_alloc(&ctx->d_blk_sum, (size_t)nblk * 2);
    dev_alloc(&ctx->d_rho_acc, (size_t)nblk * BLOCK_PTS * 4);  // per-point sums of the rho pass
    PDFXC_CUDA(cudaMemsetAsync(ctx->d_rho, 0, sizeof(double) * (size_t)nblk * BLOCK_PTS * 4, s));
    if (cudaMalloc(&ctx->d_ws, max_ws) != cudaSuccess) {
        ctx->d_ws = nullptr;
        throw std::bad_alloc();
    }
    ctx->ws_bytes = max_ws;
    ctx->phi_map_ok = mixed && ctx->opt.split_terms == 10 && pdfxc::make_phi_map(ctx->d_ws, max_ws, &ctx->phi_map);
    ctx->nblk = nblk;
    ctx->blk_lo = 0, ctx->blk_hi = nblk;
    ctx->npts = npts;
    ctx->contraction_flops = flops;
    ctx->mean_nb = sum_nb / nblk;
    PDFXC_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

extern "C" {

pdfxc_status pdfxc_set_grid(pdfxc_ctx* ctx, int64_t npts, const double* xyzw, const int* atom) {
    return guarded(ctx, [&]() -> pdfxc_status {
        if (ctx->nao == 0) {
            ctx->err = "pdfxc_set_grid: call pdfxc_set_system first";
            return PDFXC_ERR_STATE;
        }
        if (npts <= 0 || !xyzw) {
            ctx->err = "pdfxc_set_grid: empty grid or null pointer";
            return PDFXC_ERR_ARG;
        }
        // the owning atom is not needed by the quadrature itself; the gradient keeps it per point
        if (atom)
            for (int64_t i = 0; i < npts; ++i)
                if (atom[i] < 0 || atom[i] >= ctx->natom) {
                    ctx->err = "pdfxc_set_grid: owner atom index out of range";
                    return PDFXC_ERR_ARG;
                }
        ctx->mol.clear();
        build_grid(ctx, npts, xyzw, atom, {GridSegment{0, npts, 0, ctx->nshell}});
        return PDFXC_OK;
    });
}

}  // extern "C"

namespace {

// Partition weights on the device: Becke (ss = false) or Stratmann-Scuseria (ss = true).
// Partition weights of device-resident points: d_wo = d_ws * P_owner / sum_m P_m (Becke or
// Stratmann-Scuseria), enqueued on the context's stream; d_br (natom Becke radii) only for Becke.
void partition_weights_device(pdfxc_ctx* ctx, bool ss, int64_t npts, const double* d_xyz, const int* d_own,
                              const double* d_ws, const double* d_br, int size_adjust, double* d_wo) {
    cudaStream_t s = ctx->stream;
    double* d_pair = nullptr;
    try {
        if (ss) {
            const int na = ctx->natom, nn = na - 1;
            if (!ctx->d_nbr_idx && nn > 0) {  // once per system: neighbour lists by distance
                std::vector<int> idx((size_t)na * nn);
                std::vector<double> dst((size_t)na * nn);
                std::vector<std::pair<double, int>> row(nn);
                for (int m = 0; m < na; ++m) {
                    const double* A = &ctx->h_atom_xyz[3 * m];
                    int k = 0;
                    for (int n = 0; n < na; ++n) {
                        if (n == m) continue;
                        const double* B = &ctx->h_atom_xyz[3 * n];
                        row[k++] = {std::sqrt((A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) +
                                              (A[2] - B[2]) * (A[2] - B[2])),
                                    n};
                    }
                    std::sort(row.begin(), row.end());
                    for (int j = 0; j < nn; ++j) idx[(size_t)m * nn + j] = row[j].second, dst[(size_t)m * nn + j] = row[j].first;
                }
                upload(&ctx->d_nbr_idx, idx, s);
                upload(&ctx->d_nbr_dist, dst, s);
            }
            dev_alloc(&d_pair, 2 * (size_t)ctx->natom * ctx->natom);
            pdfxc::launch_ss(ctx->d_atom_xyz, ctx->natom, d_pair, d_pair + (size_t)ctx->natom * ctx->natom,
                             ctx->d_nbr_idx, ctx->d_nbr_dist, npts, d_xyz, d_own, d_ws, d_wo, s);
        } else if ((size_t)ctx->natom <= pdfxc::becke_small_atoms()) {
            dev_alloc(&d_pair, 2 * (size_t)ctx->natom * ctx->natom);
            pdfxc::launch_becke_tab(ctx->d_atom_xyz, d_br, ctx->d_ghost, ctx->natom, size_adjust, d_pair,
                                    d_pair + (size_t)ctx->natom * ctx->natom, npts, d_xyz, d_own, d_ws, d_wo, s);
        } else if ((size_t)ctx->natom <= pdfxc::becke_warp_max_atoms()) {
            dev_alloc(&d_pair, 4 * (size_t)ctx->natom * ctx->natom);
            pdfxc::launch_becke_warp(ctx->d_atom_xyz, d_br, ctx->d_ghost, ctx->natom, size_adjust, d_pair, npts, d_xyz,
                                     d_own, d_ws, d_wo, s);
        } else if ((size_t)ctx->natom <= pdfxc::becke_max_atoms()) {
            pdfxc::launch_becke(ctx->d_atom_xyz, d_br, ctx->d_ghost, ctx->natom, size_adjust, npts, d_xyz, d_own,
                                d_ws, d_wo, s);
        } else {
            throw std::runtime_error("Becke partition: at most " + std::to_string(pdfxc::becke_max_atoms()) +
                                     " atoms (use the Stratmann-Scuseria partition)");
        }
        PDFXC_CUDA(cudaGetLastError());
        PDFXC_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        dev_free(d_pair);
        throw;
    }
    dev_free(d_pair);
}

pdfxc_status partition_weights(pdfxc_ctx* ctx, bool ss, int64_t npts, const double* xyz, const int* atom,
                               const double* w_single, const double* becke_radius, int size_adjust, double* w_out) {
    const char* name = ss ? "pdfxc_ss_weights" : "pdfxc_becke_weights";
    return guarded(ctx, [&]() -> pdfxc_status {
        if (ctx->natom == 0) {
            ctx->err = std::string(name) + ": call pdfxc_set_system first";
            return PDFXC_ERR_STATE;
        }
        if (npts <= 0 || !xyz || !atom || !w_single || !w_out || (!ss && !becke_radius)) {
            ctx->err = std::string(name) + ": empty input or null pointer";
            return PDFXC_ERR_ARG;
        }
        if (ss && ctx->natom > 6000) {
            ctx->err = "pdfxc_ss_weights: at most 6000 atoms (atoms are staged in shared memory)";
            return PDFXC_ERR_UNSUPPORTED;
        }
        for (int64_t i = 0; i < npts; ++i)
            if (atom[i] < 0 || atom[i] >= ctx->natom) {
                ctx->err = std::string(name) + ": owner atom index out of range";
                return PDFXC_ERR_ARG;
            }
        cudaStream_t s = ctx->stream;
        double *d_xyz = nullptr, *d_ws = nullptr, *d_wo = nullptr, *d_br = nullptr;
        int* d_own = nullptr;
        try {
            dev_alloc(&d_xyz, 3 * (size_t)npts);
            dev_alloc(&d_ws, (size_t)npts);
            dev_alloc(&d_wo, (size_t)npts);
            dev_alloc(&d_br, (size_t)ctx->natom);
            dev_alloc(&d_own, (size_t)npts);
            PDFXC_CUDA(cudaMemcpyAsync(d_xyz, xyz, 3 * sizeof(double) * npts, cudaMemcpyHostToDevice, s));
            PDFXC_CUDA(cudaMemcpyAsync(d_ws, w_single, sizeof(double) * npts, cudaMemcpyHostToDevice, s));
            if (!ss)
                PDFXC_CUDA(cudaMemcpyAsync(d_br, becke_radius, sizeof(double) * ctx->natom, cudaMemcpyHostToDevice, s));
            PDFXC_CUDA(cudaMemcpyAsync(d_own, atom, sizeof(int) * npts, cudaMemcpyHostToDevice, s));
            partition_weights_device(ctx, ss, npts, d_xyz, d_own, d_ws, d_br, size_adjust, d_wo);
            PDFXC_CUDA(cudaMemcpyAsync(w_out, d_wo, sizeof(double) * npts, cudaMemcpyDeviceToHost, s));
            PDFXC_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            dev_free(d_xyz), dev_free(d_ws), dev_free(d_wo), dev_free(d_br), dev_free(d_own);
            throw;
        }
        dev_free(d_xyz), dev_free(d_ws), dev_free(d_wo), dev_free(d_br), dev_free(d_own);
        return PDFXC_OK;
    });
}

}  // namespace

extern "C" {

pdfxc_status pdfxc_becke_weights(pdfxc_ctx* ctx, int64_t npts, const double* xyz, const int* atom,
                                 const double* w_single, const double* becke_radius, int size_adjust, double* w_out) {
    return partition_weights(ctx, false, npts, xyz, atom, w_single, becke_radius, size_adjust, w_out);
}

pdfxc_status pdfxc_ss_weights(pdfxc_ctx* ctx, int64_t npts, const double* xyz, const int* atom,
                              const double* w_single, double* w_out) {
    return partition_weights(ctx, true, npts, xyz, atom, w_single, nullptr, 0, w_out);
}

}  // extern "C"

namespace {

// Radial abscissa and weight of shell i (1-based) of nr: Gauss-Chebyshev of the second kind
// with the Becke, Treutler-Ahlrichs or Knowles-Kaltenborn map
// (DfGenerateGrid::getRadialAbscissaAndWeight_GaussChebyshev, src/libpdf/DfGenerateGrid.cpp:1612-1655).
void radial_gc(double R, int nr, int i, int mapping, double* r, double* w) {
    const double pi = 3.14159265358979323846;
    const double n1 = nr + 1.0;
    const double t = i * pi / n1;
    const double sn = std::sin(t), cs = std::cos(t);
    const double ss = sn * sn;
    const double x = (n1 - 2.0 * i) / n1 + (2.0 / pi) * (1.0 + (2.0 / 3.0) * ss) * cs * sn;
    const double inv_x1 = 1.0 / (x - 1.0);
    const double inv_ln2 = 1.0 / std::log(2.0);
    double jac;
    if (mapping == PDFXC_MAP_BECKE) {
        *r = R * (1.0 + x) / (1.0 - x);
        jac = R * ((x + 1.0) * inv_x1 * inv_x1 - inv_x1);
    } else if (mapping == PDFXC_MAP_TA) {
        *r = inv_ln2 * std::log(2.0 * (-inv_x1)) * R;
        jac = R * inv_ln2 / (1.0 - x);
    } else {
        *r = inv_ln2 * std::log(2.0 * (-inv_x1));
        jac = inv_ln2 / (1.0 - x);
    }
    *w = (16.0 / (3.0 * n1)) * ss * ss * jac * *r * *r * 4.0 * pi;
}

// Euler-Maclaurin (DfGenerateGrid::getRadialAbscissaAndWeight_EulerMaclaurin, :1597-1610).
void radial_em(double R, int nr, int i, double* r, double* w) {
    const double pi = 3.14159265358979323846;
    const double inv = 1.0 / double(nr + 1 - i);
    *r = R * double(i * i) * inv * inv;
    const double i5 = double((long long)i * i * i * i * i);
    *w = 2.0 * std::pow(R, 3) * double(nr + 1) * i5 * std::pow(inv, 7) * 4.0 * pi;
}

// Angular order of a shell at r_i: nang without pruning; Murray-Handy-Laming with K = 5
// (min(int(5 r / R * nang), nang), rounded down to a tabulated order or the smallest,
// :1658-1688); SG-1 regions of r / R by atomic number (:1690-1713, parameters :960-982).
int angular_order(int pruning, double r, double R, int nang, int Z, const std::vector<int>& orders) {
    if (pruning == PDFXC_PRUNE_SG1) {
        double a[4] = {0.0, 0.0, 0.0, 10000.0};
        if (Z == 1 || Z == 2) a[0] = 0.25, a[1] = 0.5, a[2] = 1.0, a[3] = 4.5;
        else if (Z >= 3 && Z <= 10) a[0] = 0.1667, a[1] = 0.5, a[2] = 0.9, a[3] = 3.5;
        else if (Z >= 11 && Z <= 18) a[0] = 0.1, a[1] = 0.4, a[2] = 0.8, a[3] = 2.5;
        const double q = r * (1.0 / R);
        if (q < a[1]) return q < a[0] ? 6 : 38;
        if (q < a[2]) return 86;
        return q < a[3] ? 194 : 86;
    }
    int n = nang;
    if (pruning == PDFXC_PRUNE_MHL) n = std::min<int>((5.0 * r / R) * nang, nang);
    const auto it = std::upper_bound(orders.begin(), orders.end(), n);
    return it == orders.begin() ? orders[0] : *(it - 1);
}

}  // namespace

extern "C" {

pdfxc_status pdfxc_generate_grid(pdfxc_ctx* ctx, const pdfxc_grid_params* prm, int64_t* npts_out) {
    return guarded(ctx, [&]() -> pdfxc_status {
        if (ctx->natom == 0) {
            ctx->err = "pdfxc_generate_grid: call pdfxc_set_system first";
            return PDFXC_ERR_STATE;
        }
        if (!prm || prm->nrad <= 0 || prm->n_orders <= 0 || !prm->orders || !prm->unit_grids || !prm->atom_radius ||
            prm->radial < PDFXC_RADIAL_GC || prm->radial > PDFXC_RADIAL_EM || prm->mapping < PDFXC_MAP_BECKE ||
            prm->mapping > PDFXC_MAP_KK || prm->pruning < PDFXC_PRUNE_NONE || prm->pruning > PDFXC_PRUNE_SG1 ||
            (prm->partition != PDFXC_PARTITION_BECKE && prm->partition != PDFXC_PARTITION_SS) ||
            (prm->partition == PDFXC_PARTITION_BECKE && !prm->becke_radius)) {
            ctx->err = "pdfxc_generate_grid: missing table or parameter out of range";
            return PDFXC_ERR_ARG;
        }
        const int natom = ctx->natom;
        std::vector<int> orders(prm->orders, prm->orders + prm->n_orders);
        std::vector<int64_t> urow(orders.size());
        int64_t nrows = 0;
        for (size_t k = 0; k < orders.size(); ++k) {
            if (orders[k] <= 0 || (k > 0 && orders[k] <= orders[k - 1])) {
                ctx->err = "pdfxc_generate_grid: unit-grid orders must be positive and ascending";
                return PDFXC_ERR_ARG;
            }
            urow[k] = nrows;
            nrows += orders[k];
        }
        for (int a = 0; a < natom; ++a)
            if (!(prm->atom_radius[a] >= 0.0) ||
                (prm->atom_radius[a] > 0.0 && prm->pruning == PDFXC_PRUNE_SG1 && ctx->h_atom_z[a] <= 0)) {
                ctx->err = "pdfxc_generate_grid: atom radius negative (or SG-1 without atomic numbers)";
                return PDFXC_ERR_ARG;
            }
        // shells (host: O(natom nrad)), then the points and weights on the device
        std::vector<pdfxc::GridShell> shells;
        int64_t np = 0;
        for (int a = 0; a < natom; ++a) {
            const double R = prm->atom_radius[a];
            if (R == 0.0) continue;  // no grid on this atom (a dummy atom of the reference)
            for (int i = 1; i <= prm->nrad; ++i) {
                double r, wr;
                if (prm->radial == PDFXC_RADIAL_GC) radial_gc(R, prm->nrad, i, prm->mapping, &r, &wr);
                else radial_em(R, prm->nrad, i, &r, &wr);
                if (r > 30.0) continue;
                const int n = angular_order(prm->pruning, r, R, prm->nang, ctx->h_atom_z[a], orders);
                const auto it = std::lower_bound(orders.begin(), orders.end(), n);
                if (it == orders.end() || *it != n) {
                    ctx->err = "pdfxc_generate_grid: angular order " + std::to_string(n) + " is not tabulated";
                    return PDFXC_ERR_ARG;
                }
                shells.push_back(pdfxc::GridShell{a, n, urow[it - orders.begin()], np, r, wr});
                np += n;
            }
        }
        if (np == 0) {
            ctx->err = "pdfxc_generate_grid: every point was screened out (no atom has a grid)";
            return PDFXC_ERR_ARG;
        }
        cudaStream_t s = ctx->stream;
        const double ident[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
        std::vector<double> O(prm->orientation ? prm->orientation : ident, (prm->orientation ? prm->orientation : ident) + 9);
        pdfxc::GridShell* d_sh = nullptr;
        double *d_unit = nullptr, *d_O = nullptr, *d_xyz = nullptr, *d_ws = nullptr, *d_wo = nullptr, *d_br = nullptr;
        int* d_own = nullptr;
        std::vector<double> xyz(3 * (size_t)np), w((size_t)np);
        std::vector<int> own((size_t)np);
        try {
            upload(&d_sh, shells, s);
            upload(&d_unit, std::vector<double>(prm->unit_grids, prm->unit_grids + 4 * nrows), s);
            upload(&d_O, O, s);
            dev_alloc(&d_xyz, 3 * (size_t)np);
            dev_alloc(&d_ws, (size_t)np);
            dev_alloc(&d_wo, (size_t)np);
            dev_alloc(&d_own, (size_t)np);
            pdfxc::launch_grid_points(d_sh, (int)shells.size(), d_unit, d_O, ctx->d_atom_xyz, d_xyz, d_ws, d_own, s);
            PDFXC_LAUNCHED("k_grid_points");
            if (prm->partition == PDFXC_PARTITION_BECKE)
                upload(&d_br, std::vector<double>(prm->becke_radius, prm->becke_radius + natom), s);
            partition_weights_device(ctx, prm->partition == PDFXC_PARTITION_SS, np, d_xyz, d_own, d_ws, d_br,
                                     prm->size_adjust, d_wo);
            PDFXC_CUDA(cudaMemcpyAsync(xyz.data(), d_xyz, sizeof(double) * xyz.size(), cudaMemcpyDeviceToHost, s));
            PDFXC_CUDA(cudaMemcpyAsync(w.data(), d_wo, sizeof(double) * w.size(), cudaMemcpyDeviceToHost, s));
            PDFXC_CUDA(cudaMemcpyAsync(own.data(), d_own, sizeof(int) * own.size(), cudaMemcpyDeviceToHost, s));
            PDFXC_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            dev_free(d_sh), dev_free(d_unit), dev_free(d_O), dev_free(d_xyz), dev_free(d_ws), dev_free(d_wo);
            dev_free(d_br), dev_free(d_own);
            throw;
        }
        dev_free(d_sh), dev_free(d_unit), dev_free(d_O), dev_free(d_xyz), dev_free(d_ws), dev_free(d_wo);
        dev_free(d_br), dev_free(d_own);
        // the weight screen, in point order
        std::vector<double> xyzw;
        std::vector<int> atom;
        xyzw.reserve(4 * (size_t)np);
        atom.reserve((size_t)np);
        for (int64_t i = 0; i < np; ++i)
            if (std::fabs(w[i]) > prm->weight_cutoff) {
                xyzw.insert(xyzw.end(), {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], w[i]});
                atom.push_back(own[i]);
            }
        const int64_t n = (int64_t)atom.size();
        if (n == 0) {
            ctx->err = "pdfxc_generate_grid: every point was screened out";
            return PDFXC_ERR_ARG;
        }
        const pdfxc_status st = pdfxc_set_grid(ctx, n, xyzw.data(), atom.data());
        if (st == PDFXC_OK && npts_out) *npts_out = n;
        return st;
    });
}

pdfxc_status pdfxc_get_grid(pdfxc_ctx* ctx, double* xyzw, int* atom) {
    return guarded(ctx, [&]() -> pdfxc_status {
        if (!xyzw) return PDFXC_ERR_ARG;
        if (ctx->nblk == 0) {
            ctx->err = "pdfxc_get_grid: no grid";
            return PDFXC_ERR_STATE;
        }
        const size_t nslot = (size_t)ctx->nblk * BLOCK_PTS;
        std::vector<double> c[4] = {std::vector<double>(nslot), std::vector<double>(nslot), std::vector<double>(nslot),
                                    std::vector<double>(nslot)};
        const double* src[4] = {ctx->d_px, ctx->d_py, ctx->d_pz, ctx->d_pw};
        for (int k = 0; k < 4; ++k)
            PDFXC_CUDA(cudaMemcpyAsync(c[k].data(), src[k], sizeof(double) * nslot, cudaMemcpyDeviceToHost, ctx->stream));
        PDFXC_CUDA(cudaStreamSynchronize(ctx->stream));
        for (size_t slot = 0; slot < nslot; ++slot) {
            const int64_t i = ctx->h_src[slot];
            if (i < 0) continue;
            for (int k = 0; k < 4; ++k) xyzw[4 * i + k] = c[k][slot];
            if (atom && !ctx->h_owner.empty()) atom[i] = ctx->h_owner[slot];
        }
        return PDFXC_OK;
    });
}

}  // extern "C"

namespace {

// Enqueue one build on ctx->stream: d_PA -> ctx->d_V (= Vxc), scalars -> ctx->d_scalars.
void enqueue_build(pdfxc_ctx* ctx, int fn, const double* d_PA, bool incremental) {
    cudaStream_t s = ctx->stream;
    const bool gga = pdfxc::functional_is_gga(fn);
    const int nao = ctx->nao;
    const pdfxc::BasisView bv = basis_view(ctx);
    const pdfxc::GridView gv = grid_view(ctx);
    char* ws = static_cast<char*>(ctx->d_ws);
    const size_t nev = 5 * ctx->chunks.size() + 1;
    while (ctx->stage_ev.size() < nev) {
        cudaEvent_t e;
        PDFXC_CUDA(cudaEventCreate(&e));
        ctx->stage_ev.push_back(e);
    }
    memset_async(ctx->d_Vacc, sizeof(double) * (size_t)nao * nao, s);
    int64_t launches = 0;
    const bool mixed = ctx->opt.precision == PDFXC_PRECISION_MIXED;
    if (mixed) {
        memset_async(ctx->d_rho_acc, sizeof(double) * (size_t)ctx->nblk * BLOCK_PTS * 4, s);
        PDFXC_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), s));
        if (ctx->d_counters) PDFXC_CUDA(cudaMemsetAsync(ctx->d_counters, 0, sizeof(int) * 2 * ctx->chunks.size(), s));
        if (ctx->opt.split_terms == 10) {
            pdfxc::oz_p_digits(d_PA, nao, ctx->d_row_cols, ctx->d_p_rowexp, ctx->d_p_words, s);
            ++launches;
        }
    }
    // the context's block range (all blocks unless pdfxc_set_block_range narrowed it)
    auto clip = [&](const Chunk& c, int& b0, int& n) {
        b0 = std::max(c.b0, ctx->blk_lo);
        n = std::min(c.b1, ctx->blk_hi) - b0;
        return n > 0;
    };
    for (size_t ci = 0; ci < ctx->chunks.size() && mixed; ++ci) {
        const Chunk& c = ctx->chunks[ci];
        cudaEvent_t* e = &ctx->stage_ev[5 * ci];
        int cb0, cn;
        if (!clip(c, cb0, cn)) {
            for (int k = 0; k < 5; ++k) PDFXC_CUDA(cudaEventRecord(e[k], s));
            continue;
        }
        const int g_lo = (int)(std::lower_bound(ctx->h_grp.begin(), ctx->h_grp.end(), cb0) - ctx->h_grp.begin());
        const int g_hi = (int)(std::lower_bound(ctx->h_grp.begin(), ctx->h_grp.end(), cb0 + cn) - ctx->h_grp.begin());
        pdfxc::MixedArgs a{bv, gv, cb0, cn, c.max_nbp, fn, incremental ? 1 : 0, ctx->opt.split_terms, nao,
                           ctx->opt.rho_cutoff, d_PA, ws, ctx->d_rho_acc, ctx->d_rho, ctx->d_coef, ctx->d_blk_sum,
                           ctx->d_Vacc, ctx->d_err, ctx->d_grp + g_lo, g_hi - g_lo, ctx->d_p_rowexp,
                           ctx->d_p_words, nullptr, 0, nullptr, 0, nullptr, ctx->tuned_stages,
                           ctx->phi_map_ok ? &ctx->phi_map : nullptr};
        if (ctx->d_items) {
            a.items_rho = ctx->d_items + ctx->items_off_rho[ci], a.n_rho = ctx->items_n_rho[ci];
            a.items_vxc = ctx->d_items + ctx->items_off_vxc[ci], a.n_vxc = ctx->items_n_vxc[ci];
            a.counters = ctx->d_counters + 2 * ci;
        }
        const bool oz = ctx->opt.split_terms == 10;
        PDFXC_CUDA(cudaEventRecord(e[0], s));
        oz ? pdfxc::oz_prepare(a, s) : pdfxc::mixed_prepare(a, s);
        PDFXC_LAUNCHED("prepare (AO values, operand slices)");
        PDFXC_CUDA(cudaEventRecord(e[1], s));
        oz ? pdfxc::oz_rho(a, s) : pdfxc::mixed_rho(a, s);
        PDFXC_LAUNCHED("rho contraction");
        PDFXC_CUDA(cudaEventRecord(e[2], s));
        oz ? pdfxc::oz_functional(a, s) : pdfxc::mixed_functional(a, s);
        PDFXC_LAUNCHED("functional / Z");
        PDFXC_CUDA(cudaEventRecord(e[3], s));
        oz ? pdfxc::oz_vxc(a, s) : pdfxc::mixed_vxc(a, s);
        PDFXC_LAUNCHED("Vxc contraction");
        PDFXC_CUDA(cudaEventRecord(e[4], s));
        launches += oz ? 7 : 6;
    }
    for (size_t ci = 0; ci < ctx->chunks.size() && !mixed; ++ci) {
        const Chunk& c = ctx->chunks[ci];
        cudaEvent_t* e = &ctx->stage_ev[5 * ci];
        int cb0, nb;
        if (!clip(c, cb0, nb)) {
            for (int k = 0; k < 5; ++k) PDFXC_CUDA(cudaEventRecord(e[k], s));
            continue;
        }
        // per block: phi, X (then Z), and for GGA the shells' radial sums (block_ws_doubles_rad)
        PDFXC_CUDA(cudaEventRecord(e[0], s));
        if (gga) pdfxc::launch_ao_eval_rad(bv, gv, cb0, nb, ws, s);
        else pdfxc::launch_ao_eval(bv, gv, cb0, nb, false, ws, 0, s);
        PDFXC_LAUNCHED("k_ao_eval");
        PDFXC_CUDA(cudaEventRecord(e[1], s));
        pdfxc::launch_gemm_x(gv, d_PA, nao, cb0, nb, c.max_nbp, 1, ws, s);
        PDFXC_LAUNCHED("k_gemm_x");
        PDFXC_CUDA(cudaEventRecord(e[2], s));
        if (gga) {
            pdfxc::launch_rho_rad(bv, gv, cb0, nb, ws, ctx->d_rho_acc, s);
            pdfxc::launch_functional_points(gv, cb0, nb, fn, incremental, ctx->opt.rho_cutoff, ctx->d_rho_acc,
                                            ctx->d_rho, ctx->d_coef, ctx->d_blk_sum, s);
            pdfxc::launch_z_rad(bv, gv, cb0, nb, ctx->d_coef, ws, s);
        } else
            pdfxc::launch_rho_functional(gv, cb0, nb, fn, incremental, ctx->opt.rho_cutoff, ws, ctx->d_rho,
                                         ctx->d_coef, ctx->d_blk_sum, s);
        PDFXC_LAUNCHED("k_rho_functional");
        PDFXC_CUDA(cudaEventRecord(e[3], s));
        pdfxc::launch_gemm_v_plane(gv, cb0, nb, c.max_nbp, 1, ws, ctx->d_Vacc, nao, s);
        PDFXC_LAUNCHED("k_gemm_v");
        PDFXC_CUDA(cudaEventRecord(e[4], s));
        launches += gga ? 6 : 4;
    }
    pdfxc::launch_finish(ctx->d_Vacc, ctx->d_V, nao, ctx->d_blk_sum + 2 * (size_t)ctx->blk_lo,
                         ctx->blk_hi - ctx->blk_lo, ctx->d_scalars, s);
    launches += 2;
    PDFXC_CUDA(cudaGetLastError());
    PDFXC_CUDA(cudaEventRecord(ctx->stage_ev[nev - 1], s));
    ctx->last_profile.launches = launches;
}

// F += V for a host F from the device V (n2 elements): V goes through two pinned staging
// buffers in pieces of at most 8 Mi elements, each piece added on the host by several threads
// while the next one is copied.
void accumulate_to_host(pdfxc_ctx* ctx, const double* d_V, double* F, size_t n2) {
    constexpr size_t kPiece = size_t(8) << 20;
    const size_t piece = std::min(kPiece, n2);
    if (ctx->stage_elems < piece) {
        if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
        ctx->h_stage = nullptr;
        ctx->stage_elems = 0;
        if (cudaMallocHost(&ctx->h_stage, 2 * piece * sizeof(double)) != cudaSuccess) {
            ctx->h_stage = nullptr;
            throw std::bad_alloc();
        }
        ctx->stage_elems = piece;
    }
    cudaEvent_t ev[2];
    PDFXC_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
    if (cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming) != cudaSuccess) {
        cudaEventDestroy(ev[0]);
        throw CudaError("cudaEventCreate");
    }
    auto add = [&](const double* src, double* dst, size_t n) {
        const unsigned nt = n < (size_t(1) << 20) ? 1u : std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
        if (nt == 1) {
            for (size_t i = 0; i < n; ++i) dst[i] += src[i];
            return;
        }
        std::vector<std::thread> th;
        const size_t per = (n + nt - 1) / nt;
        for (unsigned t = 0; t < nt; ++t) {
            const size_t a = t * per, b = std::min(n, a + per);
            if (a < b) th.emplace_back([=]() {
                for (size_t i = a; i < b; ++i) dst[i] += src[i];
            });
        }
        for (auto& x : th) x.join();
    };
    try {
        const size_t npieces = (n2 + piece - 1) / piece;
        for (size_t k = 0; k <= npieces; ++k) {
            if (k < npieces) {  // copy piece k while the host adds piece k - 1
                const size_t off = k * piece, len = std::min(piece, n2 - off);
                PDFXC_CUDA(cudaMemcpyAsync(ctx->h_stage + (k & 1) * piece, d_V + off, len * sizeof(double),
                                           cudaMemcpyDeviceToHost, ctx->stream));
                PDFXC_CUDA(cudaEventRecord(ev[k & 1], ctx->stream));
            }
            if (k >= 1) {
                const size_t j = k - 1, off = j * piece, len = std::min(piece, n2 - off);
                PDFXC_CUDA(cudaEventSynchronize(ev[j & 1]));
                add(ctx->h_stage + (j & 1) * piece, F + off, len);
            }
        }
    } catch (...) {
        cudaEventDestroy(ev[0]), cudaEventDestroy(ev[1]);
        throw;
    }
    cudaEventDestroy(ev[0]), cudaEventDestroy(ev[1]);
}

// After the stream has synchronised: the device error word (0 = no expired wait).
int device_error(pdfxc_ctx* ctx) {
    int code = 0;
    PDFXC_CUDA(cudaMemcpy(&code, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    return code;
}

// After the stream has synchronised: fold the stage events into last_profile.
void collect_profile(pdfxc_ctx* ctx) {
    pdfxc_profile& p = ctx->last_profile;
    p.total_ms = p.ao_ms = p.gemm_x_ms = p.rho_ms = p.gemm_v_ms = p.finish_ms = 0.f;
    PDFXC_CUDA(cudaEventElapsedTime(&p.total_ms, ctx->ev[0], ctx->ev[1]));
    // stage timings are diagnostics: an event pair that cannot be timed reads 0
    auto dt = [](cudaEvent_t a, cudaEvent_t b) {
        float t = 0.f;
        if (cudaEventElapsedTime(&t, a, b) != cudaSuccess) {
            cudaGetLastError();
            t = 0.f;
        }
        return t;
    };
    if (!ctx->last_staged) return;  // graph replay: only the total is timed
    for (size_t ci = 0; ci < ctx->chunks.size(); ++ci) {
        cudaEvent_t* e = &ctx->stage_ev[5 * ci];
        p.ao_ms += dt(e[0], e[1]);
        p.gemm_x_ms += dt(e[1], e[2]);
        p.rho_ms += dt(e[2], e[3]);
        p.gemm_v_ms += dt(e[3], e[4]);
    }
    const size_t last = 5 * ctx->chunks.size();
    p.finish_ms = dt(ctx->stage_ev[last - 1], ctx->stage_ev[last]);
}

// The open-shell build's launches on ctx->stream (FP64 path): per chunk phi (and grad phi), X_A
// and X_B, the open-shell functional with Z_A and Z_B in place of X, and the two Vxc
// contractions. P_A, P_B in ctx->d_P, d_P_b; Vacc, Vacc_b zeroed. Returns the launch count.
int64_t enqueue_uks_fp64(pdfxc_ctx* ctx, int functional, bool incremental) {
    const bool gga = pdfxc::functional_is_gga(functional);
    const int nao = ctx->nao, nphi = gga ? 4 : 1;
    cudaStream_t s = ctx->stream;
    ensure_plan(ctx, ctx->uplan, nphi + 2);  // phi planes, X_A, X_B
    pdfxc::GridView gv = grid_view(ctx);
    gv.meta = ctx->uplan.d_meta;
    const pdfxc::BasisView bv = basis_view(ctx);
    char* ws = static_cast<char*>(ctx->uplan.d_ws);
    int64_t launches = 0;
    for (const Chunk& c : ctx->uplan.chunks) {
        const int b0 = std::max(c.b0, ctx->blk_lo), nb = std::min(c.b1, ctx->blk_hi) - b0;
        if (nb <= 0) continue;
        pdfxc::launch_ao_eval(bv, gv, b0, nb, gga, ws, 0, s);
        pdfxc::launch_gemm_x_planes(gv, ctx->d_P, nao, b0, nb, c.max_nbp, 0, nphi, 1, ws, s);
        pdfxc::launch_gemm_x_planes(gv, ctx->d_P_b, nao, b0, nb, c.max_nbp, 0, nphi + 1, 1, ws, s);
        pdfxc::launch_rho_functional_uks(gv, b0, nb, functional, incremental, ctx->opt.rho_cutoff, ws, ctx->d_rho,
                                         ctx->d_rho_b, ctx->d_blk_sum, ctx->d_blk_sum_b, s);
        pdfxc::launch_gemm_v_plane(gv, b0, nb, c.max_nbp, nphi, ws, ctx->d_Vacc, nao, s);
        pdfxc::launch_gemm_v_plane(gv, b0, nb, c.max_nbp, nphi + 1, ws, ctx->d_Vacc_b, nao, s);
        PDFXC_CUDA(cudaGetLastError());
        launches += 6;
    }
    return launches;
}

// The open-shell build on the INT8 path, per chunk: the phi digits and P_A's P_sub digits, the
// rho_A contraction, P_B's P_sub digits over the same region, the rho_B contraction, the
// open-shell functional (both spins' coefficients), then per spin its Z' digits and its Vxc
// contraction. The beta spin's P words, accumulators, coefficients and work counters have their
// own buffers; the workspace of the closed-shell build is reused. Returns the launch count.
int64_t enqueue_uks_int8(pdfxc_ctx* ctx, int functional, bool incremental) {
    cudaStream_t s = ctx->stream;
    const int nao = ctx->nao;
    const size_t n2 = (size_t)nao * nao, nslot = (size_t)ctx->nblk * BLOCK_PTS;
    if (!ctx->d_p_words_b) dev_alloc(&ctx->d_p_words_b, n2);
    if (!ctx->d_p_rowexp_b) dev_alloc(&ctx->d_p_rowexp_b, (size_t)nao);
    if (!ctx->d_rho_acc_b) dev_alloc(&ctx->d_rho_acc_b, nslot * 4);
    if (!ctx->d_coef_b) dev_alloc(&ctx->d_coef_b, nslot * 4);
    if (!ctx->d_counters_b) dev_alloc(&ctx->d_counters_b, 2 * ctx->chunks.size());
    memset_async(ctx->d_rho_acc, sizeof(double) * nslot * 4, s);
    memset_async(ctx->d_rho_acc_b, sizeof(double) * nslot * 4, s);
    PDFXC_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), s));
    PDFXC_CUDA(cudaMemsetAsync(ctx->d_counters, 0, sizeof(int) * 2 * ctx->chunks.size(), s));
    PDFXC_CUDA(cudaMemsetAsync(ctx->d_counters_b, 0, sizeof(int) * 2 * ctx->chunks.size(), s));
    pdfxc::oz_p_digits(ctx->d_P, nao, ctx->d_row_cols, ctx->d_p_rowexp, ctx->d_p_words, s);
    pdfxc::oz_p_digits(ctx->d_P_b, nao, ctx->d_row_cols, ctx->d_p_rowexp_b, ctx->d_p_words_b, s);
    int64_t launches = 2;
    const pdfxc::BasisView bv = basis_view(ctx);
    const pdfxc::GridView gv = grid_view(ctx);
    char* ws = static_cast<char*>(ctx->d_ws);
    for (size_t ci = 0; ci < ctx->chunks.size(); ++ci) {
        const Chunk& c = ctx->chunks[ci];
        const int cb0 = std::max(c.b0, ctx->blk_lo), cn = std::min(c.b1, ctx->blk_hi) - cb0;
        if (cn <= 0) continue;
        const int g_lo = (int)(std::lower_bound(ctx->h_grp.begin(), ctx->h_grp.end(), cb0) - ctx->h_grp.begin());
        const int g_hi = (int)(std::lower_bound(ctx->h_grp.begin(), ctx->h_grp.end(), cb0 + cn) - ctx->h_grp.begin());
        pdfxc::MixedArgs a{bv, gv, cb0, cn, c.max_nbp, functional, incremental ? 1 : 0, ctx->opt.split_terms, nao,
                           ctx->opt.rho_cutoff, ctx->d_P, ws, ctx->d_rho_acc, ctx->d_rho, ctx->d_coef, ctx->d_blk_sum,
                           ctx->d_Vacc, ctx->d_err, ctx->d_grp + g_lo, g_hi - g_lo, ctx->d_p_rowexp,
                           ctx->d_p_words, ctx->d_items + ctx->items_off_rho[ci], ctx->items_n_rho[ci],
                           ctx->d_items + ctx->items_off_vxc[ci], ctx->items_n_vxc[ci], ctx->d_counters + 2 * ci,
                           ctx->tuned_stages, ctx->phi_map_ok ? &ctx->phi_map : nullptr};
        pdfxc::MixedArgs b = a;  // the beta spin
        b.P = ctx->d_P_b, b.rho_acc = ctx->d_rho_acc_b, b.rho_store = ctx->d_rho_b, b.coef = ctx->d_coef_b;
        b.Vacc = ctx->d_Vacc_b, b.p_rowexp = ctx->d_p_rowexp_b, b.p_words = ctx->d_p_words_b;
        b.counters = ctx->d_counters_b + 2 * ci;
        pdfxc::oz_prepare(a, s);
        pdfxc::oz_rho(a, s);
        pdfxc::oz_pack_p(b, s);
        pdfxc::oz_rho(b, s);
        pdfxc::oz_functional_uks(a, b.rho_acc, b.rho_store, b.coef, ctx->d_blk_sum_b, s);
        pdfxc::oz_pack_z(a, s);
        pdfxc::oz_vxc(a, s);
        pdfxc::oz_pack_z(b, s);
        pdfxc::oz_vxc(b, s);
        PDFXC_CUDA(cudaGetLastError());
        launches += 9;
    }
    return launches;
}

// One build on ctx->stream. The sequence of launches is captured once into a
// CUDA graph per (functional, incremental, density pointer) and replayed.
void run_build(pdfxc_ctx* ctx, int fn, const double* d_PA, bool incremental) {
    ctx->last_staged = !ctx->use_graph || ctx->profiling;
    if (ctx->last_staged) {
        PDFXC_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream));
        enqueue_build(ctx, fn, d_PA, incremental);
        PDFXC_CUDA(cudaEventRecord(ctx->ev[1], ctx->stream));
        return;
    }
    if (!ctx->graph_exec || ctx->graph_fn != fn || ctx->graph_inc != (int)incremental || ctx->graph_P != d_PA) {
        drop_graph(ctx);
        cudaGraph_t g = nullptr;
        PDFXC_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue_build(ctx, fn, d_PA, incremental);
        } catch (...) {
            cudaStreamEndCapture(ctx->stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        PDFXC_CUDA(cudaStreamEndCapture(ctx->stream, &g));
        cudaError_t e = cudaGraphInstantiate(&ctx->graph_exec, g, 0);
        cudaGraphDestroy(g);
        PDFXC_CUDA(e);
        ctx->graph_fn = fn, ctx->graph_inc = incremental, ctx->graph_P = d_PA;
    }
    PDFXC_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream));
    PDFXC_CUDA(cudaGraphLaunch(ctx->graph_exec, ctx->stream));
    PDFXC_CUDA(cudaEventRecord(ctx->ev[1], ctx->stream));
}

pdfxc_status check_build(pdfxc_ctx* ctx, int functional, int incremental) {
    if (ctx->nblk == 0) {
        ctx->err = "pdfxc_build_vxc: call pdfxc_set_system and pdfxc_set_grid first";
        return PDFXC_ERR_STATE;
    }
    if (functional < PDFXC_SVWN || functional > PDFXC_PBE) {
        ctx->err = "pdfxc_build_vxc: unknown functional id " + std::to_string(functional);
        return PDFXC_ERR_ARG;
    }
    if (incremental && (!ctx->rho_valid || ctx->rho_spin != 1 ||
                        ctx->rho_gga != (int)pdfxc::functional_is_gga(functional))) {
        ctx->err = "pdfxc_build_vxc: incremental build needs a previous closed-shell build (or pdfxc_set_rho) of the "
                   "same functional type";
        return PDFXC_ERR_STATE;
    }
    return PDFXC_OK;
}

}  // namespace

extern "C" {

pdfxc_status pdfxc_build_vxc_device(pdfxc_ctx* ctx, int functional, const double* d_PA, int incremental, double* d_V,
                                    double* exc, double* nelec_alpha) {
    return guarded(ctx, [&]() -> pdfxc_status {
        pdfxc_status st = check_build(ctx, functional, incremental);
        if (st) return st;
        if (!d_PA || !d_V) {
            ctx->err = "pdfxc_build_vxc_device: null device pointer";
            return PDFXC_ERR_ARG;
        }
        run_build(ctx, functional, d_PA, incremental != 0);
        const size_t n2 = (size_t)ctx->nao * ctx->nao;
        PDFXC_CUDA(cudaMemcpyAsync(d_V, ctx->d_V, n2 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        double sc[2];
        PDFXC_CUDA(cudaMemcpyAsync(sc, ctx->d_scalars, sizeof(sc), cudaMemcpyDeviceToHost, ctx->stream));
        PDFXC_CUDA(cudaStreamSynchronize(ctx->stream));
        collect_profile(ctx);
        if (int code = device_error(ctx)) {
            ctx->err = "a bounded device wait expired in the tensor-core contraction (code " + std::to_string(code) + ")";
            return PDFXC_ERR_TIMEOUT;
        }
        if (exc) *exc = sc[0];
        if (nelec_alpha) *nelec_alpha = sc[1];
        ctx->rho_valid = true;
        ctx->rho_gga = pdfxc::functional_is_gga(functional);
        ctx->rho_spin = 1;
        return PDFXC_OK;
    });
}

pdfxc_status pdfxc_build_vxc_delta_device(pdfxc_ctx* ctx, int functional, const double* d_PA, int incremental,
                                          int iteration, double* d_V, double* d_dV, double* exc, double* nelec_alpha) {
    return guarded(ctx, [&]() -> pdfxc_status {
        pdfxc_status st = check_build(ctx, functional, incremental);
        if (st) return st;
        if (!d_PA || !d_dV) {
            ctx->err = "pdfxc_build_vxc_delta_device: null device pointer";
            return PDFXC_ERR_ARG;
        }
        if (iteration < 1) {
            ctx->err = "pdfxc_build_vxc_delta_device: iteration must be >= 1";
            return PDFXC_ERR_ARG;
        }
        if (iteration >= 2 && ctx->vprev_iter != iteration - 1) {
            ctx->err = "pdfxc_build_vxc_delta_device: the context holds no Vxc of iteration " +
                       std::to_string(iteration - 1);
            return PDFXC_ERR_STATE;
        }
        const size_t n2 = (size_t)ctx->nao * ctx->nao;
        if (!ctx->d_Vprev) dev_alloc(&ctx->d_Vprev, n2);
        // the difference kernel overwrites d_Vprev: until this call has completed, the context
        // holds no usable previous iteration
        ctx->vprev_iter = 0;
        run_build(ctx, functional, d_PA, incremental != 0);
        if (d_V) PDFXC_CUDA(cudaMemcpyAsync(d_V, ctx->d_V, n2 * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
        pdfxc::launch_fock_delta(ctx->d_V, ctx->d_Vprev, d_dV, n2, iteration >= 2, ctx->stream);
        PDFXC_LAUNCHED("fock delta");
        double sc[2];
        PDFXC_CUDA(cudaMemcpyAsync(sc, ctx->d_scalars, sizeof(sc), cudaMemcpyDeviceToHost, ctx->stream));
        PDFXC_CUDA(cudaStreamSynchronize(ctx->stream));
        collect_profile(ctx);
        if (int code = device_error(ctx)) {
            ctx->vprev_iter = 0;
            ctx->err = "a bounded device wait expired in the tensor-core contraction (code " + std::to_string(code) + ")";
            return PDFXC_ERR_TIMEOUT;
        }
        ctx->vprev_iter = iteration;
        if (exc) *exc = sc[0];
        if (nelec_alpha) *nelec_alpha = sc[1];
        ctx->rho_valid = true;
        ctx->rho_gga = pdfxc::functional_is_gga(functional);
        ctx->rho_spin = 1;
        return PDFXC_OK;
    });
}

pdfxc_status pdfxc_build_vxc(pdfxc_ctx* ctx, int functional, const double* PA, int incremental, double* F, double* exc,
                             double* nelec_alpha) {
    return guarded(ctx, [&]() -> pdfxc_status {
        pdfxc_status st = check_build(ctx, functional, incremental);
        if (st) return st;
        if (!PA || !F) {
            ctx->err = "pdfxc_build_vxc: null host pointer";
            return PDFXC_ERR_ARG;
        }
        const size_t n2 = (size_t)ctx->nao * ctx->nao;
        PDFXC_CUDA(cudaMemcpyAsync(ctx->d_P, PA, n2 * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        run_build(ctx, functional, ctx->d_P, incremental != 0);
        double sc[2];
        PDFXC_CUDA(cudaMemcpyAsync(sc, ctx->d_scalars, sizeof(sc), cudaMemcpyDeviceToHost, ctx->stream));
        PDFXC_CUDA(cudaStreamSynchronize(ctx->stream));
        collect_profile(ctx);
        if (int code = device_error(ctx)) {
            ctx->err = "a bounded device wait expired in the tensor-core contraction (code " + std::to_string(code) + ")";
            return PDFXC_ERR_TIMEOUT;
        }
        accumulate_to_host(ctx, ctx->d_V, F, n2);
        if (exc) *exc = sc[0];
        if (nelec_alpha) *nelec_alpha = sc[1];
        ctx->rho_valid = true;
        ctx->rho_gga = pdfxc::functional_is_gga(functional);
        ctx->rho_spin = 1;
        return PDFXC_OK;
    });
}

pdfxc_status pdfxc_get_rho(pdfxc_ctx* ctx, int gga, double* rho) {
    return guarded(ctx, [&]() -> pdfxc_status {
        if (!rho) return PDFXC_ERR_ARG;
        if (ctx->nblk == 0) {
            ctx->err = "pdfxc_get_rho: no grid";
            return PDFXC_ERR_STATE;
        }
        std::vector<double> r((size_t)ctx->nblk * BLOCK_PTS * 4);
        PDFXC_CUDA(cudaMemcpyAsync(r.data(), ctx->d_rho, r.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        PDFXC_CUDA(cudaStreamSynchronize(ctx->stream));
        const int nc = gga ? 4 : 1;
        for (size_t slot = 0; slot < ctx->h_src.size(); ++slot) {
            const int64_t i = ctx->h_src[slot];
            if (i < 0) continue;
            for (int k = 0; k < nc; ++k) rho[i * nc + k] = r[slot * 4 + k];
        }
        return PDFXC_OK;
    });
}

pdfxc_status pdfxc_density(pdfxc_ctx* ctx, const double* P, int64_t npts, const double* xyz, double* rho) {
    return guarded(ctx, [&]() -> pdfxc_status {
        if (ctx->natom == 0) {
            ctx->err = "pdfxc_density: call pdfxc_set_system first";
            return PDFXC_ERR_STATE;
        }
        if (npts < 0 || (npts > 0 && (!P || !xyz || !rho))) {
            ctx->err = "pdfxc_density: negative count or null pointer";
            return PDFXC_ERR_ARG;
        }
        if (npts == 0) return PDFXC_OK;
        auto sub_check = [&](pdfxc_status st, const char* what) {
            if (st != PDFXC_OK) throw std::runtime_error(std::string("pdfxc_density: ") + what + ": " + ctx->dens->err);
        };
        if (!ctx->dens) {
            pdfxc_options o;
            pdfxc_default_options(&o);
            o.ao_cutoff = ctx->opt.ao_cutoff;
            o.workspace_bytes = ctx->opt.workspace_bytes;
            if (pdfxc_create(&ctx->dens, ctx->device, &o) != PDFXC_OK) throw std::runtime_error("pdfxc_density: create");
            sub_check(pdfxc_set_system(ctx->dens, ctx->natom, ctx->h_atom_xyz.data(), ctx->h_atom_z.data(), ctx->nshell,
                                       ctx->h_sh_atom.data(), ctx->h_sh_l.data(), ctx->h_sh_nprim.data(),
                                       ctx->h_p_exp.data(), ctx->h_p_coef.data()),
                      "set_system");
        }
        pdfxc_ctx* d = ctx->dens;
        // the points as a grid of zero weights: the FP64 rho kernel stores rho at every
        // point and evaluates the functional only where the weight is non-zero
        std::vector<double> xyzw(4 * (size_t)npts);
        for (int64_t i = 0; i < npts; ++i)
            xyzw[4 * i] = xyz[3 * i], xyzw[4 * i + 1] = xyz[3 * i + 1], xyzw[4 * i + 2] = xyz[3 * i + 2], xyzw[4 * i + 3] = 0.0;
        sub_check(pdfxc_set_grid(d, npts, xyzw.data(), nullptr), "set_grid");
        cudaStream_t s = d->stream;
        const int nao = d->nao;
        PDFXC_CUDA(cudaMemcpyAsync(d->d_P, P, sizeof(double) * nao * nao, cudaMemcpyHostToDevice, s));
        const pdfxc::BasisView bv = basis_view(d);
        const pdfxc::GridView gv = grid_view(d);
        char* ws = static_cast<char*>(d->d_ws);
        for (const Chunk& c : d->chunks) {
            const int nb = c.b1 - c.b0;
            pdfxc::launch_ao_eval(bv, gv, c.b0, nb, false, ws, 0, s);
            pdfxc::launch_gemm_x(gv, d->d_P, nao, c.b0, nb, c.max_nbp, 1, ws, s);
            pdfxc::launch_rho_functional(gv, c.b0, nb, PDFXC_SVWN, false, d->opt.rho_cutoff, ws, d->d_rho, d->d_coef,
                                         d->d_blk_sum, s);
            PDFXC_LAUNCHED("density (AO values, X, rho)");
        }
        sub_check(pdfxc_get_rho(d, 0, rho), "get_rho");
        return PDFXC_OK;
    });
}

pdfxc_status pdfxc_set_rho(pdfxc_ctx* ctx, int gga, const double* rho) {
    return guarded(ctx, [&]() -> pdfxc_status {
        if (!rho) return PDFXC_ERR_ARG;
        if (ctx->nblk == 0) {
            ctx->err = "pdfxc_set_rho: no grid";
            return PDFXC_ERR_STATE;
        }
        std::vector<double> r((size_t)ctx->nblk * BLOCK_PTS * 4, 0.0);
        const int nc = gga ? 4 : 1;
        for (size_t slot = 0; slot < ctx->h_src.size(); ++slot) {
            const int64_t i = ctx->h_src[slot];
            if (i < 0) continue;
            for (int k = 0; k < nc; ++k) r[slot * 4 + k] = rho[i * nc + k];
        }
        PDFXC_CUDA(cudaMemcpyAsync(ctx->d_rho, r.data(), r.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        PDFXC_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->rho_valid = true;
        ctx->rho_gga = gga ? 1 : 0;
        ctx->rho_spin = 1;
        return PDFXC_OK;
    });
}

pdfxc_status pdfxc_build_vxc_uks(pdfxc_ctx* ctx, int functional, const double* PA, const double* PB, int incremental,
                                 double* FA, double* FB, double* exc, double* nelec_alpha, double* nelec_beta) {
    return guarded(ctx, [&]() -> pdfxc_status {
        if (ctx->nblk == 0) {
            ctx->err = "pdfxc_build_vxc_uks: call pdfxc_set_system and pdfxc_set_grid first";
            return PDFXC_ERR_STATE;
        }
        if (functional < PDFXC_SVWN || functional > PDFXC_PBE || !PA || !PB || !FA || !FB) {
            ctx->err = "pdfxc_build_vxc_uks: unknown functional or null pointer";
            return PDFXC_ERR_ARG;
        }
        const bool int8 = ctx->opt.precision == PDFXC_PRECISION_MIXED;
        if (int8 && ctx->opt.split_terms != 10) {
            ctx->err = "pdfxc_build_vxc_uks: the open-shell build runs on the FP64 path and on the INT8 digits "
                       "(split_terms 10), not on the BF16 split";
            return PDFXC_ERR_UNSUPPORTED;
        }
        const bool gga = pdfxc::functional_is_gga(functional);
        if (incremental && (!ctx->rho_valid || ctx->rho_spin != 2 || ctx->rho_gga != (int)gga)) {
            ctx->err = "pdfxc_build_vxc_uks: incremental build needs a previous open-shell build (or "
                       "pdfxc_set_rho_uks) of the same functional type";
            return PDFXC_ERR_STATE;
        }
        const int nao = ctx->nao;
        const size_t n2 = (size_t)nao * nao;
        cudaStream_t s = ctx->stream;
        if (!ctx->d_P_b) dev_alloc(&ctx->d_P_b, n2);
        if (!ctx->d_V_b) dev_alloc(&ctx->d_V_b, n2);
        if (!ctx->d_Vacc_b) dev_alloc(&ctx->d_Vacc_b, n2);
        if (!ctx->d_scalars_b) dev_alloc(&ctx->d_scalars_b, 2);
        if (!ctx->d_rho_b) {
            dev_alloc(&ctx->d_rho_b, (size_t)ctx->nblk * BLOCK_PTS * 4);
            PDFXC_CUDA(cudaMemsetAsync(ctx->d_rho_b, 0, sizeof(double) * (size_t)ctx->nblk * BLOCK_PTS * 4, s));
        }
        if (!ctx->d_blk_sum_b) dev_alloc(&ctx->d_blk_sum_b, (size_t)ctx->nblk * 2);
        PDFXC_CUDA(cudaMemcpyAsync(ctx->d_P, PA, n2 * sizeof(double), cudaMemcpyHostToDevice, s));
        PDFXC_CUDA(cudaMemcpyAsync(ctx->d_P_b, PB, n2 * sizeof(double), cudaMemcpyHostToDevice, s));
        memset_async(ctx->d_Vacc, n2 * sizeof(double), s);
        memset_async(ctx->d_Vacc_b, n2 * sizeof(double), s);
        PDFXC_CUDA(cudaEventRecord(ctx->ev[0], s));
        const int64_t launches = int8 ? enqueue_uks_int8(ctx, functional, incremental != 0)
                                      : enqueue_uks_fp64(ctx, functional, incremental != 0);
        const size_t lo = ctx->blk_lo;
        const int nr = ctx->blk_hi - ctx->blk_lo;
        pdfxc::launch_finish(ctx->d_Vacc, ctx->d_V, nao, ctx->d_blk_sum + 2 * lo, nr, ctx->d_scalars, s);
        pdfxc::launch_finish(ctx->d_Vacc_b, ctx->d_V_b, nao, ctx->d_blk_sum_b + 2 * lo, nr, ctx->d_scalars_b, s);
        PDFXC_CUDA(cudaEventRecord(ctx->ev[1], s));
        PDFXC_CUDA(cudaGetLastError());
        double sa[2], sb[2];
        PDFXC_CUDA(cudaMemcpyAsync(sa, ctx->d_scalars, sizeof(sa), cudaMemcpyDeviceToHost, s));
        PDFXC_CUDA(cudaMemcpyAsync(sb, ctx->d_scalars_b, sizeof(sb), cudaMemcpyDeviceToHost, s));
        PDFXC_CUDA(cudaStreamSynchronize(s));
        if (int code = int8 ? device_error(ctx) : 0) {
            ctx->err = "pdfxc_build_vxc_uks: a bounded device wait expired (code " + std::to_string(code) + ")";
            return PDFXC_ERR_TIMEOUT;
        }
        pdfxc_profile& p = ctx->last_profile;
        p = pdfxc_profile{};
        PDFXC_CUDA(cudaEventElapsedTime(&p.total_ms, ctx->ev[0], ctx->ev[1]));
        p.launches = launches + 4;
        accumulate_to_host(ctx, ctx->d_V, FA, n2);
        accumulate_to_host(ctx, ctx->d_V_b, FB, n2);
        if (exc) *exc = sa[0];
        if (nelec_alpha) *nelec_alpha = sa[1];
        if (nelec_beta) *nelec_beta = sb[0];
        ctx->rho_valid = true;
        ctx->rho_gga = gga;
        ctx->rho_spin = 2;
        return PDFXC_OK;
    });
}

pdfxc_status pdfxc_get_rho_uks(pdfxc_ctx* ctx, int gga, double* rho) {
    return guarded(ctx, [&]() -> pdfxc_status {
        if (!rho) return PDFXC_ERR_ARG;
        if (ctx->nblk == 0 || !ctx->d_rho_b) {
            ctx->err = "pdfxc_get_rho_uks: no open-shell densities (no grid or no open-shell build)";
            return PDFXC_ERR_STATE;
        }
        const size_t ns = (size_t)ctx->nblk * BLOCK_PTS * 4;
        std::vector<double> ra(ns), rb(ns);
        PDFXC_CUDA(cudaMemcpyAsync(ra.data(), ctx->d_rho, ns * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        PDFXC_CUDA(cudaMemcpyAsync(rb.data(), ctx->d_rho_b, ns * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        PDFXC_CUDA(cudaStreamSynchronize(ctx->stream));
        const int nc = gga ? 4 : 1;
        for (size_t slot = 0; slot < ctx->h_src.size(); ++slot) {
            const int64_t i = ctx->h_src[slot];
            if (i < 0) continue;
            for (int k = 0; k < nc; ++k) rho[i * 2 * nc + k] = ra[slot * 4 + k], rho[i * 2 * nc + nc + k] = rb[slot * 4 + k];
        }
        return PDFXC_OK;
    });
}

pdfxc_status pdfxc_set_rho_uks(pdfxc_ctx* ctx, int gga, const double* rho) {
    return guarded(ctx, [&]() -> pdfxc_status {
        if (!rho) return PDFXC_ERR_ARG;
        if (ctx->nblk == 0) {
            ctx->err = "pdfxc_set_rho_uks: no grid";
            return PDFXC_ERR_STATE;
        }
        const size_t ns = (size_t)ctx->nblk * BLOCK_PTS * 4;
        std::vector<double> ra(ns, 0.0), rb(ns, 0.0);
        const int nc = gga ? 4 : 1;
        for (size_t slot = 0; slot < ctx->h_src.size(); ++slot) {
            const int64_t i = ctx->h_src[slot];
            if (i < 0) continue;
            for (int k = 0; k < nc; ++k) ra[slot * 4 + k] = rho[i * 2 * nc + k], rb[slot * 4 + k] = rho[i * 2 * nc + nc + k];
        }
        if (!ctx->d_rho_b) dev_alloc(&ctx->d_rho_b, ns);
        PDFXC_CUDA(cudaMemcpyAsync(ctx->d_rho, ra.data(), ns * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        PDFXC_CUDA(cudaMemcpyAsync(ctx->d_rho_b, rb.data(), ns * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
        PDFXC_CUDA(cudaStreamSynchronize(ctx->stream));
        ctx->rho_valid = true;
        ctx->rho_gga = gga ? 1 : 0;
        ctx->rho_spin = 2;
        return PDFXC_OK;
    });
}

}  // extern "C"

namespace {

// The XC nuclear gradient (pdfxc_xc_gradient) and the adjoint of Exc (pdfxc_xc_backward): per
// chunk phi, grad phi and the second derivatives are recomputed (k_ao_grad), X = P_sub phi
// (k_gemm_x), then the functional and the AO-centre term per point (k_grad_point); with
// dexc_dP, the density adjoint Z replaces X and Vacc += phi Z^T (k_gemm_v), then
// dexc_dP = Vacc + Vacc^T. Every derivative is scaled by `seed`.
pdfxc_status xc_derivatives(pdfxc_ctx* ctx, const char* name, int functional, const double* PA,
                            const double* w_single, const double* becke_radius, int size_adjust, double seed,
                            double* grad_orbital, double* grad_weight, double* dexc_dP, double* exc) {
    return guarded(ctx, [&]() -> pdfxc_status {
        if (ctx->nblk == 0) {
            ctx->err = std::string(name) + ": call pdfxc_set_system and pdfxc_set_grid first";
            return PDFXC_ERR_STATE;
        }
        if (ctx->h_owner.empty()) {
            ctx->err = std::string(name) + ": the grid was set without owner atoms (pass atom to pdfxc_set_grid)";
            return PDFXC_ERR_STATE;
        }
        if (functional < PDFXC_SVWN || functional > PDFXC_PBE || !PA || !grad_orbital) {
            ctx->err = std::string(name) + ": unknown functional or null pointer";
            return PDFXC_ERR_ARG;
        }
        if (w_single && (!becke_radius || !grad_weight)) {
            ctx->err = std::string(name) + ": the weight term needs becke_radius and grad_weight";
            return PDFXC_ERR_ARG;
        }
        const bool gga = pdfxc::functional_is_gga(functional);
        const int nao = ctx->nao, natom = ctx->natom;
        cudaStream_t s = ctx->stream;
        if (!ctx->d_ao_atom) {
            std::vector<int> ao_atom(nao);
            for (int sh = 0; sh < ctx->nshell; ++sh)
                for (int c = 0; c < 2 * ctx->h_sh_l[sh] + 1; ++c) ao_atom[ctx->h_sh_ao0[sh] + c] = ctx->h_sh_atom[sh];
            upload(&ctx->d_ao_atom, ao_atom, s);
        }
        if (!ctx->d_owner) upload(&ctx->d_owner, ctx->h_owner, s);
        // gradient workspace: its own per-block offsets and chunks
        ensure_plan(ctx, ctx->gplan, pdfxc::grad_workspace_planes(gga));
        const size_t nslots = (size_t)ctx->nblk * BLOCK_PTS;
        if (!ctx->d_grad) dev_alloc(&ctx->d_grad, 6 * (size_t)natom);
        if (!ctx->d_fdens) dev_alloc(&ctx->d_fdens, nslots);
        PDFXC_CUDA(cudaMemsetAsync(ctx->d_grad, 0, sizeof(double) * 6 * natom, s));
        PDFXC_CUDA(cudaMemcpyAsync(ctx->d_P, PA, sizeof(double) * nao * nao, cudaMemcpyHostToDevice, s));
        if (dexc_dP) memset_async(ctx->d_Vacc, sizeof(double) * (size_t)nao * nao, s);
        pdfxc::GridView gv = grid_view(ctx);
        gv.meta = ctx->gplan.d_meta;
        const pdfxc::BasisView bv = basis_view(ctx);
        char* ws = static_cast<char*>(ctx->gplan.d_ws);
        for (const Chunk& ch : ctx->gplan.chunks) {
            const int b0 = std::max(ch.b0, ctx->blk_lo), n = std::min(ch.b1, ctx->blk_hi) - b0;
            if (n <= 0) continue;
            pdfxc::launch_ao_grad(bv, gv, b0, n, gga, ws, s);
            pdfxc::launch_grad_x(gv, ctx->d_P, nao, b0, n, ch.max_nbp, gga, ws, s);
            pdfxc::launch_grad_point(gv, ctx->d_ao_atom, ctx->d_owner, b0, n, functional, ctx->opt.rho_cutoff, ws,
                                     seed, dexc_dP != nullptr, ctx->d_fdens, ctx->d_blk_sum, ctx->d_grad, s);
            if (dexc_dP)
                pdfxc::launch_gemm_v_plane(gv, b0, n, ch.max_nbp, pdfxc::grad_z_plane(gga), ws, ctx->d_Vacc, nao, s);
            PDFXC_CUDA(cudaGetLastError());
        }
        pdfxc::launch_block_sums(ctx->d_blk_sum + 2 * (size_t)ctx->blk_lo, ctx->blk_hi - ctx->blk_lo, ctx->d_scalars, s);
        if (w_single) {
            std::vector<double> wslot(nslots, 0.0);
            for (size_t k = 0; k < nslots; ++k)
                if (ctx->h_src[k] >= 0) wslot[k] = w_single[ctx->h_src[k]];
            upload(&ctx->d_wslot, wslot, s);
            std::vector<double> brad(becke_radius, becke_radius + natom);
            upload(&ctx->d_brad, brad, s);
            dev_alloc(&ctx->d_pair, 2 * (size_t)natom * natom);
            double* inv = ctx->d_pair;
            double* adj = ctx->d_pair + (size_t)natom * natom;
            pdfxc::launch_becke_pairs(ctx->d_atom_xyz, ctx->d_brad, natom, size_adjust, inv, adj, s);
            // the slots of this context's block range
            const size_t s0 = (size_t)ctx->blk_lo * BLOCK_PTS;
            const int64_t ns = (int64_t)(ctx->blk_hi - ctx->blk_lo) * BLOCK_PTS;
            // atom rows in device memory above the shared-memory limit (or when the environment asks for
            // that form: PDFXC_GRAD_WEIGHT_ROWS=dram, used by the tests to compare the two forms)
            const char* rows_env = std::getenv("PDFXC_GRAD_WEIGHT_ROWS");
            const bool dram_rows = natom > pdfxc::grad_weight_max_atoms() ||
                                   (rows_env && std::string(rows_env) == "dram");
            if (dram_rows) dev_alloc(&ctx->d_wscratch, pdfxc::grad_weight_scratch_doubles(natom));
            pdfxc::launch_grad_weight(ctx->d_atom_xyz, natom, inv, adj, ns, ctx->d_px + s0, ctx->d_py + s0,
                                      ctx->d_pz + s0, ctx->d_owner + s0, ctx->d_wslot + s0, ctx->d_fdens + s0,
                                      ctx->d_grad + 3 * natom, dram_rows ? ctx->d_wscratch : nullptr, s);
            PDFXC_CUDA(cudaGetLastError());
        }
        std::vector<double> g(6 * (size_t)natom);
        double sc[2];
        if (dexc_dP) {
            pdfxc::launch_finish(ctx->d_Vacc, ctx->d_V, nao, ctx->d_blk_sum + 2 * (size_t)ctx->blk_lo,
                                 ctx->blk_hi - ctx->blk_lo, ctx->d_scalars, s);
            PDFXC_LAUNCHED("dExc/dP symmetrisation");
            PDFXC_CUDA(cudaMemcpyAsync(dexc_dP, ctx->d_V, sizeof(double) * (size_t)nao * nao, cudaMemcpyDeviceToHost, s));
        }
        PDFXC_CUDA(cudaMemcpyAsync(g.data(), ctx->d_grad, sizeof(double) * g.size(), cudaMemcpyDeviceToHost, s));
        PDFXC_CUDA(cudaMemcpyAsync(sc, ctx->d_scalars, sizeof(sc), cudaMemcpyDeviceToHost, s));
        PDFXC_CUDA(cudaStreamSynchronize(s));
        std::copy(g.begin(), g.begin() + 3 * natom, grad_orbital);
        if (w_single) std::copy(g.begin() + 3 * natom, g.end(), grad_weight);
        if (exc) *exc = sc[0];
        return PDFXC_OK;
    });
}

}  // namespace

extern "C" {

pdfxc_status pdfxc_xc_gradient(pdfxc_ctx* ctx, int functional, const double* PA, const double* w_single,
                               const double* becke_radius, int size_adjust, double* grad_orbital, double* grad_weight,
                               double* exc) {
    return xc_derivatives(ctx, "pdfxc_xc_gradient", functional, PA, w_single, becke_radius, size_adjust, 1.0,
                          grad_orbital, grad_weight, nullptr, exc);
}

pdfxc_status pdfxc_xc_backward(pdfxc_ctx* ctx, int functional, const double* PA, double dexc,
                               const double* w_single, const double* becke_radius, int size_adjust,
                               double* dexc_dP, double* grad_orbital, double* grad_weight, double* exc) {
    if (ctx && !dexc_dP) {
        ctx->err = "pdfxc_xc_backward: null dexc_dP";
        return PDFXC_ERR_ARG;
    }
    return xc_derivatives(ctx, "pdfxc_xc_backward", functional, PA, w_single, becke_radius, size_adjust, dexc,
                          grad_orbital, grad_weight, dexc_dP, exc);
}


pdfxc_status pdfxc_set_batch(pdfxc_ctx* ctx, int nmol, const pdfxc_mol* mols) {
    if (!ctx) return PDFXC_ERR_ARG;
    if (nmol <= 0 || !mols) {
        ctx->err = "pdfxc_set_batch: no molecules";
        return PDFXC_ERR_ARG;
    }
    std::vector<double> xyz, pexp, pcoef, xyzw;
    std::vector<int> z, shatom, shl, shnp, owner;
    std::vector<GridSegment> segs;
    std::vector<int> aoff(1, 0);
    int atom_off = 0, shell_off = 0;
    int64_t pt_off = 0;
    bool owners = true;
    for (int m = 0; m < nmol; ++m) {
        const pdfxc_mol& M = mols[m];
        if (M.natom <= 0 || M.nshell <= 0 || M.npts <= 0 || !M.atom_xyz || !M.shell_atom || !M.shell_l ||
            !M.shell_nprim || !M.prim_exp || !M.prim_coef || !M.xyzw) {
            ctx->err = "pdfxc_set_batch: molecule " + std::to_string(m) + " is empty or has a null pointer";
            return PDFXC_ERR_ARG;
        }
        xyz.insert(xyz.end(), M.atom_xyz, M.atom_xyz + 3 * M.natom);
        for (int a = 0; a < M.natom; ++a) z.push_back(M.atom_z ? M.atom_z[a] : 0);
        int np = 0, nao_m = 0;
        for (int sh = 0; sh < M.nshell; ++sh) {
            if (M.shell_atom[sh] < 0 || M.shell_atom[sh] >= M.natom) {
                ctx->err = "pdfxc_set_batch: molecule " + std::to_string(m) + ": shell atom out of range";
                return PDFXC_ERR_ARG;
            }
            shatom.push_back(M.shell_atom[sh] + atom_off);
            shl.push_back(M.shell_l[sh]);
            shnp.push_back(M.shell_nprim[sh]);
            np += M.shell_nprim[sh];
            nao_m += 2 * M.shell_l[sh] + 1;
        }
        pexp.insert(pexp.end(), M.prim_exp, M.prim_exp + np);
        pcoef.insert(pcoef.end(), M.prim_coef, M.prim_coef + np);
        xyzw.insert(xyzw.end(), M.xyzw, M.xyzw + 4 * M.npts);
        if (!M.atom) owners = false;
        for (int64_t i = 0; owners && i < M.npts; ++i) {
            if (M.atom[i] < 0 || M.atom[i] >= M.natom) {
                ctx->err = "pdfxc_set_batch: molecule " + std::to_string(m) + ": owner atom out of range";
                return PDFXC_ERR_ARG;
            }
            owner.push_back(M.atom[i] + atom_off);
        }
        segs.push_back(GridSegment{pt_off, pt_off + M.npts, shell_off, shell_off + M.nshell});
        aoff.push_back(aoff.back() + nao_m);
        atom_off += M.natom, shell_off += M.nshell, pt_off += M.npts;
    }
    pdfxc_status st = pdfxc_set_system(ctx, atom_off, xyz.data(), z.data(), shell_off, shatom.data(), shl.data(),
                                       shnp.data(), pexp.data(), pcoef.data());
    if (st != PDFXC_OK) return st;
    return guarded(ctx, [&]() -> pdfxc_status {
        build_grid(ctx, pt_off, xyzw.data(), owners ? owner.data() : nullptr, segs);
        ctx->mol = aoff;
        dev_alloc(&ctx->d_mol_sums, 2 * (size_t)nmol);
        // the joint P holds each molecule's P_A in its diagonal block and nothing else: rows
        // read only their own molecule's columns
        std::vector<int> cols(2 * (size_t)aoff.back());
        for (int m = 0; m < nmol; ++m)
            for (int r = aoff[m]; r < aoff[m + 1]; ++r) cols[2 * r] = aoff[m], cols[2 * r + 1] = aoff[m + 1];
        upload(&ctx->d_row_cols, cols, ctx->stream);
        PDFXC_CUDA(cudaStreamSynchronize(ctx->stream));
        return PDFXC_OK;
    });
}

pdfxc_status pdfxc_build_vxc_batched(pdfxc_ctx* ctx, int functional, const double* const* PA, int incremental,
                                     double* const* F, double* exc, double* nelec_alpha) {
    return guarded(ctx, [&]() -> pdfxc_status {
        if (ctx->mol.size() < 2) {
            ctx->err = "pdfxc_build_vxc_batched: call pdfxc_set_batch first";
            return PDFXC_ERR_STATE;
        }
        pdfxc_status st = check_build(ctx, functional, incremental);
        if (st) return st;
        const int nmol = (int)ctx->mol.size() - 1;
        if (!PA || !F) {
            ctx->err = "pdfxc_build_vxc_batched: null pointer array";
            return PDFXC_ERR_ARG;
        }
        for (int m = 0; m < nmol; ++m)
            if (!PA[m] || !F[m]) {
                ctx->err = "pdfxc_build_vxc_batched: null density or Fock pointer of molecule " + std::to_string(m);
                return PDFXC_ERR_ARG;
            }
        cudaStream_t s = ctx->stream;
        const size_t n = ctx->nao;
        // each molecule's P_A into its diagonal block of the joint matrix; the blocks of the
        // grid only touch their own molecule's AOs, so the off-diagonal blocks are never read
        for (int m = 0; m < nmol; ++m) {
            const size_t a0 = ctx->mol[m], nm = ctx->mol[m + 1] - ctx->mol[m];
            PDFXC_CUDA(cudaMemcpy2DAsync(ctx->d_P + a0 * n + a0, n * sizeof(double), PA[m], nm * sizeof(double),
                                         nm * sizeof(double), nm, cudaMemcpyHostToDevice, s));
        }
        run_build(ctx, functional, ctx->d_P, incremental != 0);
        pdfxc::launch_segment_sums(ctx->d_blk_sum, ctx->d_seg_blk, nmol, ctx->d_mol_sums, s);
        PDFXC_CUDA(cudaGetLastError());
        std::vector<std::vector<double>> V(nmol);
        std::vector<double> sums(2 * (size_t)nmol);
        for (int m = 0; m < nmol; ++m) {
            const size_t a0 = ctx->mol[m], nm = ctx->mol[m + 1] - ctx->mol[m];
            V[m].resize(nm * nm);
            PDFXC_CUDA(cudaMemcpy2DAsync(V[m].data(), nm * sizeof(double), ctx->d_V + a0 * n + a0, n * sizeof(double),
                                         nm * sizeof(double), nm, cudaMemcpyDeviceToHost, s));
        }
        PDFXC_CUDA(cudaMemcpyAsync(sums.data(), ctx->d_mol_sums, sums.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
        PDFXC_CUDA(cudaStreamSynchronize(s));
        collect_profile(ctx);
        if (int code = device_error(ctx)) {
            ctx->err = "a bounded device wait expired in the tensor-core contraction (code " + std::to_string(code) + ")";
            return PDFXC_ERR_TIMEOUT;
        }
        for (int m = 0; m < nmol; ++m) {
            double* Fm = F[m];
            for (size_t i = 0; i < V[m].size(); ++i) Fm[i] += V[m][i];
            if (exc) exc[m] = sums[2 * m];
            if (nelec_alpha) nelec_alpha[m] = sums[2 * m + 1];
        }
        ctx->rho_valid = true;
        ctx->rho_gga = pdfxc::functional_is_gga(functional);
        ctx->rho_spin = 1;
        return PDFXC_OK;
    });
}

pdfxc_status pdfxc_block_costs(pdfxc_ctx* ctx, double* cost) {
    return guarded(ctx, [&]() -> pdfxc_status {
        if (!cost) return PDFXC_ERR_ARG;
        if (ctx->nblk == 0) {
            ctx->err = "pdfxc_block_costs: no grid";
            return PDFXC_ERR_STATE;
        }
        for (int b = 0; b < ctx->nblk; ++b)
            cost[b] = 4.0 * double(ctx->h_meta[b].nb) * ctx->h_meta[b].nb * ctx->h_meta[b].npts;
        return PDFXC_OK;
    });
}

pdfxc_status pdfxc_set_block_range(pdfxc_ctx* ctx, int64_t b_lo, int64_t b_hi) {
    return guarded(ctx, [&]() -> pdfxc_status {
        if (ctx->nblk == 0) {
            ctx->err = "pdfxc_set_block_range: no grid";
            return PDFXC_ERR_STATE;
        }
        if (b_lo < 0 || b_hi > ctx->nblk || b_lo > b_hi) {
            ctx->err = "pdfxc_set_block_range: range outside [0, nblocks]";
            return PDFXC_ERR_ARG;
        }
        drop_graph(ctx);
        // a group is built whole, by the range that holds its first block: both ends move
        // up to the next group start (no move when every block is its own group)
        auto snap = [&](int64_t b) {
            const auto it = std::lower_bound(ctx->h_grp.begin(), ctx->h_grp.end(), (int)b);
            return it == ctx->h_grp.end() ? ctx->nblk : *it;
        };
        ctx->blk_lo = snap(b_lo), ctx->blk_hi = snap(b_hi);
        ctx->rho_valid = false;  // stored densities outside the new range are not this context's
        return PDFXC_OK;
    });
}

pdfxc_status pdfxc_partition_blocks(int64_t nblk, const double* cost, int nparts, int64_t* bounds) {
    if (nblk < 0 || nparts <= 0 || !bounds || (nblk > 0 && !cost)) return PDFXC_ERR_ARG;
    double total = 0.0;
    for (int64_t b = 0; b < nblk; ++b) {
        if (!(cost[b] >= 0.0)) return PDFXC_ERR_ARG;
        total += cost[b];
    }
    // contiguous ranges cut where the running cost crosses r / nparts of the total
    bounds[0] = 0;
    double run = 0.0;
    int64_t b = 0;
    for (int r = 1; r < nparts; ++r) {
        const double target = total * r / nparts;
        while (b < nblk && run + 0.5 * cost[b] < target) run += cost[b++];
        bounds[r] = std::max(b, bounds[r - 1]);
    }
    bounds[nparts] = nblk;
    return PDFXC_OK;
}

pdfxc_status pdfxc_plan_grid(const pdfxc_options* opt, int natom, const double* atom_xyz, int nshell,
                              const int* shell_atom, const int* shell_l, const int* shell_nprim,
                              const double* prim_exp, const double* prim_coef, int64_t npts, const double* xyzw,
                              pdfxc_grid_plan* out) {
    if (!out || npts <= 0 || !xyzw) return PDFXC_ERR_ARG;
    pdfxc_ctx c;  // host fields only: nothing here touches a device
    pdfxc_default_options(&c.opt);
    if (opt) c.opt = *opt;
    if (c.opt.block_points <= 0 || c.opt.block_points > BLOCK_PTS) c.opt.block_points = BLOCK_PTS;
    if (c.opt.workspace_bytes == 0) c.opt.workspace_bytes = size_t(4) << 30;
    if (c.opt.split_terms != 3 && c.opt.split_terms != 6 && c.opt.split_terms != 10) c.opt.split_terms = 10;
    if (c.opt.precision != PDFXC_PRECISION_FP64 && c.opt.precision != PDFXC_PRECISION_MIXED) return PDFXC_ERR_ARG;
    try {
        if (const pdfxc_status st = set_host_system(&c, natom, atom_xyz, nullptr, nshell, shell_atom, shell_l,
                                                    shell_nprim, prim_exp, prim_coef))
            return st;
        HostGrid G;
        resolve_shapes(&c, npts, 1);
        plan_grid(&c, npts, xyzw, nullptr, {GridSegment{0, npts, 0, c.nshell}}, G);
        out->nblocks = G.nblk;
        out->ngroups = G.ngrp;
        out->npts_padded = (int64_t)G.nblk * BLOCK_PTS;
        out->max_nb = G.max_nb;
        out->contraction_flops = G.flops;
        out->mean_nb = G.nblk ? G.sum_nb / G.nblk : 0.0;
        out->workspace_bytes = G.max_ws;
        out->nchunks = (int)c.chunks.size();
    } catch (const Unsupported&) {
        return PDFXC_ERR_UNSUPPORTED;
    } catch (const std::bad_alloc&) {
        return PDFXC_ERR_NOMEM;
    } catch (const std::exception&) {
        return PDFXC_ERR_ARG;
    }
    return PDFXC_OK;
}

pdfxc_status pdfxc_pack_upper(const double* d_V, int n, double* d_packed, void* stream) {
    if (n <= 0 || !d_V || !d_packed) return PDFXC_ERR_ARG;
    pdfxc::launch_pack_upper(d_V, n, d_packed, static_cast<cudaStream_t>(stream));
    return cudaPeekAtLastError() == cudaSuccess ? PDFXC_OK : PDFXC_ERR_CUDA;
}

pdfxc_status pdfxc_unpack_upper(const double* d_packed, int n, double* d_V, void* stream) {
    if (n <= 0 || !d_V || !d_packed) return PDFXC_ERR_ARG;
    pdfxc::launch_unpack_upper(d_packed, n, d_V, static_cast<cudaStream_t>(stream));
    return cudaPeekAtLastError() == cudaSuccess ? PDFXC_OK : PDFXC_ERR_CUDA;
}

pdfxc_status pdfxc_grid_stats(pdfxc_ctx* ctx, int64_t* nblocks, int64_t* npts_padded, double* contraction_flops,
                              double* mean_nb) {
    if (!ctx) return PDFXC_ERR_ARG;
    if (nblocks) *nblocks = ctx->nblk;
    if (npts_padded) *npts_padded = (int64_t)ctx->nblk * BLOCK_PTS;
    if (contraction_flops) *contraction_flops = ctx->contraction_flops;
    if (mean_nb) *mean_nb = ctx->mean_nb;
    return PDFXC_OK;
}

pdfxc_status pdfxc_set_profiling(pdfxc_ctx* ctx, int enable) {
    if (!ctx) return PDFXC_ERR_ARG;
    ctx->profiling = enable != 0;
    return PDFXC_OK;
}

pdfxc_status pdfxc_last_profile(pdfxc_ctx* ctx, pdfxc_profile* out) {
    if (!ctx || !out) return PDFXC_ERR_ARG;
    *out = ctx->last_profile;
    return PDFXC_OK;
}

pdfxc_status pdfxc_autotune(pdfxc_ctx* ctx, int functional, const double* d_PA, pdfxc_tuning* out, int max_out,
                            int* n_out) {
    return guarded(ctx, [&]() -> pdfxc_status {
        pdfxc_status st = check_build(ctx, functional, 0);
        if (st) return st;
        const bool int8 = ctx->opt.precision == PDFXC_PRECISION_MIXED && ctx->opt.split_terms == 10;
        // the grid as given, to block it again for every candidate
        const int64_t npts = ctx->npts;
        const size_t nslot = (size_t)ctx->nblk * BLOCK_PTS;
        std::vector<double> c[4] = {std::vector<double>(nslot), std::vector<double>(nslot), std::vector<double>(nslot),
                                    std::vector<double>(nslot)};
        const double* src[4] = {ctx->d_px, ctx->d_py, ctx->d_pz, ctx->d_pw};
        for (int k = 0; k < 4; ++k)
            PDFXC_CUDA(cudaMemcpyAsync(c[k].data(), src[k], sizeof(double) * nslot, cudaMemcpyDeviceToHost, ctx->stream));
        PDFXC_CUDA(cudaStreamSynchronize(ctx->stream));
        std::vector<double> xyzw(4 * (size_t)npts);
        std::vector<int> atom(ctx->h_owner.empty() ? 0 : (size_t)npts);
        for (size_t slot = 0; slot < nslot; ++slot) {
            const int64_t i = ctx->h_src[slot];
            if (i < 0) continue;
            for (int k = 0; k < 4; ++k) xyzw[4 * i + k] = c[k][slot];
            if (!atom.empty()) atom[i] = ctx->h_owner[slot];
        }
        std::vector<GridSegment> segs;
        for (size_t k = 0; k < ctx->seg_pts.size(); ++k)
            segs.push_back(GridSegment{ctx->seg_pts[k].first, ctx->seg_pts[k].second, ctx->seg_sh[k].first,
                                       ctx->seg_sh[k].second});
        const std::vector<int> mol = ctx->mol;
        const double* P = d_PA ? d_PA : ctx->d_P;
        auto reblock = [&](int g, int stg) {
            ctx->opt.group_blocks = g, ctx->opt.vxc_stages = stg;
            build_grid(ctx, npts, xyzw.data(), atom.empty() ? nullptr : atom.data(), segs);
            if (mol.size() > 1) {  // a batch: its per-molecule sums
                ctx->mol = mol;
                dev_alloc(&ctx->d_mol_sums, 2 * (mol.size() - 1));
            }
        };
        // candidates: INT8 groups of 1, 2 or 4 blocks x 2 or 3 Vxc stages; the FP64 path has no shape to choose
        std::vector<TuneChoice> cand;
        if (int8)
            for (int g : {4, 2, 1})
                for (int stg : {3, 2}) cand.push_back({g, stg});
        else
            cand.push_back({1, 3});
        std::vector<float> ms(cand.size(), 0.f);
        const bool profiling = ctx->profiling;
        ctx->profiling = false;
        for (size_t k = 0; k < cand.size(); ++k) {
            if (int8) reblock(cand[k].group_blocks, cand[k].vxc_stages);
            float best = 1e30f;
            for (int rep = 0; rep < 3; ++rep) {  // a warm-up (graph capture), then the better of two
                run_build(ctx, functional, P, false);
                PDFXC_CUDA(cudaStreamSynchronize(ctx->stream));
                collect_profile(ctx);
                if (int code = device_error(ctx)) {
                    ctx->profiling = profiling;
                    ctx->err = "pdfxc_autotune: a bounded device wait expired (code " + std::to_string(code) + ")";
                    return PDFXC_ERR_TIMEOUT;
                }
                if (rep > 0) best = std::min(best, ctx->last_profile.total_ms);
            }
            ms[k] = best;
        }
        ctx->profiling = profiling;
        const size_t win = (size_t)(std::min_element(ms.begin(), ms.end()) - ms.begin());
        if (int8) {
            if (win != cand.size() - 1) reblock(cand[win].group_blocks, cand[win].vxc_stages);
            std::lock_guard<std::mutex> lock(g_tune_mutex);
            g_tune_cache[tune_class(ctx, npts, segs.size())] = cand[win];
        }
        const int n = (int)std::min<size_t>(cand.size(), max_out > 0 ? (size_t)max_out : 0);
        for (int k = 0; out && k < n; ++k) {
            const size_t j = k == 0 ? win : (k <= (int)win ? k - 1 : k);  // the winner first
            out[k] = pdfxc_tuning{cand[j].group_blocks, cand[j].vxc_stages, ctx->opt.block_points, ms[j]};
        }
        if (n_out) *n_out = n;
        return PDFXC_OK;
    });
}

pdfxc_status pdfxc_get_tuning(pdfxc_ctx* ctx, pdfxc_tuning* out) {
    if (!ctx || !out) return PDFXC_ERR_ARG;
    const bool int8 = ctx->opt.precision == PDFXC_PRECISION_MIXED && ctx->opt.split_terms == 10;
    *out = pdfxc_tuning{int8 ? ctx->tuned_group : 1, int8 ? ctx->tuned_stages : 0, ctx->opt.block_points,
                        ctx->last_profile.total_ms};
    return PDFXC_OK;
}

pdfxc_status pdfxc_selftest_wait(pdfxc_ctx* ctx, double limit_seconds) {
    return guarded(ctx, [&]() -> pdfxc_status {
        if (!(limit_seconds > 0.0) || limit_seconds > 10.0) {
            ctx->err = "pdfxc_selftest_wait: the limit must lie in (0, 10] seconds";
            return PDFXC_ERR_ARG;
        }
        PDFXC_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
        pdfxc::launch_wait_selftest(ctx->d_err, (uint64_t)(limit_seconds * 1e9), ctx->stream);
        PDFXC_LAUNCHED("k_wait_selftest");
        PDFXC_CUDA(cudaStreamSynchronize(ctx->stream));
        const int code = device_error(ctx);
        PDFXC_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), ctx->stream));
        PDFXC_CUDA(cudaStreamSynchronize(ctx->stream));
        if (code) {
            ctx->err = "a bounded device wait expired (self test, code " + std::to_string(code) + ")";
            return PDFXC_ERR_TIMEOUT;
        }
        return PDFXC_OK;
    });
}

const char* pdfxc_last_error(const pdfxc_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void pdfxc_destroy(pdfxc_ctx* ctx) {
    if (!ctx) return;
    if (ctx->dens) pdfxc_destroy(ctx->dens);
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    free_grid(ctx);
    dev_free(ctx->d_atom_xyz), dev_free(ctx->d_p_exp), dev_free(ctx->d_p_coef);
    dev_free(ctx->d_nbr_idx), dev_free(ctx->d_nbr_dist), dev_free(ctx->d_ghost);
    dev_free(ctx->d_sh_atom), dev_free(ctx->d_sh_l), dev_free(ctx->d_sh_nprim), dev_free(ctx->d_sh_p0), dev_free(ctx->d_sh_ao0);
    dev_free(ctx->d_P), dev_free(ctx->d_V), dev_free(ctx->d_Vacc), dev_free(ctx->d_scalars), dev_free(ctx->d_err);
    dev_free(ctx->d_p_rowexp); dev_free(ctx->d_Vprev); dev_free(ctx->d_p_words); dev_free(ctx->d_row_cols);
    dev_free(ctx->d_P_b), dev_free(ctx->d_V_b), dev_free(ctx->d_Vacc_b), dev_free(ctx->d_scalars_b);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : ctx->stage_ev) cudaEventDestroy(e);
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

}  // extern "C"
