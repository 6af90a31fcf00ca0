// Internal structures of libpdfxc: the device-resident system, the blocked
// grid, and the launch interfaces of the kernels.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/pdfxc.h"

namespace pdfxc {

constexpr int BLOCK_PTS = 128;  // grid points per block (padded with zero weight)

// One spatial block of grid points and its screened basis.
// Points live at [blk * BLOCK_PTS, (blk + 1) * BLOCK_PTS) of the SoA point arrays.
struct BlockMeta {
    int sh0;       // first entry in blk_shells / blk_shell_row
    int nsh;       // screened shells
    int ao0;       // first entry in blk_aos
    int nb;        // screened AOs
    int nbp;       // nb rounded up to the contraction tile
    int npts;      // real points in the block (<= BLOCK_PTS)
    int lead;      // first block of this block's group (the block itself when ungrouped)
    int gn;        // blocks in the group; a group's blocks are consecutive and share one screened basis
    int64_t ws;    // byte offset of this block's intermediates inside its chunk's workspace
};

// A contiguous range of blocks whose intermediates fit the workspace together.
struct Chunk {
    int b0, b1;
    int max_nbp;
    size_t ws_bytes;
};

// Device views of the basis (shell-major structure of arrays).
struct BasisView {
    const double* atom_xyz;
    const int* sh_atom;
    const int* sh_l;
    const int* sh_nprim;
    const int* sh_p0;
    const int* sh_ao0;
    const double* p_exp;
    const double* p_coef;
};

// Device views of the blocked grid.
struct GridView {
    const double* px;  // [nblk * BLOCK_PTS]
    const double* py;
    const double* pz;
    const double* pw;
    const BlockMeta* meta;
    const int* blk_shells;     // shell id
    const int* blk_shell_row;  // local AO row of the shell's first component
    const int* blk_aos;        // global AO index of each local row
    const int* blk_row_info;   // per local row: 16 * (shell slot in the block's list) + L^2 + component
    const struct RowGeom* blk_row_geom;  // per local row: its shell's atom and blk_row_info (INT8 path)
    // The FP64 contractions' tiles, so that a launch has no idle CTAs: {block, 64-row M tile} for
    // X = P_sub phi, {block, M << 16 | N} (64 x 64 tiles) for Vacc += phi Z^T, block by block; and
    // each block's first tile (prefix sums, host memory: read by the launchers, not the kernels).
    // Null (the no-allocation build): the launch covers max_nbp tiles per block, surplus CTAs exit.
    const int2* xtiles;
    const int2* vtiles;
    const int64_t* h_xtile0;
    const int64_t* h_vtile0;
};

// One AO row of a block's screened basis: the atom of its shell and its blk_row_info entry.
struct __align__(16) RowGeom {
    double ax, ay, az;
    int info;
    int pad;
};

// One radial shell of an atom-centred grid: n points from the unit grid rows [u0, u0 + n),
// abscissa r and radial weight wr, written to points [p0, p0 + n).
struct GridShell {
    int atom, n;
    int64_t u0, p0;
    double r, wr;
};

// A workspace layout for a build with its own number of [nbp][BLOCK_PTS] FP64 planes per
// block (the XC gradient, the open-shell build): per-block offsets, chunks, workspace.
struct Plan {
    BlockMeta* d_meta = nullptr;
    std::vector<Chunk> chunks;
    void* d_ws = nullptr;
    size_t ws_bytes = 0;
    int planes = -1;
};

}  // namespace pdfxc

struct pdfxc_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    pdfxc_options opt{};
    std::string err;

    // system
    int natom = 0, nshell = 0, nao = 0;
    std::vector<double> h_atom_xyz;
    std::vector<int> h_atom_z, h_sh_atom, h_sh_l, h_sh_nprim, h_sh_p0, h_sh_ao0;
    std::vector<double> h_p_exp, h_p_coef;
    double *d_atom_xyz = nullptr, *d_p_exp = nullptr, *d_p_coef = nullptr;
    int *d_sh_atom = nullptr, *d_sh_l = nullptr, *d_sh_nprim = nullptr, *d_sh_p0 = nullptr,
        *d_sh_ao0 = nullptr;

    // blocked grid
    int64_t npts = 0;
    int nblk = 0;
    std::vector<pdfxc::BlockMeta> h_meta;
    std::vector<pdfxc::Chunk> chunks;
    std::vector<int64_t> h_src;  // original index of each padded point slot (-1 = padding)
    double *d_px = nullptr, *d_py = nullptr, *d_pz = nullptr, *d_pw = nullptr;
    pdfxc::BlockMeta* d_meta = nullptr;
    int *d_blk_shells = nullptr, *d_blk_shell_row = nullptr, *d_blk_aos = nullptr, *d_blk_row_info = nullptr;
    pdfxc::RowGeom* d_blk_row_geom = nullptr;
    double contraction_flops = 0.0;
    double mean_nb = 0.0;
    int blk_lo = 0, blk_hi = 0;  // the blocks this context builds (pdfxc_set_block_range; default all)
    std::vector<int> seg_blk;    // blocks of grid segment i (a molecule of a batch): [seg_blk[i], seg_blk[i+1])
    int* d_seg_blk = nullptr;
    std::vector<int> h_grp;      // first block of every group, ascending (groups: consecutive blocks, one basis)
    int* d_grp = nullptr;
    // INT8 path: per chunk the contraction work items (rho, then Vxc) sorted by decreasing cost,
    // their offsets in d_items, and two work counters per chunk
    std::vector<int> items_off_rho, items_n_rho, items_off_vxc, items_n_vxc;
    int2* d_items = nullptr;
    int* d_counters = nullptr;
    // batch of molecules (pdfxc_set_batch): AO offset and count of each molecule in the joint system
    std::vector<int> mol;        // AO offsets, size nmol + 1 (empty: a single molecule)
    double* d_mol_sums = nullptr;  // [2 * nmol]: Exc, electron count per molecule

    // per-build buffers
    void* d_ws = nullptr;
    size_t ws_bytes = 0;
    double* d_rho = nullptr;    // [nblk * BLOCK_PTS * 4]: rho, grad x, y, z
    double* d_coef = nullptr;   // [nblk * BLOCK_PTS * 4]: 0.5 w vrho, c_x, c_y, c_z
    double* d_blk_sum = nullptr;  // [nblk * 2]: per-block Exc, Nel
    double* d_rho_acc = nullptr;  // mixed path: [nblk * BLOCK_PTS * 4] rho partial sums of the contraction
    int* d_err = nullptr;         // device error word (bounded waits that expired)
    double* d_scalars = nullptr;  // [2]
    double* d_P = nullptr;        // n_ao^2 staging for host-pointer builds
    double* d_V = nullptr;        // n_ao^2
    double* d_Vprev = nullptr;    // n_ao^2: Vxc of the last delta build (pdfxc_build_vxc_delta_device)
    int vprev_iter = 0;           // its SCF iteration, 0 = none
    double* d_Vacc = nullptr;     // n_ao^2 non-symmetric accumulator
    int* d_p_rowexp = nullptr;    // n_ao: exponents of the rows of P (INT8 path)
    uint32_t* d_p_words = nullptr;  // n_ao^2: the four digits of each element of P (INT8 path)
    int* d_row_cols = nullptr;      // batch: per AO row its molecule's columns [c0, c1) (2 ints)
    bool rho_valid = false;
    pdfxc_ctx* dens = nullptr;  // pdfxc_density: FP64 context over the requested points (same system)
    double* h_stage = nullptr;  // pinned host staging of Vxc for the host-array builds (2 x stage_elems)
    size_t stage_elems = 0;
    int* d_ghost = nullptr;       // [natom] dummy atoms (atomic number <= 0 given to set_system), or null
    int* d_nbr_idx = nullptr;     // Stratmann-Scuseria weights: per atom the other atoms by distance
    double* d_nbr_dist = nullptr;
    int rho_gga = 0;

    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // stage events: per chunk 5 (before ao, gemm_x, rho, gemm_v, after gemm_v), then finish end
    std::vector<cudaEvent_t> stage_ev;
    pdfxc_profile last_profile{};

    // one captured CUDA graph per build configuration (functional, incremental, density pointer)
    bool use_graph = true;
    bool profiling = false;    // launch stage by stage so that stage events can be timed
    bool last_staged = false;  // the last build ran stage by stage
    cudaGraphExec_t graph_exec = nullptr;
    int graph_fn = -1, graph_inc = -1;
    const double* graph_P = nullptr;

    // XC nuclear gradient (pdfxc_xc_gradient); freed with the grid
    std::vector<int> h_owner;              // owner atom per point slot (empty: set_grid had no atoms)
    int* d_owner = nullptr;
    int* d_ao_atom = nullptr;              // [n_ao]
    pdfxc::Plan gplan;                     // gradient workspace layout
    double* d_grad = nullptr;   // [2 * natom * 3]: AO-centre term, grid-weight term
    double* d_fdens = nullptr;  // [nblk * BLOCK_PTS] energy density per slot
    double* d_wslot = nullptr;  // [nblk * BLOCK_PTS] single-centre weight per slot
    double* d_brad = nullptr;   // [natom]
    double* d_pair = nullptr;   // [2 * natom^2] Becke pair constants
    double* d_wscratch = nullptr;  // weight-term atom rows in device memory (above 400 atoms)
    int2 *d_xtiles = nullptr, *d_vtiles = nullptr;  // GridView::xtiles, vtiles
    std::vector<int64_t> h_xtile0, h_vtile0;         // GridView::h_xtile0, h_vtile0 (nblk + 1 each)

    // open-shell build (pdfxc_build_vxc_uks): beta-spin buffers beside the alpha ones above
    pdfxc::Plan uplan;
    double* d_rho_b = nullptr;      // [nblk * BLOCK_PTS * 4]
    double* d_blk_sum_b = nullptr;  // [nblk * 2]: N_beta, 0
    double* d_scalars_b = nullptr;  // [2]
    double *d_P_b = nullptr, *d_V_b = nullptr, *d_Vacc_b = nullptr;  // n_ao^2 each
    // INT8 path: the beta spin's digit words of P (n_ao^2) and row exponents, rho accumulators and
    // Vxc coefficients (nblk * BLOCK_PTS * 4 each), and work counters (two per chunk)
    uint32_t* d_p_words_b = nullptr;
    int* d_p_rowexp_b = nullptr;
    double *d_rho_acc_b = nullptr, *d_coef_b = nullptr;
    int* d_counters_b = nullptr;
    int rho_spin = 0;               // the stored densities: 1 closed shell, 2 open shell

    // the grid as given (for re-blocking: pdfxc_autotune): its segments (one per molecule of a batch)
    std::vector<std::pair<int64_t, int64_t>> seg_pts;  // points [p0, p1) of each segment
    std::vector<std::pair<int, int>> seg_sh;           // shells [sh0, sh1) of each segment
    int tuned_group = 0, tuned_stages = 0;             // the choices in use (0: not tuned)
    alignas(64) CUtensorMap phi_map{};                 // see MixedArgs::phi_map
    bool phi_map_ok = false;
};

namespace pdfxc {

// gridgen.cu: the points and single-centre weights of the shells
void launch_grid_points(const GridShell* shells, int nshell, const double* unit, const double* O,
                        const double* atom_xyz, double* xyz, double* w, int* owner, cudaStream_t s);

// kernels_fp64.cu
void launch_ao_eval(const BasisView& b, const GridView& g, int blk0, int nblk, bool gga,
                    char* ws, int max_nsh, cudaStream_t s);
void launch_gemm_x(const GridView& g, const double* P, int nao, int blk0, int nblk, int max_nbp,
                   int nplanes, char* ws, cudaStream_t s);
// the same contraction over nz planes: plane dst0 + z = P_sub * plane src0 + z
void launch_gemm_x_planes(const GridView& g, const double* P, int nao, int blk0, int nblk, int max_nbp, int src0,
                          int dst0, int nz, char* ws, cudaStream_t s);
// the GGA closed-shell build from radial sums (layout block_ws_doubles_rad)
void launch_ao_eval_rad(const BasisView& b, const GridView& g, int blk0, int nblk, char* ws, cudaStream_t s);
void launch_rho_functional_rad(const BasisView& b, const GridView& g, int blk0, int nblk, int fn, bool incremental,
                               double rho_cut, char* ws, double* rho, double* coef, double* blk_sum, cudaStream_t s);
void launch_rho_rad(const BasisView& b, const GridView& g, int blk0, int nblk, const char* ws, double* rho_acc,
                    cudaStream_t s);
void launch_z_rad(const BasisView& b, const GridView& g, int blk0, int nblk, const double* coef, char* ws,
                  cudaStream_t s);
// per point: rho = rho_acc (+ stored, incremental), grad rho = 2 rho_acc[1..3] (+ stored), the
// functional, the Vxc coefficients and the block sums (kernels_mixed.cu)
void launch_functional_points(const GridView& g, int blk0, int nblk, int fn, bool incremental, double rho_cut,
                              const double* rho_acc, double* rho_store, double* coef, double* blk_sum,
                              cudaStream_t s);
void launch_rho_functional(const GridView& g, int blk0, int nblk, int fn, bool incremental,
                           double rho_cut, char* ws, double* rho, double* coef, double* blk_sum,
                           cudaStream_t s);
void launch_gemm_v(const GridView& g, int blk0, int nblk, int max_nbp, bool gga, const double* coef,
                   char* ws, double* Vacc, int nao, cudaStream_t s);
void launch_fock_delta(const double* V, double* Vprev, double* dV, size_t n, bool has_prev, cudaStream_t s);
void launch_finish(const double* Vacc, double* V, int nao, const double* blk_sum, int nblk,
                   double* scalars, cudaStream_t s);
// the upper triangle (j >= i) of a symmetric n x n matrix packed row by row, and back (both triangles)
void launch_pack_upper(const double* V, int n, double* packed, cudaStream_t s);
void launch_unpack_upper(const double* packed, int n, double* V, cudaStream_t s);
// Vacc += phi Z^T with Z in plane zplane of each block's workspace
void launch_gemm_v_plane(const GridView& g, int blk0, int nblk, int max_nbp, int zplane, char* ws, double* Vacc,
                         int nao, cudaStream_t s);
// open shell: rho/grad rho of X_A, X_B (the two planes after phi), the functional, Z_A/Z_B over X_A/X_B;
// blk_sum = (Exc, N_alpha) pairs, blk_sum_b = (N_beta, 0) pairs
void launch_rho_functional_uks(const GridView& g, int blk0, int nblk, int fn, bool incremental, double rho_cut,
                               char* ws, double* rho_a, double* rho_b, double* blk_sum, double* blk_sum_b,
                               cudaStream_t s);
void launch_block_sums(const double* blk_sum, int nblk, double* scalars, cudaStream_t s);
// per grid segment: out[2 i], out[2 i + 1] = sums over blocks [seg_blk[i], seg_blk[i+1])
void launch_segment_sums(const double* blk_sum, const int* seg_blk, int nseg, double* out, cudaStream_t s);

// gradient.cu: XC nuclear gradient (FP64)
int grad_workspace_planes(bool gga);  // [nbp][BLOCK_PTS] double planes per block
void launch_ao_grad(const BasisView& b, const GridView& g, int blk0, int nblk, bool gga, char* ws, cudaStream_t s);
void launch_grad_x(const GridView& g, const double* P, int nao, int blk0, int nblk, int max_nbp, bool gga, char* ws,
                   cudaStream_t s);
// seed: the cotangent of Exc that scales every derivative; want_z: the density adjoint
// Z = 0.5 a phi + c . grad phi replaces X (plane grad_z_plane) for the dExc/dP contraction
void launch_grad_point(const GridView& g, const int* ao_atom, const int* owner, int blk0, int nblk, int fn,
                       double rho_cut, char* ws, double seed, bool want_z, double* fdens, double* blk_sum,
                       double* grad, cudaStream_t s);
int grad_z_plane(bool gga);
// the weight term keeps each point's atom rows in shared memory up to grad_weight_max_atoms()
// atoms; above that (or when scratch is given) in grad_weight_scratch_doubles(natom) of device memory
int grad_weight_max_atoms();
size_t grad_weight_scratch_doubles(int natom);
void launch_grad_weight(const double* atom_xyz, int natom, const double* inv, const double* adj, int64_t nslots,
                        const double* px, const double* py, const double* pz, const int* owner, const double* wsingle,
                        const double* fdens, double* grad, double* scratch, cudaStream_t s);

// becke.cu
// Stratmann-Scuseria weights (n_atom <= 6000: atoms in shared memory); inv/adj: n_atom^2 scratch each
// nbr_idx / nbr_dist: per atom the other atoms in ascending distance, natom x (natom - 1)
void launch_ss(const double* atom_xyz, int natom, double* inv, double* adj, const int* nbr_idx,
               const double* nbr_dist, int64_t npts, const double* xyz, const int* owner, const double* w_single,
               double* w_out, cudaStream_t s);
void launch_becke_pairs(const double* atom_xyz, const double* brad, int natom, int size_adjust, double* inv,
                        double* adj, cudaStream_t s);
// ghost (n_atom ints, may be null): partner atoms left out of every product (atomic number <= 0)
void launch_becke(const double* atom_xyz, const double* brad, const int* ghost, int natom, int size_adjust,
                  int64_t npts, const double* xyz, const int* owner, const double* w_single,
                  double* w_out, cudaStream_t s);
size_t becke_max_atoms();
// the table form, one point per thread (pair constants in inv/adj, n_atom^2 doubles each), for
// n_atom <= becke_small_atoms()
void launch_becke_tab(const double* atom_xyz, const double* brad, const int* ghost, int natom, int size_adjust,
                      double* inv, double* adj, int64_t npts, const double* xyz, const int* owner,
                      const double* w_single, double* w_out, cudaStream_t s);
size_t becke_small_atoms();
// the same weights with a warp per point (lanes over the atoms); tab: 4 n_atom^2 doubles
void launch_becke_warp(const double* atom_xyz, const double* brad, const int* ghost, int natom, int size_adjust,
                       double* tab, int64_t npts, const double* xyz, const int* owner, const double* w_single,
                       double* w_out, cudaStream_t s);
size_t becke_warp_max_atoms();

// Intermediates of one block inside its chunk workspace (doubles):
//   phi   [nbp][BLOCK_PTS]           AO values, row = local AO
//   dphi  [3][nbp][BLOCK_PTS]        gradients (GGA only)
//   X     [nbp][BLOCK_PTS]           P_sub * phi
__host__ __device__ inline size_t block_ws_doubles(int nbp, bool gga) {
    return (size_t)nbp * BLOCK_PTS * (gga ? 5 : 2);
}

// The closed-shell FP64 build: phi and X (then Z) planes, then the shells' radial sums S0, S1
// (the GGA form; the LDA form uses the two planes only).
__host__ __device__ inline size_t block_ws_doubles_rad(int nbp, int nsh) {
    return (size_t)BLOCK_PTS * (2 * (size_t)nbp + 2 * (size_t)nsh);
}

// Intermediates of one block on the mixed path (byte offsets; nbp % 128 == 0).
// Packed operands use the layout of umma.cuh, three split planes each.
struct MixedLayout {
    size_t phi32;                // FP32 phi and grad phi, [4][nbp][128]
    size_t phi1, phi1_plane;     // phi^T packed: rows = 128 points, K = nbp AOs
    size_t phi2, phi2_plane;     // phi packed: rows = nbp AOs, K = 128 points
    size_t ppack, ppack_plane;   // P_sub packed: rows = nbp, K = nbp
    size_t zpack, zpack_plane;   // Z packed: rows = nbp, K = 128 points
    size_t total;
};

__host__ __device__ inline MixedLayout mixed_layout(int nbp) {
    MixedLayout L;
    size_t o = 0;
    L.phi32 = o;
    o += (size_t)4 * nbp * BLOCK_PTS * 4;
    L.phi1 = o;
    L.phi1_plane = (size_t)BLOCK_PTS * nbp * 2;
    o += 3 * L.phi1_plane;
    L.phi2 = o;
    L.phi2_plane = (size_t)nbp * BLOCK_PTS * 2;
    o += 3 * L.phi2_plane;
    L.ppack = o;
    L.ppack_plane = (size_t)nbp * nbp * 2;
    o += 3 * L.ppack_plane;
    L.zpack = o;
    L.zpack_plane = (size_t)nbp * BLOCK_PTS * 2;
    o += 3 * L.zpack_plane;
    L.total = o;
    return L;
}

// Intermediates of one block on the fixed-point (INT8 slice) path. Operands are
// cut into OZ_SLICES signed digits in [-128, 127] with a power-of-two scale per row:
// v = 2^e (s_1 + s_2/256 + s_3/256^2 + s_4/256^3)/127; digit planes
// are packed K-major in 64-byte slabs. AO values are not stored: the block keeps each
// shell's radial sums S0, S1 at its points ([2][nsh][128] FP64) and every consumer forms
// phi = A S0, grad phi = grad A S0 - 2 r A S1 from them. One set of phi digits serves both
// contractions: phi^T with a scale per point (e_pt), K-major for rho and read as an MN-major
// operand by the Vxc contraction, whose other operand is Z' = 2^e_pt Z with a scale per AO row
// over the group's points (e_z_g, written by the group's first block). P_sub is shared by the
// group and lives only in the first block's region, after `total` (`total_lead` bytes in all).
constexpr int OZ_SLICES = 4;
// Largest K (screened AOs of a group, padded to 128) of the INT8 rho contraction: its order-5
// int32 accumulator sums four digit products of at most 128^2 per K index (exact in int32 while
// 4 * 128^2 * K < 2^31, K < 32768), and the FP64 combination of the orders,
// n = ((D2 256 + D3) 256 + D4) 256 + D5 with |D_k| <= (k - 1) 128^2 K, stays below 2^53 while
// K < 32515.
constexpr int OZ_MAX_K = 32512;
struct OzLayout {
    size_t rad;                 // radial sums: S0 [nsh][128], then S1 [nsh][128]
    size_t phi1, phi1_plane;    // phi^T digits: rows = 128 points, K = nbp AOs
    size_t zpack, zpack_plane;  // Z' digits: rows = nbp AOs (128-row tiles), K = 128 points
    size_t e_pt, e_z_g, e_p;    // int exponents: per point, per AO row of the group (Z'), P_sub
    size_t total;
    size_t ppack, ppack_plane;  // P_sub digits of the group: rows = nbp, K = nbp (first block only)
    size_t total_lead;
};

__host__ __device__ inline OzLayout oz_layout(int nbp, int nsh) {
    auto a256 = [](size_t x) { return (x + 255) & ~size_t(255); };
    OzLayout L;
    size_t o = 0;
    L.rad = o;
    o = a256(o + (size_t)2 * nsh * BLOCK_PTS * 8);
    L.phi1 = o;
    L.phi1_plane = (size_t)BLOCK_PTS * nbp;
    o = a256(o + OZ_SLICES * L.phi1_plane);
    L.zpack = o;
    L.zpack_plane = (size_t)nbp * BLOCK_PTS;
    o = a256(o + OZ_SLICES * L.zpack_plane);
    L.e_pt = o;
    o = a256(o + sizeof(int) * BLOCK_PTS);
    size_t* e[2] = {&L.e_z_g, &L.e_p};
    for (size_t* f : e) {
        *f = o;
        o = a256(o + sizeof(int) * nbp);
    }
    L.total = o;
    L.ppack = o;
    L.ppack_plane = (size_t)nbp * nbp;
    o = a256(o + OZ_SLICES * L.ppack_plane);
    L.total_lead = o;
    return L;
}

// kernels_mixed.cu: the four stages of one chunk on the mixed path
struct MixedArgs {
    BasisView b;
    GridView g;
    int blk0, nblk, max_nbp, fn, incremental, nterms, nao;
    double rho_cut;
    const double* P;
    char* ws;
    double *rho_acc, *rho_store, *coef, *blk_sum, *Vacc;
    int* err;
    const int* grp;  // first blocks of the chunk's groups (INT8 path)
    int ngrp;
    const int* p_rowexp;      // exponents of the rows of P (INT8 path)
    const uint32_t* p_words;  // the four digits of each element of P (INT8 path)
    // INT8 path: the chunk's contraction work items, by decreasing cost (see kernels_mixed.cu),
    // and the two work counters of the chunk's contraction launches (zero before the build)
    const int2* items_rho;
    int n_rho;
    const int2* items_vxc;
    int n_vxc;
    int* counters;
    int vxc_stages;  // operand stages of the Vxc contraction (2 or 3)
    // INT8 path: a tensor map over the chunk workspace that moves the Vxc contraction's phi operand
    // of one stage (16 pieces of 1 KiB) in one copy; null: 16 bulk copies
    const CUtensorMap* phi_map;
};
// The tensor map of MixedArgs::phi_map over a workspace of ws_bytes bytes (false: the driver has
// no tensor-map encoder or refused the map; the contraction then copies piece by piece).
bool make_phi_map(const void* ws, size_t ws_bytes, CUtensorMap* map);
void mixed_prepare(const MixedArgs& a, cudaStream_t s);     // AO values, P_sub packing
void mixed_rho(const MixedArgs& a, cudaStream_t s);         // X^T = phi^T P_sub + rho epilogue
void mixed_functional(const MixedArgs& a, cudaStream_t s);  // functional, Z packing
void mixed_vxc(const MixedArgs& a, cudaStream_t s);         // Vacc += phi Z^T
size_t umma_smem_bytes(int nterms);
// a bounded wait on an mbarrier nothing completes; records code 8 in *err after limit_ns
void launch_wait_selftest(int* err, uint64_t limit_ns, cudaStream_t s);
// the same four stages with INT8 fixed-point slices (split_terms == 10)
// once per build; row_cols (batch, may be null): each row's molecule's columns, the only ones read
void oz_p_digits(const double* P, int nao, const int* row_cols, int* e, uint32_t* words, cudaStream_t s);
void oz_prepare(const MixedArgs& a, cudaStream_t s);
void oz_rho(const MixedArgs& a, cudaStream_t s);
void oz_functional(const MixedArgs& a, cudaStream_t s);
void oz_vxc(const MixedArgs& a, cudaStream_t s);
// the open shell on the INT8 path: P_sub's digits alone (the phi digits stay), the open-shell
// functional from both spins' rho accumulators (coefficients of each spin, block sums E and
// N_alpha into a.blk_sum, N_beta and 0 into blk_sum_b), and the Z' digits of one spin
void oz_pack_p(const MixedArgs& a, cudaStream_t s);
void oz_functional_uks(const MixedArgs& a, const double* rho_acc_b, double* rho_store_b, double* coef_b,
                       double* blk_sum_b, cudaStream_t s);
void oz_pack_z(const MixedArgs& a, cudaStream_t s);

}  // namespace pdfxc
