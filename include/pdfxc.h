/*
 * pdfxc.h -- C ABI of the B200 grid exchange-correlation quadrature.
 *
 * This is the boundary that replaces ProteinDF's DfCalcGridX engine
 * (src/libpdf/DfCalcGridX.{h,cpp}). A host-side DfCalcGridX-compatible class
 * (or any FFI) calls these entry points; they take plain pointers and sizes,
 * never throw, and return a pdfxc_status (0 = success). One context drives
 * one GPU; calls on a context are synchronous and not re-entrant.
 *
 * Units: coordinates in bohr, energies in hartree. Matrices are dense,
 * row-major, n_ao x n_ao FP64. The closed-shell convention of the reference
 * applies: the caller passes the alpha density P_A = P/2
 * (src/libpdf/DfXCFunctional.cpp:133-139) and receives the alpha Kohn-Sham
 * matrix, accumulated into (F += Vxc) as DfCalcGridX does
 * (src/libpdf/DfCalcGridX.cpp:2351-2500).
 */
#ifndef PDFXC_H
#define PDFXC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int pdfxc_status;

enum {
    PDFXC_OK = 0,
    PDFXC_ERR_ARG = 1,      /* bad argument (null pointer, size out of range) */
    PDFXC_ERR_CUDA = 2,     /* a CUDA runtime call failed; see pdfxc_last_error */
    PDFXC_ERR_STATE = 3,    /* call out of order (e.g. build before set_grid) */
    PDFXC_ERR_TIMEOUT = 4,  /* a bounded device wait expired */
    PDFXC_ERR_NOMEM = 5,    /* device allocation failed */
    PDFXC_ERR_UNSUPPORTED = 6
};

/* Functional identifiers; names as the reference's xc-potential keyword
 * (src/libpdf/DfXCFunctional.cpp:70-104). */
enum {
    PDFXC_SVWN = 0,  /* Slater + VWN5 (LDA) */
    PDFXC_HFS = 1,   /* Slater (LDA) */
    PDFXC_HFB = 2,   /* Becke 88 (GGA) */
    PDFXC_BLYP = 3,  /* Becke 88 + LYP (GGA) */
    PDFXC_B3LYP = 4, /* 0.80 Slater + 0.72 B88 + 0.19 VWN3 + 0.81 LYP (GGA) */
    PDFXC_PBE = 5    /* PBE exchange + PBE correlation (GGA); not in the reference, written from the
                        published papers (Perdew, Burke, Ernzerhof 1996; Perdew, Wang 1992) */
};

enum {
    PDFXC_PRECISION_FP64 = 0,  /* the drop-in: every product in FP64 */
    PDFXC_PRECISION_MIXED = 1  /* the two contractions on tensor cores with split operands (INT8 digits by
                                  default, see split_terms), FP64 AO values, functional and sums */
};

typedef struct {
    int precision;       /* PDFXC_PRECISION_* */
    int block_points;    /* grid points per block, 1..128 (default 128) */
    double ao_cutoff;    /* drop a shell from a block when its value/gradient bound is below (default 1e-14) */
    double rho_cutoff;   /* xc-density-threshold: points with rho_A <= it are skipped (default 1e-16) */
    size_t workspace_bytes; /* device workspace budget for block intermediates (0 = default 4 GiB) */
    int split_terms;     /* mixed path operand split: 10 (default) = four balanced base-256 INT8 digits
                            per operand (about 31 bits), the 10 digit products of order i + j <= 5 on
                            the integer tensor cores; 3 or 6 = BF16 hi/mid(/lo) split with FP32
                            accumulation (about 1e-6 relative, for comparison only) */
    int group_blocks;    /* INT8 path: consecutive blocks per group sharing one screened basis, 1..4;
                            0 (default) = the tuned choice for the workload class if pdfxc_autotune has
                            made one in this process, else 4 */
    int vxc_stages;      /* INT8 path: operand stages of the Vxc contraction, 2 or 3; 0 (default) =
                            the tuned choice, else 3 */
} pdfxc_options;

typedef struct pdfxc_ctx pdfxc_ctx;

/* Fill *opt with the defaults. */
void pdfxc_default_options(pdfxc_options* opt);

/* Create a context on CUDA device `device`. Replaces the DfCalcGridX
 * constructor (src/libpdf/DfCalcGridX.cpp:47-74). */
pdfxc_status pdfxc_create(pdfxc_ctx** out, int device, const pdfxc_options* opt);

/* Molecule and basis (TlOrbitalInfo, src/libpdf/TlOrbitalInfoObject.cpp:38-256).
 * Shells in AO order; shell s has angular momentum shell_l[s] in {0,1,2}
 * (components s; px,py,pz; dxy,dxz,dyz,d(x2-y2),dz2), shell_nprim[s]
 * primitives whose exponents/normalised coefficients follow consecutively in
 * prim_exp/prim_coef. */
pdfxc_status pdfxc_set_system(pdfxc_ctx* ctx, int natom, const double* atom_xyz,
                              const int* atom_z, int nshell, const int* shell_atom,
                              const int* shell_l, const int* shell_nprim,
                              const double* prim_exp, const double* prim_coef);

/* The quadrature grid: npts rows of (x, y, z, w) with w the final
 * (partitioned) weight, and the owning atom of each point -- the grid matrix
 * columns GM_X..GM_ATOM_INDEX of src/libpdf/DfCalcGridX.h:35-54. Points are
 * regrouped into spatial blocks and the per-block shell lists are screened
 * here, once per geometry. */
pdfxc_status pdfxc_set_grid(pdfxc_ctx* ctx, int64_t npts, const double* xyzw, const int* atom);

/* Becke partition weights with atomic-size adjustment
 * (DfGenerateGrid::calcMultiCenterWeight_Becke, src/libpdf/DfGenerateGrid.cpp:1811-1876,
 * Ps_uij :2043-2086): w_out[i] = w_single[i] * P_owner(r_i) / sum_m P_m(r_i).
 * becke_radius[a] is the size-adjustment radius of atom a (0.35 for H,
 * Bragg-Slater otherwise, :1958-1968). Requires pdfxc_set_system. */
pdfxc_status pdfxc_becke_weights(pdfxc_ctx* ctx, int64_t npts, const double* xyz,
                                 const int* atom, const double* w_single,
                                 const double* becke_radius, int size_adjust, double* w_out);

/* Stratmann-Scuseria partition weights (DfGenerateGrid::calcMultiCenterWeight_SS,
 * src/libpdf/DfGenerateGrid.cpp:1878-1956; grid/partitioning_method = SSWeight):
 * w_out[i] = w_single[i] * P_owner(r_i) / sum_m P_m(r_i) with the SS cell function
 * (a = 0.64, no size adjustment). Exact zeros of the cell function end each atom's
 * product early, so large systems stay near O(N_atom) per point; at most 6000 atoms.
 * Requires pdfxc_set_system. */
pdfxc_status pdfxc_ss_weights(pdfxc_ctx* ctx, int64_t npts, const double* xyz, const int* atom,
                              const double* w_single, double* w_out);

/* Grid generation on the device (DfGenerateGrid::generateGrid_atom,
 * src/libpdf/DfGenerateGrid.cpp:934-1091): per atom and radial shell i = 1..nrad an
 * abscissa r_i and weight w_i (Gauss-Chebyshev of the second kind with a Becke, Treutler-
 * Ahlrichs or Knowles-Kaltenborn map, :1612-1655, or Euler-Maclaurin, :1597-1610) scaled
 * by the atom's radius; shells with r_i > 30 bohr are dropped (:1005-1007); the angular
 * order is nang, or pruned (Murray-Handy-Laming with K = 5, rounded down to a tabulated
 * order, :1658-1688; or the SG-1 regions by atomic number, :1690-1713 and :960-982); the
 * points are the unit grid of that order rotated by `orientation`, scaled by r_i about
 * the atom, with weights w_unit * w_i (getSphericalGrids, :1715-1734); then the
 * partition weights (Becke with optional size adjustment, or Stratmann-Scuseria) and the
 * weight screen |w| > weight_cutoff (screeningGridsByWeight0, :1979-2004). The result
 * becomes the context's grid, as after pdfxc_set_grid with owner atoms, in the
 * reference's point order (atom, shell, angular point); *npts receives its size. The
 * unit grids are input data (the caller's Lebedev tables). */
enum { PDFXC_RADIAL_GC = 0, PDFXC_RADIAL_EM = 1 };
enum { PDFXC_MAP_BECKE = 0, PDFXC_MAP_TA = 1, PDFXC_MAP_KK = 2 };
enum { PDFXC_PRUNE_NONE = 0, PDFXC_PRUNE_MHL = 1, PDFXC_PRUNE_SG1 = 2 };
enum { PDFXC_PARTITION_BECKE = 0, PDFXC_PARTITION_SS = 1 };
typedef struct {
    int nrad;                   /* radial shells per atom (before the 30 bohr cut) */
    int nang;                   /* angular order without pruning; the MHL cap */
    int radial;                 /* PDFXC_RADIAL_* */
    int mapping;                /* PDFXC_MAP_* (Gauss-Chebyshev only) */
    int pruning;                /* PDFXC_PRUNE_* */
    int partition;              /* PDFXC_PARTITION_* */
    int size_adjust;            /* Becke atomic-size adjustment (Becke partition only) */
    double weight_cutoff;       /* points with |w| <= weight_cutoff are dropped (the reference: 1e-16) */
    const double* atom_radius;  /* natom: radial scale and pruning radius (Bragg-Slater; the SG-1 radii for SG-1);
                                   0 = no grid on that atom (the reference skips dummy atoms) */
    const double* becke_radius; /* natom: size-adjustment radii (Becke partition only) */
    int n_orders;               /* unit-sphere grids: n_orders orders in ascending order, */
    const int* orders;          /* and their points, x y z w per row, order after order */
    const double* unit_grids;
    const double* orientation;  /* 3 x 3 row-major rotation of the unit grids; NULL = identity */
} pdfxc_grid_params;
pdfxc_status pdfxc_generate_grid(pdfxc_ctx* ctx, const pdfxc_grid_params* prm, int64_t* npts);

/* The context's grid in input order: xyzw (npts x 4, final weights) and, when the grid
 * has owner atoms, atom (npts; may be NULL) -- the grid matrix's first five columns. */
pdfxc_status pdfxc_get_grid(pdfxc_ctx* ctx, double* xyzw, int* atom);

/* One closed-shell XC build: rho pass + Vxc pass
 * (DfCalcGridX::calcXCIntegForFockAndEnergy, src/libpdf/DfCalcGridX.cpp:2280-2315).
 * PA: n_ao x n_ao alpha density (host). If incremental != 0 the density
 * rho/grad rho of PA is added to the stored per-point values of the previous
 * build (xc-update = yes, :1862-1889, PA is then the alpha density
 * difference); otherwise they are recomputed from PA. F (host, n_ao x n_ao)
 * is accumulated into: F += Vxc. exc receives the XC energy, nelec_alpha
 * sum_i w_i rho_A(r_i) (DfCalcGridX::getWholeDensity, :2502-2537).
 * Either of exc, nelec_alpha may be NULL. */
pdfxc_status pdfxc_build_vxc(pdfxc_ctx* ctx, int functional, const double* PA, int incremental,
                             double* F, double* exc, double* nelec_alpha);

/* Same build on device-resident operands (d_PA, d_V: n_ao*n_ao FP64 device
 * pointers; d_V is overwritten with Vxc, not accumulated), enqueued on the
 * context's stream; exc/nelec_alpha are host pointers filled after the stream
 * synchronises. */
pdfxc_status pdfxc_build_vxc_device(pdfxc_ctx* ctx, int functional, const double* d_PA,
                                    int incremental, double* d_V, double* exc,
                                    double* nelec_alpha);

/* The XC part of the Fock update kept on the device: replaces the host round trip of
 * DfFockMatrix::setXC_DIRECT (src/libpdf/DfFockMatrix.h:711-721), which loads Fxc of this
 * iteration and, from the second iteration on, subtracts Fxc of the previous one. Builds Vxc of
 * SCF iteration `iteration` (>= 1) from d_PA as pdfxc_build_vxc_device does, keeps it in the
 * context, and writes d_dV = Vxc(iteration) - Vxc(iteration - 1) for iteration >= 2, d_dV =
 * Vxc(1) for iteration 1 (device n_ao*n_ao FP64, overwritten). d_V (optional, NULL to skip)
 * receives Vxc(iteration). For iteration >= 2 the context's previous call of this function must
 * have been iteration - 1 (else PDFXC_ERR_STATE; pdfxc_set_system clears the history). */
pdfxc_status pdfxc_build_vxc_delta_device(pdfxc_ctx* ctx, int functional, const double* d_PA,
                                          int incremental, int iteration, double* d_V,
                                          double* d_dV, double* exc, double* nelec_alpha);

/* Per-point densities of the last build in input point order: npts x 1
 * (LDA: rho_A) or npts x 4 (GGA: rho_A, d/dx, d/dy, d/dz) -- the rho columns
 * of the grid matrix (src/libpdf/DfCalcGridX.h:35-54). pdfxc_set_rho seeds
 * them (restart with xc-update = yes). */
pdfxc_status pdfxc_get_rho(pdfxc_ctx* ctx, int gga, double* rho);
pdfxc_status pdfxc_set_rho(pdfxc_ctx* ctx, int gga, const double* rho);

/* Density at arbitrary points: rho[i] = sum_jk P[j][k] phi_j(r_i) phi_k(r_i) for the
 * row-major n_ao x n_ao host matrix P and the points xyz (npts x 3, bohr). Replaces
 * DfCalcGridX::gridDensity (src/libpdf/DfCalcGridX.cpp:1038-1044, AO values of every
 * basis function then getRhoAtGridPoint, :865-881), which TlDensField::makeDensFld
 * (src/tools/TlDensField.cpp:35-53) calls once per point of a density-field grid. Needs
 * pdfxc_set_system; runs on the FP64 path of a private grid, so the context's own grid,
 * stored densities and build graphs are untouched. No weights, no functional. */
pdfxc_status pdfxc_density(pdfxc_ctx* ctx, const double* P, int64_t npts, const double* xyz, double* rho);

/* Open-shell build, on the FP64 path and on the INT8 digits (split_terms 10; the
 * BF16 split returns PDFXC_ERR_UNSUPPORTED). Replaces the UKS overloads
 * DfCalcGridX::calcXCIntegForFockAndEnergy(P_A, P_B, functional, F_A, F_B)
 * (src/libpdf/DfCalcGridX.cpp:2292-2303 LDA, :2317-2328 GGA): calcRho_*_part
 * on both spin densities (:1891-1922, :1963-2016) and buildVxc(gridMatrix,
 * functional, F_A, F_B) (:2093-2135, :2195-2278). PA, PB: n_ao x n_ao (host).
 * FA, FB: accumulated into. A point contributes when rho_A or rho_B exceeds
 * the density cut-off. Per spin s the GGA coefficient is the reference's,
 * w (2 vgamma_ss + vgamma_AB) grad rho_s (its build_XC_Matrix, :2455-2500, is
 * given the spin's own gradient only). incremental: as pdfxc_build_vxc, for
 * both spins. nelec_alpha, nelec_beta: sum_i w_i rho_s(r_i). */
pdfxc_status pdfxc_build_vxc_uks(pdfxc_ctx* ctx, int functional, const double* PA, const double* PB,
                                 int incremental, double* FA, double* FB, double* exc,
                                 double* nelec_alpha, double* nelec_beta);

/* Open-shell per-point densities in input point order, the grid-matrix
 * columns of the open shell (src/libpdf/DfCalcGridX.h:35-54): npts x 2 (LDA:
 * rho_A, rho_B) or npts x 8 (GGA: rho_A, grad rho_A, rho_B, grad rho_B). */
pdfxc_status pdfxc_get_rho_uks(pdfxc_ctx* ctx, int gga, double* rho);
pdfxc_status pdfxc_set_rho_uks(pdfxc_ctx* ctx, int gga, const double* rho);

/* XC nuclear gradient (closed shell, FP64) at a fixed density, on the grid of
 * pdfxc_set_grid, which must have been given the owning atom of every point
 * (each point moves with its atom). Replaces DfCalcGridX::energyGradient
 * (src/libpdf/DfCalcGridX.cpp:1073-1099 LDA, :1209-1235 GGA) and its
 * energyGradient_part (:1101-1207, :1237-1415).
 * grad_orbital (host, n_atom x 3, overwritten): the AO-centre term, the
 *   reference's Fxc_f after its closed-shell factor 2.
 * w_single (host, npts in set_grid order, or NULL): single-centre weights of
 *   the points; with it grad_weight (host, n_atom x 3, overwritten) receives
 *   the grid-weight term, the derivative of the Becke partition (radii
 *   becke_radius[n_atom], size_adjust as in pdfxc_becke_weights; at most 400
 *   atoms). The reference's own weight term (Fxc_w, JGP_nablaB_omegaA,
 *   src/libpdf/DfGenerateGrid.cpp:2259-2393) is identically zero, because its
 *   JGP_t returns 0 for every |mu| <= 1; pass w_single = NULL for its output.
 * exc (may be NULL): the XC energy on the grid. */
pdfxc_status pdfxc_xc_gradient(pdfxc_ctx* ctx, int functional, const double* PA,
                               const double* w_single, const double* becke_radius, int size_adjust,
                               double* grad_orbital, double* grad_weight, double* exc);

/* The adjoint of the closed-shell XC energy, Exc(P, R), on the grid of pdfxc_set_grid (owner
 * atoms required), FP64. dexc is the cotangent of Exc (the upstream derivative dL/dExc; 1 for
 * the derivatives themselves); every output is scaled by it. Per workspace chunk the AO values,
 * gradients and second derivatives are recomputed (none is kept from a build), X = P_sub phi,
 * the functional's derivatives at every point, then
 *   dexc_dP (host, n_ao x n_ao, overwritten): dL/dP for the total density P = 2 PA, each
 *     element taken as independent -- sum over points of phi Z^T + Z phi^T with the density
 *     adjoint Z = 0.5 w vrho phi + w (2 vgAA + vgAB) grad rho . grad phi, which is the
 *     build's Vxc (SCF codes such as the reference feed Vxc = dExc/dP into F); dL/dPA is
 *     2 dexc_dP;
 *   grad_orbital, grad_weight (host, n_atom x 3, as pdfxc_xc_gradient): dL/dR, the AO-centre
 *     term with the points moving with their atoms, and, with w_single, the derivative of the
 *     Becke partition (at most 400 atoms; NULL w_single leaves the weight term out);
 *   exc (may be NULL): Exc itself.
 * Replaces the derivative side of DfCalcGridX (energyGradient / energyGradient_part,
 * src/libpdf/DfCalcGridX.cpp:1073-1415); the dExc/dP output has no separate routine in the
 * reference, whose calcXCIntegForFockAndEnergy returns the same matrix from the forward pass. */
pdfxc_status pdfxc_xc_backward(pdfxc_ctx* ctx, int functional, const double* PA, double dexc,
                               const double* w_single, const double* becke_radius, int size_adjust,
                               double* dexc_dP, double* grad_orbital, double* grad_weight, double* exc);

/* A batch of independent molecules in one context: every stage of a build runs
 * once for all of them (one launch per stage over the blocks of every molecule,
 * one captured CUDA graph per build). Each molecule's points are blocked and
 * screened against its own shells only; the joint AO space is the molecules'
 * AO spaces one after another, and P, Vxc are kept as one dense matrix of that
 * size whose diagonal blocks are used. No counterpart in the reference (its
 * DfCalcGridX holds one molecule). */
typedef struct {
    int natom;
    const double* atom_xyz;   /* natom x 3, bohr */
    const int* atom_z;        /* may be NULL */
    int nshell;
    const int* shell_atom;    /* 0..natom-1, this molecule's atoms */
    const int* shell_l;
    const int* shell_nprim;
    const double* prim_exp;
    const double* prim_coef;
    int64_t npts;
    const double* xyzw;       /* npts x 4 */
    const int* atom;          /* owner atom per point (this molecule's numbering), or NULL */
} pdfxc_mol;
pdfxc_status pdfxc_set_batch(pdfxc_ctx* ctx, int nmol, const pdfxc_mol* mols);
/* PA[m]: n_m x n_m alpha density of molecule m (host); F[m] += Vxc_m; exc[m],
 * nelec_alpha[m] per molecule (either array may be NULL). */
pdfxc_status pdfxc_build_vxc_batched(pdfxc_ctx* ctx, int functional, const double* const* PA, int incremental,
                                     double* const* F, double* exc, double* nelec_alpha);

/* Sharding one molecule over several GPUs (the reference's MPI variant distributes
 * grid rows and all-reduces F and E, src/libpdf/DfCalcGridX_Parallel.cpp:191-239).
 * pdfxc_block_costs gives each block's contraction cost 4 nb^2 np (nblocks
 * values, see pdfxc_grid_stats); pdfxc_partition_blocks (no context, no device)
 * cuts blocks 0..nblk-1 into nparts contiguous ranges of near-equal cost,
 * bounds[0..nparts]; pdfxc_set_block_range restricts every later build
 * (closed shell, open shell, gradient) of the context to blocks [b_lo, b_hi), so
 * that each rank's Vxc, Exc, electron count and gradient are partial sums whose
 * all-reduce is the whole. The stored densities of xc-update stay per rank. */
pdfxc_status pdfxc_block_costs(pdfxc_ctx* ctx, double* cost);
pdfxc_status pdfxc_partition_blocks(int64_t nblk, const double* cost, int nparts, int64_t* bounds);
pdfxc_status pdfxc_set_block_range(pdfxc_ctx* ctx, int64_t b_lo, int64_t b_hi);

/* The blocking and screening of a grid, planned on the host without a device or
 * context: what pdfxc_set_grid would build for these options, system and points
 * (same blocks, groups, screened shells and workspace chunks). Returns
 * PDFXC_ERR_UNSUPPORTED where pdfxc_set_grid would: a mixed-precision (INT8)
 * context takes at most 32,512 screened AOs per group, the bound up to which its
 * int32 accumulation and the FP64 combination of its digit orders are exact. No counterpart in the reference (it does not
 * screen, src/libpdf/DfCalcGridX.cpp:655-665); tile and group shapes can be
 * compared with it before a context is made. */
typedef struct {
    int64_t nblocks, ngroups, npts_padded;
    int max_nb;               /* largest screened AO count of a block */
    double contraction_flops; /* sum over blocks of 4 nb^2 np */
    double mean_nb;
    size_t workspace_bytes;   /* the largest workspace chunk */
    int nchunks;
} pdfxc_grid_plan;
pdfxc_status pdfxc_plan_grid(const pdfxc_options* opt, int natom, const double* atom_xyz, int nshell,
                             const int* shell_atom, const int* shell_l, const int* shell_nprim,
                             const double* prim_exp, const double* prim_coef, int64_t npts, const double* xyzw,
                             pdfxc_grid_plan* out);

/* The exchange step of a sharded build (the reference all-reduces F,
 * src/libpdf/DfCalcGridX_Parallel.cpp:191-239): a symmetric n x n device
 * matrix's upper triangle (j >= i) packed row by row into n (n + 1) / 2
 * doubles, so that one all-reduce moves half the matrix, and the inverse, which
 * writes both triangles. Device pointers; enqueued on `stream` (a cudaStream_t,
 * NULL = the default stream) without synchronising. */
pdfxc_status pdfxc_pack_upper(const double* d_V, int n, double* d_packed, void* stream);
pdfxc_status pdfxc_unpack_upper(const double* d_packed, int n, double* d_V, void* stream);

/* Statistics of the blocked grid: blocks, points (after padding), the sum of
 * 4 * nb^2 * np over blocks (the algorithmic contraction FLOPs of one build)
 * and the mean screened AO count per block. */
pdfxc_status pdfxc_grid_stats(pdfxc_ctx* ctx, int64_t* nblocks, int64_t* npts_padded,
                              double* contraction_flops, double* mean_nb);

/* Device time (ms) of the last build, measured with CUDA events on the
 * context's stream, split by stage and summed over the workspace chunks, and
 * the number of kernels the build launched. */
typedef struct {
    float total_ms;     /* first to last event of the build */
    float ao_ms;        /* basis-function (and gradient) evaluation */
    float gemm_x_ms;    /* X = P_sub * phi contraction */
    float rho_ms;       /* rho / grad rho reduction and the functional */
    float gemm_v_ms;    /* Vxc += phi Z^T contraction */
    float finish_ms;    /* symmetrisation and FP64 block sums */
    int64_t launches;   /* kernels launched by the build */
} pdfxc_profile;

pdfxc_status pdfxc_last_profile(pdfxc_ctx* ctx, pdfxc_profile* out);

/* Builds normally replay one captured CUDA graph per configuration, which
 * times the build as a whole (total_ms). With profiling enabled the build is
 * launched stage by stage instead, so that the per-stage times of
 * pdfxc_last_profile are filled in. */
pdfxc_status pdfxc_set_profiling(pdfxc_ctx* ctx, int enable);

/* The autotuner. Times one closed-shell build of `functional` (device density d_PA, n_ao x n_ao;
 * NULL = the context's staging matrix as it stands) for every candidate shape of the context's
 * path -- on the INT8 path groups of 4, 2 or 1 blocks sharing one screened basis, times 3 or 2
 * operand stages of the Vxc contraction; the FP64 path has none to choose -- on the context's own
 * grid (re-blocked per candidate), a warm-up and the better of two timed builds each. Leaves the
 * context on the fastest shape, and keeps it for the process under the workload's class
 * (precision, operand split, batch or not, the AO and point counts to a factor of two): later
 * contexts of that class whose options leave group_blocks / vxc_stages at 0 start from it. The
 * stored densities of xc-update are dropped (call it before the first SCF build). out[0] is the
 * winner, then the other candidates; *n_out = min(candidates, max_out). No counterpart in the
 * reference. */
typedef struct {
    int group_blocks;
    int vxc_stages;
    int block_points;
    float ms;           /* the build's device time with this shape */
} pdfxc_tuning;
pdfxc_status pdfxc_autotune(pdfxc_ctx* ctx, int functional, const double* d_PA, pdfxc_tuning* out, int max_out,
                            int* n_out);
/* The shapes the context's grid uses (group_blocks 1 and vxc_stages 0 on the FP64 path) and, in
 * ms, the device time of its last build. */
pdfxc_status pdfxc_get_tuning(pdfxc_ctx* ctx, pdfxc_tuning* out);

/* The failure path of the library's bounded device waits, exercised without a fault: a kernel
 * waits on an mbarrier that nothing completes, through the same bounded wait as the tensor-core
 * contraction kernels, gives up after limit_seconds (0 < limit <= 10) and records its code in the
 * context's device error word; the host reads it as the builds do and returns
 * PDFXC_ERR_TIMEOUT, the expected result. The error word is cleared again, so the context stays
 * usable. No counterpart in the reference (its waits are MPI and OpenMP barriers). */
pdfxc_status pdfxc_selftest_wait(pdfxc_ctx* ctx, double limit_seconds);

const char* pdfxc_last_error(const pdfxc_ctx* ctx);
void pdfxc_destroy(pdfxc_ctx* ctx);

/* FP64 XC build that allocates nothing. This entry point has no counterpart
 * in the reference; it exists for callers that cannot call cudaMalloc (their
 * device memory belongs to a pool or arena they do not control, or they run
 * where allocation is forbidden). Every operand is a device pointer the caller
 * owns: the shells as in pdfxc_set_system (each shell's primitives by ascending exponent,
 * the reference's order), npts grid rows (x, y, z, w), the
 * n_ao x n_ao alpha density d_PA; d_V (n_ao x n_ao) is overwritten with Vxc
 * and d_exc_nelec[0..1] with Exc and sum_i w_i rho_A(r_i). The intermediates
 * live in a fixed 32 MiB __device__ array of the library, held by every GPU
 * that loads it until the process exits. Limits: n_ao <= 256, nshell <= 256,
 * else PDFXC_ERR_ARG. Every call shares that array (the accumulators are
 * cleared at the start of a call), so calls that overlap on the GPU race; the
 * call synchronises `stream` (a cudaStream_t, NULL = default stream) before it
 * returns. Its first call on a device looks up the array's device address;
 * make that first call before any stream capture. */
pdfxc_status pdfxc_build_vxc_noalloc(int device, int functional, int natom, const double* d_atom_xyz,
                                     int nshell, const int* d_shell_atom, const int* d_shell_l,
                                     const int* d_shell_nprim, const double* d_prim_exp,
                                     const double* d_prim_coef, int nao, int64_t npts,
                                     const double* d_xyzw, const double* d_PA, double* d_V,
                                     double* d_exc_nelec, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PDFXC_H */
