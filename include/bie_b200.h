/*
 * bie_b200.h -- C ABI of libbie_b200.so, the B200 (sm_100a) layer-potential
 * library for the dielectric boundary-integral equation of DielectricBIE.jl.
 *
 * Conventions
 *   - Host arrays are borrowed for the duration of a call, Float64, in Julia's
 *     column-major layout: points/normals 3 x N (x, y, z of node i contiguous),
 *     multi-column vectors N x k (column c contiguous).
 *   - Device arrays passed to the *_device entry points use the library's
 *     device layout: N x k row-major ("node-major", the k values of node i
 *     contiguous). For k = 1 the two layouts coincide.
 *   - Every entry point returns a bie_status; no exception crosses the ABI. The
 *     message of the last failure on the calling thread is kept for
 *     bie_last_error.
 *   - A bie_geom is bound to one CUDA device and one stream; calls on distinct
 *     handles may run concurrently from different threads, calls on one handle
 *     must be serialised by the caller.
 *   - Node order is the reference's: panels in mesher order, within a panel the
 *     (b - a) Gauss index outer and the (d - a) index inner
 *     (src/shape/box3d.jl:44-52, src/core/panels.jl:87-115).
 */
#ifndef BIE_B200_H
#define BIE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    BIE_OK = 0,
    BIE_EINVAL = 1,        /* bad argument (sizes, null pointers, options) */
    BIE_ENOMEM = 2,        /* device or host allocation failed */
    BIE_ECUDA = 3,         /* CUDA runtime error (message in bie_last_error) */
    BIE_ENOCONV = 4,       /* solver stopped at itmax before reaching the tolerance */
    BIE_ETIMEOUT = 5,      /* a bounded device wait ran out (kernel returned early) */
    BIE_EUNSUPPORTED = 6,  /* valid request outside what this build supports */
    BIE_ENODEVICE = 7      /* no CUDA device (the library has no CPU fallback) */
} bie_status;

/* Arithmetic of the layer-potential sum inside a matvec / solve. */
typedef enum {
    BIE_FP64 = 0,   /* plain: FP64 end to end */
    BIE_FP32 = 1,   /* FP32 direct sum (FP64 tile partials), FP64 corrections/diag */
    BIE_BF16X3 = 2, /* split-BF16 three-term tensor-core RHS contraction (FP32 sum for k = 1, 2, 4),
                       FP32 kernel tiles, FP64 corrections/diag */
    BIE_BF16X6 = 3  /* three bf16 pieces per operand, six tensor-core products (idem):
                       about FP32 accuracy; the refinement's residual updates use it */
} bie_precision;

/* matvec flags */
#define BIE_NO_CORRECTIONS 1u /* skip the near-field correction blocks */
#define BIE_NO_DIAG 2u        /* skip the diagonal contrast term */
#define BIE_NO_VERIFY 4u      /* solve: skip the final FP64 true-residual evaluation (stats then
                                 report the solver's own residual estimate) */

/* Copies the message of the last failed call on this thread (always NUL-terminated).
 * Returns the full message length. */
int bie_last_error(char* buf, size_t len);
/* Library version string, e.g. "bie_b200 0.1 sm_100a". */
const char* bie_version(void);
/* Number of visible CUDA devices (0 on a machine without a GPU). */
int bie_device_count(void);

/* ------------------------------------------------------------------------- */
/* Host-side geometry setup                                                   */
/* ------------------------------------------------------------------------- */
/* gausslegendre(n) of FastGaussQuadrature.jl (ascending nodes). Called by the
 * reference at src/shape/box3d_single.jl:50. */
int bie_gausslegendre(int n, double* x, double* w);
/* best_grid_mn (src/utils/best_grid.jl:120-126): m x n tiling with aspect <= alpha. */
int bie_best_grid(double W, double H, double alpha, int* m, int* n);

typedef struct bie_mesh bie_mesh;
/* single_dielectric_box3d(Lx, Ly, Lz, n_quad, l_ec, eps_in, eps_out; alpha)
 * (src/shape/box3d_single.jl:49-70). */
int bie_mesh_single_box(double Lx, double Ly, double Lz, int n_quad, double l_ec, double eps_in, double eps_out,
                        double alpha, bie_mesh** out);
/* multi_dielectric_box3d(n_quad, l_ec, boxes, epses, eps_out; alpha)
 * (src/shape/box3d_multi.jl:358-386). centers/dims are 3 x nbox. */
int bie_mesh_multi_box(int n_quad, double l_ec, int nbox, const double* centers, const double* dims,
                       const double* epses, double eps_out, double alpha, bie_mesh** out);
/* DielectricInterface of explicit flat panels (rect_panel3d_discretize,
 * src/shape/box3d.jl:22-64): corners 12 x P (a, b, c, d), normals 3 x P. */
int bie_mesh_from_panels(int npanels, int n_quad, const double* corners, const double* normals,
                         const int* is_edge, const double* eps_in, const double* eps_out, bie_mesh** out);
int bie_mesh_info(const bie_mesh* m, int64_t* npoints, int* npanels, int* n_quad);
/* Any output pointer may be NULL. pts/nrm are 3 x N, diag is t_P per node
 * (src/solver/dielectric_box3d.jl:5-15). */
int bie_mesh_copy(const bie_mesh* m, double* corners, double* normals, int* is_edge, double* eps_in,
                  double* eps_out, double* pts, double* nrm, double* w, double* diag);
void bie_mesh_destroy(bie_mesh* m);

/* Near-field correction options; defaults are those of the reference's
 * corrected operators (src/solver/dielectric_box3d.jl:48-60,
 * src/solver/multi_rhs.jl:273-275). */
typedef struct {
    int max_order;             /* upsampling order cap (default 8) */
    double up_tol;             /* Bernstein criterion tolerance (default 1e-9) */
    int correct_edges;         /* include edge panels and touching pairs (default 1) */
    double adaptive_atol;      /* < 0 => up_tol */
    double adaptive_rtol;      /* default sqrt(eps) */
    int adaptive_n_GL;         /* 0 => n_quad */
    int adaptive_max_depth;    /* default 20 */
    int nthreads;              /* host threads, 0 = all */
    int device;                /* >= 0: the adaptive (touching-pair) blocks' moment sums and the upsampled
                                  blocks of sources with n_up <= 8 run on this CUDA device, bitwise equal
                                  to the host's (n_quad <= 6); -1 = host only */
} bie_near_opts;
void bie_near_opts_default(bie_near_opts* o);

typedef struct bie_near bie_near;
/* build_neighbor_list (src/kernel/laplace3d_near.jl:240-392) and
 * laplace3d_DT_corrections (src/kernel/laplace3d_near_upsampling.jl:127-276),
 * stored block-sparse: block rows = target panels, blocks nb x nb (nb = n_quad^2),
 * column-major within a block (val[b*nb*nb + s*nb + r] = C[row r, col s]). */
int bie_near_build(const bie_mesh* m, const bie_near_opts* o, bie_near** out);
int bie_near_info(const bie_near* n, int64_t* nblocks, int* nb, int* n_upsample, int* n_adaptive, int* hit_max_depth);
/* rowptr: npanels + 1, col: nblocks, val: nblocks*nb*nb; pair lists (0-based
 * source panel i, target panel j, upsampling order p). Any pointer may be NULL. */
int bie_near_copy(const bie_near* n, int32_t* rowptr, int32_t* col, double* val, int32_t* ups_i, int32_t* ups_j,
                  int32_t* ups_p, int32_t* adp_i, int32_t* adp_j);
/* Frees the handle's host copy of the block values (nblocks*nb*nb doubles) once a device
 * geometry holds them; the structure (rowptr, col, pair lists) stays. Afterwards
 * bie_near_copy with val != NULL and bie_geom_create_from_mesh on this handle return
 * BIE_EINVAL; bie_geom_near_values reads the values back from a geometry. A server that
 * keeps many geometries resident holds their blocks once, on the device. No counterpart
 * in the reference (its operator closure keeps the CSC matrix). */
int bie_near_release_values(bie_near* n);
void bie_near_destroy(bie_near* n);

/* ------------------------------------------------------------------------- */
/* Device-resident geometry                                                   */
/* ------------------------------------------------------------------------- */
typedef struct bie_geom bie_geom;
/* Copies nodes, normals, weights, diagonal and (optional) BSR correction blocks
 * to `device`. Replaces the SoA gather of laplace3d_DT_fmm3d
 * (src/kernel/laplace3d.jl:84-97) and BatchedDielectricOperator's fields
 * (src/solver/multi_rhs.jl:46-54). bsr_* may be NULL (no corrections). */
int bie_geom_create(const double* pts, const double* nrm, const double* w, const double* diag, int64_t n,
                    int32_t npanels, int32_t nb, const int32_t* bsr_rowptr, const int32_t* bsr_col,
                    const double* bsr_val, int64_t nblocks, int device, bie_geom** out);
/* Convenience: from a mesh and (optional) near-field blocks. */
int bie_geom_create_from_mesh(const bie_mesh* m, const bie_near* near, int device, bie_geom** out);
int bie_geom_info(const bie_geom* g, int64_t* n, int64_t* nblocks, size_t* device_bytes);
/* Copies the geometry's device correction blocks to val (len = nblocks*nb*nb doubles, the
 * layout of bie_near_copy); BIE_EINVAL when len differs. */
int bie_geom_near_values(bie_geom* g, double* val, int64_t len);
/* The CUDA stream (cudaStream_t) the handle's work is ordered on. */
void* bie_geom_stream(bie_geom* g);
void bie_geom_destroy(bie_geom* g);

/* ------------------------------------------------------------------------- */
/* Operators                                                                  */
/* ------------------------------------------------------------------------- */
/* Y = (D^T + C + diag(t)) X for k columns: the action of lhs_dielectric_box3d
 * (dense, src/solver/dielectric_box3d.jl:1-17) and of
 * lhs_dielectric_box3d_fmm3d_corrected / BatchedDielectricOperator mul!
 * (src/solver/dielectric_box3d.jl:48-92, src/solver/multi_rhs.jl:103-136) with the
 * FMM replaced by the exact direct sum (j != i). Host arrays, N x k column-major. */
int bie_matvec(bie_geom* g, const double* X, double* Y, int32_t k, int32_t precision, uint32_t flags);
/* Same on device arrays (node-major N x k) ordered on `stream` (NULL = the handle's). */
int bie_matvec_device(bie_geom* g, const double* dX, double* dY, int32_t k, int32_t precision, uint32_t flags,
                      void* stream);

/* No counterpart in the reference. FP64 direct sum of the adjoint double layer
 * without near-field correction or diagonal, that allocates no device memory:
 *   Y[i][c] = 1/(4 pi) sum_{j != i} n_i.(x_i - y_j)/|x_i - y_j|^3 w_j X[j][c].
 * It is for callers that cannot let a library allocate: host runtimes whose pool
 * allocator owns the device memory (Julia's CUDA.jl, PyTorch's caching allocator),
 * where a foreign cudaMalloc can fail while the pool holds free memory, and
 * latency-bound services that reserve memory at start-up, since cudaMalloc and
 * cudaFree synchronise the device. The split partials live in a fixed 32 MiB
 * device array inside the library (held by every device the library runs it on,
 * until the process exits); the caller passes all inputs and outputs as device
 * pointers on the current device: node coordinates x, y, z, unit normals nx, ny,
 * nz and weights w (n each), X and Y node-major n x k (Y must not overlap X).
 * Limit: n <= 4,194,304 nodes; larger n is rejected with BIE_EINVAL before any
 * device work. The first call on a device looks up the array's address; make that
 * first call before any stream capture. Under lazy module loading (the CUDA 12
 * default) that lookup is also when the 32 MiB is committed on the device: make the
 * first call before a pool allocator reserves the device's memory, else it fails with
 * BIE_ENOMEM. With CUDA_MODULE_LOADING=EAGER every context that loads the library
 * holds the 32 MiB from the start, whether or not this entry point is used. Calls share the array: every partial a
 * call reads is written earlier in the same call, so nothing needs clearing, but
 * calls that overlap on the GPU (other streams, other threads) race on it and
 * must be serialised by the caller. Work is ordered on `stream` (NULL = the
 * default stream); the call returns without synchronising. */
int bie_dt_apply_static(const double* x, const double* y, const double* z, const double* nx, const double* ny,
                        const double* nz, const double* w, int64_t n, const double* X, int32_t k, double* Y,
                        void* stream);

/* F[:, c] = rhs_dielectric_box3d(itf, PointSource(src[:, c], q[c]), eps_src[c])
 * (src/solver/dielectric_box3d.jl:95-104). src 3 x k, F N x k (host). */
int bie_rhs_point(bie_geom* g, const double* src, const double* q, const double* eps_src, int32_t k, double* F);
int bie_rhs_point_device(bie_geom* g, const double* d_src, const double* d_q, const double* d_eps_src, int32_t k,
                         double* dF, void* stream);

/* phi[m, c] = S[Sigma[:, c]](targets[:, m]) = sum_j w_j Sigma[j, c] / (4 pi |x_m - y_j|)
 * (laplace3d_pottrg, src/kernel/laplace3d.jl:69-82). targets 3 x M, phi M x k (host). */
int bie_potential(bie_geom* g, const double* Sigma, int32_t k, const double* targets, int64_t M, double* phi);
/* Same with device arrays: d_sigma node-major N x k, d_targets 3 x M, d_phi M x k row-major. */
int bie_potential_device(bie_geom* g, const double* d_sigma, int32_t k, const double* d_targets, int64_t M,
                         double* d_phi, void* stream);
/* Near-accurate probe potentials: the operator of laplace3d_pottrg_fmm3d_corrected_hcubature
 * (src/kernel/laplace3d_near_hcubature.jl:278-316), phi = (S_refined + C) P Sigma. Panels of
 * the mesh near the probes are split 4-way down to the smallest panel size, P interpolates
 * Sigma onto the refined nodes, S_refined is their smooth-quadrature potential (GPU direct
 * sum) and C corrects every probe within range_factor * l_panel / n_quad of a refined
 * non-edge panel by that panel's adaptive integral (Genz-Malik cubature to hcubature_atol)
 * minus its smooth-quadrature terms. targets 3 x M. device < 0 builds the host operator only
 * (bie_probe_info / bie_probe_copy work, bie_probe_apply returns BIE_EINVAL). */
typedef struct bie_probe bie_probe;
int bie_probe_create(const bie_mesh* m, const double* targets, int64_t M, double hcubature_atol,
                     double range_factor, int32_t device, bie_probe** out);
/* Sizes: refined nodes and panels, nonzeros of P and C, adaptive integrals evaluated and
 * how many of them stopped at the evaluation cap (2^24 per integral) before reaching atol. */
int bie_probe_info(const bie_probe* p, int64_t* n_refined, int32_t* npanels_refined, int64_t* nnz_prolongation,
                   int64_t* nnz_corrections, int64_t* ncubatures, int64_t* capped);
/* Copies (any pointer may be null): parent coarse panel and split flag per refined panel,
 * refined panel corners (npanels_refined x 4 x 3), refined nodes 3 x n_refined and weights,
 * P in CSR (prow n_refined + 1, pcol / pval nnz) and C in CSR (crow M + 1, ccol / cval nnz). */
int bie_probe_copy(const bie_probe* p, int32_t* parent, int32_t* from_split, double* refined_corners,
                   double* refined_pts, double* refined_w, int64_t* prow, int32_t* pcol, double* pval,
                   int64_t* crow, int32_t* ccol, double* cval);
/* phi (M x k, column-major) = operator applied to Sigma (N x k, column-major). */
int bie_probe_apply(bie_probe* p, const double* Sigma, int32_t k, double* phi);
void bie_probe_destroy(bie_probe* p);
/* Polarisation energy of point sources: W[c] = 1/2 q[c] S[Sigma[:, c]](src[:, c]). src 3 x k. */
int bie_energy(bie_geom* g, const double* Sigma, int32_t k, const double* src, const double* q, double* W);

/* ------------------------------------------------------------------------- */
/* Solvers                                                                    */
/* ------------------------------------------------------------------------- */
typedef struct {
    double atol;         /* absolute residual tolerance (default 0) */
    double rtol;         /* relative residual tolerance per column (default 1e-10) */
    int itmax;           /* maximum Krylov iterations in total (default 500) */
    int restart;         /* Krylov basis capacity before restart (default 200) */
    int precision;       /* bie_precision of the Krylov operator (default BIE_FP64) */
    double inner_rtol;   /* mixed precision: relative tolerance of each inner solve (default 1e-6; never
                            tighter than twice the inner operator's relative error) */
    int max_outer;       /* mixed precision: maximum refinement steps (default 8) */
    int precondition;    /* right diagonal preconditioner 1/t_P (src/solver/multi_rhs.jl:234-247) */
    int check_every;     /* host convergence check period in iterations (default 1) */
    uint32_t flags;      /* BIE_NO_CORRECTIONS etc. applied to the operator */
    int block;           /* 1: block GMRES for 1 < k <= 64 (Krylov.block_gmres, src/solver/multi_rhs.jl:285):
                            the active columns share one block Krylov space (restart = block iterations
                            per cycle, at most 60); wider solves run one Arnoldi process per column, which
                            shares one operator application per iteration over all columns (faster here);
                            0: one Arnoldi process per column (default) */
} bie_solve_opts;
void bie_solve_opts_default(bie_solve_opts* o);

typedef struct {
    int iterations;       /* Krylov iterations (all refinement steps) */
    int outer;            /* refinement steps (1 for FP64) */
    int fp64_matvecs;     /* full FP64 operator applications */
    int lowp_matvecs;     /* reduced-precision operator applications */
    int converged;        /* all columns reached atol + rtol * ||F[:, c]|| */
    double max_rel_resid; /* max_c ||F - A Sigma||_c / ||F||_c: the FP64 true residual unless
                             BIE_NO_VERIFY is set, else the maintained residual */
    double seconds;       /* device time of the solve */
    int* col_iterations;  /* optional (k entries): Krylov iterations per column */
    double* col_resid;    /* optional (k entries): final true relative residual per column */
} bie_stats;

/* Solves (D^T + C + diag(t)) Sigma = F for k right-hand sides: solve_gmres /
 * Krylov.gmres (src/utils/linear_algebra.jl:3-5) for k = 1 and
 * solve_dielectric_box3d_block / Krylov.block_gmres (src/solver/multi_rhs.jl:270-286)
 * for k > 1, run on the device (all k columns iterate together, each with its own
 * Arnoldi process; converged columns are frozen). With precision != BIE_FP64 the
 * Krylov operator is the reduced-precision one inside FP64 iterative refinement.
 * Host arrays N x k. Returns BIE_ENOCONV (with Sigma filled) when itmax is hit. */
/* After a solve (bie_solve, bie_solve_device) the library releases the handle's solver
 * workspace, about (restart + 1) N k doubles, when less than a quarter of the device
 * memory is free (always with the environment variable BIE_TRIM_WORKSPACE), so that many
 * resident geometries solved in turn do not keep a workspace each. The next solve
 * allocates it again. The free memory is queried only when the library's own device
 * allocations changed since the last query that found enough free (a steady stream of
 * solves does not pay for the query). */
int bie_solve(bie_geom* g, const double* F, double* Sigma, int32_t k, const bie_solve_opts* o, bie_stats* st);
int bie_solve_device(bie_geom* g, const double* dF, double* dSigma, int32_t k, const bie_solve_opts* o,
                     bie_stats* st, void* stream);
/* Point-source block solve with host buffers: F[:, c] = rhs_dielectric_box3d(itf,
 * PointSource(src[:, c], q[c]), eps_src[c]) (src/solver/dielectric_box3d.jl:95-104) is built
 * on the device and solved there as bie_solve does (solve_dielectric_box3d_block,
 * src/solver/multi_rhs.jl:270-286). src 3 x k, Sigma N x k (host, column-major). Only the
 * 5 k source values go to the device and only Sigma comes back: the N x k right-hand side
 * never crosses the host link, as it does with bie_rhs_point followed by bie_solve. */
int bie_solve_point(bie_geom* g, const double* src, const double* q, const double* eps_src, int32_t k, double* Sigma,
                    const bie_solve_opts* o, bie_stats* st);

/* Several geometries at once: the reduced-precision operator of G geometries applied in
 * ONE launch of the tensor-core direct sum over a work list of every geometry's (target tile,
 * source split) items, largest geometries first, followed by each geometry's correction
 * apply: mul!(Y, ::BatchedDielectricOperator, X) (src/solver/multi_rhs.jl:103-136) for G
 * operators of uneven size. precision BIE_BF16X3 or BIE_BF16X6; member i has ks[i] <= 128
 * columns, dX[i] / dY[i] node-major n_i x k_i device arrays; the geometries must differ and
 * live on one device. Work is ordered on `stream` (NULL = the first geometry's); the
 * members' own streams are synchronised first. */
int bie_matvec_group_device(bie_geom* const* gs, int32_t G, const double* const* dX, double* const* dY,
                            const int32_t* ks, int32_t precision, uint32_t flags, void* stream);
/* Block solves of G geometries in lockstep (solve_dielectric_box3d_block per geometry,
 * src/solver/multi_rhs.jl:270-286), precision BIE_BF16X3 or BIE_BF16X6: every inner Krylov
 * iteration applies all members' operators with one work-list launch (as
 * bie_matvec_group_device) and issues their Krylov kernels and convergence reads together,
 * so a group of small geometries pays one set of per-iteration host round trips. Each
 * member runs its own FP64 refinement and Krylov processes, as bie_solve_device would; st
 * (optional) has G entries. The diagonal preconditioner is not available here
 * (BIE_EUNSUPPORTED). */
int bie_solve_group_device(bie_geom* const* gs, int32_t G, const double* const* dF, double* const* dSigma,
                           const int32_t* ks, const bie_solve_opts* o, bie_stats* st, void* stream);

/* ------------------------------------------------------------------------- */
/* Kernel timing (CUDA events on the launching stream)                        */
/* ------------------------------------------------------------------------- */
typedef enum {
    BIE_KERNEL_DIRECT_FP64 = 0,  /* K1 FP64 direct sum */
    BIE_KERNEL_DIRECT_FP32 = 1,  /* K2 FP32 direct sum */
    BIE_KERNEL_DIRECT_TC = 2,    /* K3 tensor-core block direct sum (incl. its Q packing) */
    BIE_KERNEL_COMBINE = 3,      /* K4+K5 partial reduction + BSR corrections + diagonal */
    BIE_KERNEL_KRYLOV = 4,       /* K7 orthogonalisation, Givens, updates */
    BIE_KERNEL_OTHER = 5,        /* right-hand sides, potentials, layout conversions */
    BIE_KERNEL_KINDS = 6
} bie_kernel_kind;

typedef struct {
    double ms;          /* summed device time of the launches */
    int64_t launches;   /* kernel launches */
    double pairs;       /* target-source pair interactions (direct sums) */
    double pair_cols;   /* pairs x right-hand-side columns (direct sums; padded columns for K3) */
    double bytes;       /* algorithmic bytes (combine: BSR values/indices + vectors) */
} bie_kernel_time;

/* Starts (enable = 1, counters reset) or stops (0) event timing of the handle's launches. */
int bie_profile_enable(bie_geom* g, int enable);
/* Reads the accumulated figures of one kernel kind (synchronises the stream). */
int bie_profile_read(bie_geom* g, int kind, bie_kernel_time* out);

/* Autotuned launch configuration of a direct-sum family on this geometry: family 0 =
 * tensor-core block sum (columns = min(k, 128), pieces 2 or 3), 1 = FP64 tensor-core
 * sum (columns = min(k, 64), pieces 0). The library times a few candidate launch
 * shapes (CTA shape, source split count) on the first application of each family and
 * kernel instance (widths rounded up to a multiple of 16 for family 0, to 8, 16, 32 or 64
 * for family 1, so every width of an instance reads the same entry) and keeps the
 * fastest (environment variable BIE_NO_AUTOTUNE turns this
 * off). Returns BIE_EINVAL when nothing was tuned for the key. No counterpart in the
 * reference (its FMM has no launch shapes). */
int bie_tuning_read(bie_geom* g, int32_t family, int32_t columns, int32_t pieces, int32_t* nsplit,
                    int32_t* ctas_per_sm, double* ms);

/* Arithmetic-throughput probes of a device, the compute ceilings of the direct sums:
 * which = 0 FP32 FMA, 1 FP32 FMA issued as packed f32x2 pairs, 2 MUFU reciprocal
 * square root (FP32), 3 FP64 FMA, 4 FP64 tensor-core MMA (mma.sync m8n8k4), 5 FP32 pair to
 * packed bf16x2 conversion (cvt.rn.bf16x2.f32); 6 and 7: latency of a dependent chain of
 * FP64 tensor-core MMAs (6) or FP64 FMAs (7), one warp; 8: FP64 MMAs and FP64 FMAs at once
 * (half the warps each, a quarter of probes 4 and 3's work each; *per_second = the MMA
 * flop rate, *ms = the launch), to show whether the two share throughput.
 * *per_second = lane operations per second for 0-3 and 5 (a packed f32x2 FMA counts as two),
 * flops per second for 4, and SM cycles per operation for 6 and 7 (the "per second" name
 * notwithstanding); *ms = duration of the timed launch (about 10 ms; 0 for 6 and 7).
 * No counterpart in the reference. */
int bie_peak_probe(int32_t device, int32_t which, double* per_second, double* ms);

/* ---- request server: the serving loop around the block solve -------------------
 * Requests of solve_dielectric_box3d_block (src/solver/multi_rhs.jl:270-286) --
 * a geometry handle, an N x k block of right-hand sides and solver options -- are
 * queued and solved by max_slots worker threads with continuous batching: a slot
 * takes the oldest request whose geometry is idle and whose device workspace fits
 * the HBM budget, merged with later queued requests for the same geometry and
 * options (up to max_batch_rhs columns) into one block solve; batches on different
 * geometries run concurrently on their geometries' streams. A geometry handle given
 * to a server must not be used by other calls until its requests are polled. */
typedef struct bie_server bie_server;

typedef struct {
    int max_slots;       /* block solves in flight at once (default 4) */
    int max_batch_rhs;   /* columns merged into one block solve (default 128, <= 256) */
    double hbm_fraction; /* admission budget: this fraction of the device's free memory at creation (0.8) */
    int device;          /* CUDA device of the budget (the geometries carry their own) */
    int max_group;       /* point-source batches of up to this many different geometries of at most
                            24,576 nodes (same options, split-BF16 precision, <= 128 columns each) run as
                            one group solve (bie_solve_group_device) in one slot (default 8; 1 = one
                            geometry per slot) */
} bie_server_opts;

typedef struct {
    int64_t submitted, completed, batches, merged_requests, queued;
    int inflight, peak_inflight;
    int64_t hbm_budget, hbm_in_use, hbm_peak; /* bytes of estimated solver workspace */
    int64_t workspace_releases; /* batches after which their geometry's workspace was released */
    int64_t enomem_retries;     /* batches retried after a device allocation failed */
    int64_t groups;             /* group solves (two or more geometries in lockstep) */
    int64_t grouped_batches;    /* batches that ran inside a group solve */
} bie_server_counters;

void bie_server_opts_default(bie_server_opts* o);
int bie_server_create(const bie_server_opts* o, bie_server** out);
/* Copies F (host, N x k column-major) and queues the solve; *ticket identifies it. */
int bie_server_submit(bie_server* s, bie_geom* g, const double* F, int32_t k, const bie_solve_opts* o,
                      uint64_t* ticket);
/* Queues a block solve of point-source right-hand sides, rhs_dielectric_box3d(itf,
 * PointSource(src[:, c], q[c]), eps_src[c]) (src/solver/dielectric_box3d.jl:95-104): only the
 * 5 k source values are copied; the right-hand sides are built on the device when the batch
 * runs (as bie_solve_point does), so a queue of many requests holds no N x k host blocks.
 * Point-source requests merge with each other, not with bie_server_submit's. src 3 x k. */
int bie_server_submit_point(bie_server* s, bie_geom* g, const double* src, const double* q, const double* eps_src,
                            int32_t k, const bie_solve_opts* o, uint64_t* ticket);
/* Waits up to timeout_ms (< 0: until done) for the request. *done = 1 when finished:
 * Sigma (host N x k, may be NULL), stats and the submit-to-completion latency are
 * filled, the ticket is retired and the solve's status is returned (BIE_ENOCONV
 * included); *done = 0 and BIE_OK while it is still queued or running. */
int bie_server_poll(bie_server* s, uint64_t ticket, int32_t timeout_ms, double* Sigma, bie_stats* st,
                    double* latency_ms, int* done);
int bie_server_counters_read(bie_server* s, bie_server_counters* out);
/* Stops the slots after their current batches; queued requests are dropped. */
void bie_server_destroy(bie_server* s);

#ifdef __cplusplus
}
#endif
#endif /* BIE_B200_H */
