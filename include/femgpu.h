/* femgpu: the fh-fem iterative solve path of femahoy on one B200 (sm_100a), behind a C ABI.
 *
 * Each entry point replaces one interface of the Rust crate `fh-fem` (crates/fem/src in the
 * femahoy project); the comment above it cites the item it replaces. Plain pointers and sizes
 * only. Functions ending in `_device` take device pointers (CUDA global memory on the current
 * device); all others take host pointers. Every function returns FEMGPU_OK (0) or a status
 * code below; femgpu_last_error() gives the message, with the reference's text where the
 * reference has one ("cancelled", "conjugate gradients did not converge: ...", "the matrix is
 * not positive definite: ...", "multigrid needs the box grid: ...").
 *
 * Threading: a handle is used from one host thread at a time (as the reference's `Solver`,
 * which is Send + Sync but solves synchronously). Different handles may be used from
 * different threads; each handle owns its CUDA stream.
 */
#ifndef FEMGPU_H
#define FEMGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. Each maps one-to-one onto an error string of the reference. */
enum {
    FEMGPU_OK = 0,
    FEMGPU_ERR_CANCELLED = 1,      /* "cancelled" (multigrid.rs:735-737) */
    FEMGPU_ERR_NOT_CONVERGED = 2,  /* "conjugate gradients did not converge: ..." (multigrid.rs:729-733) */
    FEMGPU_ERR_NOT_SPD = 3,        /* "the matrix is not positive definite: ..." (cholesky.rs:92-99) */
    FEMGPU_ERR_NEEDS_GRID = 4,     /* "multigrid needs the box grid: ..." (solve.rs:133-138) */
    FEMGPU_ERR_INVALID = 5,        /* an argument out of range; the message names it */
    FEMGPU_ERR_CUDA = 6,           /* a CUDA runtime error; the message names the call site */
    FEMGPU_ERR_TOO_LARGE = 7,      /* a size above a documented limit of this library */
    FEMGPU_ERR_PATTERN = 8,        /* "the pattern holds each element pair" (sparse.rs:80-82) */
    FEMGPU_ERR_MATERIAL = 9,       /* hex.rs:72-98: the moduli or Poisson ratios give no material */
    FEMGPU_ERR_TIMEOUT = 10        /* a device-side wait ran out of its iteration limit */
};

/* Element kinds of the assembly. */
enum {
    FEMGPU_P1_HEAT = 0,    /* 4-node tet, 4 x 4 conduction V G^T K G (heat.rs:972-1002) */
    FEMGPU_P1_ELASTIC = 1, /* 4-node tet, 12 x 12 V B^T D B (this library's own element) */
    FEMGPU_P2_ELASTIC = 2, /* 10-node tet, 30 x 30, 4-point rule (tet10.rs:90-120) */
    FEMGPU_P2_MASS = 3,    /* 10-node tet consistent mass, 30 x 30 (tet10.rs:173-212), coef = the
                              density per element, as modes.rs:470-476; gather mode only */
    FEMGPU_P2_ELASTIC_ORTHO = 4, /* as FEMGPU_P2_ELASTIC with an orthotropic material per
                                    element (Orthotropic::stiffness, hex.rs:69-117): coef = E_x,
                                    E_y, E_z, nu_xy, nu_xz, nu_yz, G_xy, G_xz, G_yz; gather
                                    mode only */
    FEMGPU_HEX8_HEAT = 5, /* box cell of the grid, 8 corners in VTK order, 8 x 8 conduction
                             (heat.rs:1246-1273) as heat.rs:820-826 assembles it; coef = the 3
                             conductivities; the sides are corner 6 minus corner 0; gather mode
                             only */
    FEMGPU_HEX8_ELASTIC = 6, /* box cell of the grid, 8 corners in VTK order: the 24 x 24
                               stiffness of the 8-node hex with its 9 incompatible modes condensed
                               (Hex::new, hex.rs:218-297), as elastic.rs:386-391 assembles it;
                               coef = the 9 orthotropic constants of FEMGPU_P2_ELASTIC_ORTHO; the
                               sides are corner 6 minus corner 0 (above 0); unknown 3 node +
                               component; gather mode only */
    FEMGPU_HEX8_MASS = 7 /* box cell of the grid: the consistent mass of its 8 corners
                            (hex::mass, hex.rs:337-353), coef = the density per cell, as
                            modes.rs:363-370 assembles it; gather mode only */
};

/* Assembly modes. */
enum {
    FEMGPU_ASSEMBLE_GATHER = 0, /* each row sums its element terms in increasing element order:
                                   bit-identical with Csr::add_element (sparse.rs:75-86) */
    FEMGPU_ASSEMBLE_COLOUR = 1  /* elements scattered colour by colour, no atomics: the same
                                   terms summed in colour order (a few ulp apart) */
};

/* Solver methods (solve.rs:47-50). -1 lets the crossover choose. */
enum { FEMGPU_METHOD_NONE = -1, FEMGPU_METHOD_DIRECT = 0, FEMGPU_METHOD_MULTIGRID = 1 };

/* Precision of the iterative solve. */
enum {
    FEMGPU_FP64 = 0,  /* plain form: FP64 operator, V-cycle and PCG (Hestenes-Stiefel, as
                         multigrid.rs:692-753) */
    FEMGPU_MIXED = 1  /* FP32 V-cycle (values FP32, indices int32) inside FP64 flexible CG; the
                         outer residual, dots, scalars, update and coarse factor stay FP64 */
};

typedef struct femgpu_csr femgpu_csr;       /* a device-resident square CSR matrix */
typedef struct femgpu_solver femgpu_solver; /* solve.rs:58-61 `Solver` */

/* The message of the last failure of this host thread. */
size_t femgpu_last_error(char* buf, size_t len);
/* The library version and the device it runs on. */
const char* femgpu_version(void);

/* ---------------------------------------------------------------- assembly */

/* Csr::pattern + Csr::add_element over all elements (sparse.rs:22-86), as called by
 * heat.rs:920-927 (P1 heat), elastic_tet.rs:183-193 (P2 elasticity, unknown 3 node + component)
 * and for P1 elasticity. `xyz` holds 3 coordinates per point; `nodes` 4 (P1) or 10 (P2) point
 * numbers per element; `coef` 3 conductivities (P1 heat) or E and nu (elasticity) per
 * element. The result is the full matrix on the device: n = points (heat) or 3 points. */
int femgpu_assemble(int kind, int mode, size_t npoints, const double* xyz, size_t nel,
                    const uint32_t* nodes, const double* coef, femgpu_csr** out);
int femgpu_assemble_device(int kind, int mode, size_t npoints, const double* xyz, size_t nel,
                           const uint32_t* nodes, const double* coef, femgpu_csr** out);

/* Csr::pattern alone (sparse.rs:22-65) for `nel` elements of `m` nodes each. */
int femgpu_pattern(size_t n, size_t nel, int m, const uint32_t* elements, femgpu_csr** out);

/* Element colouring for the colour-ordered scatter: elements that share a node get different
 * colours (Jones-Plassmann with a fixed hash priority; deterministic). No reference
 * counterpart: the reference assembles sequentially (sparse.rs:75). */
int femgpu_colour(size_t n, size_t nel, int m, const uint32_t* elements, uint32_t* colour,
                  int* ncolours);

/* Quadratic::new (tet10.rs:244-272): the 10 points of each tetrahedron, the edge points
 * numbered from `ncorner` in the order of first sight. `tets10` holds 10 * ntet values and
 * `edges` 2 * (6 * ntet) values; `nedges` gets the edge count. */
int femgpu_quadratic(size_t ncorner, size_t ntet, const uint32_t* tets, uint32_t* tets10,
                     uint32_t* edges, size_t* nedges);

/* The matrix's size and entries; its CSR arrays (ptr n + 1, idx nnz, val nnz) to host. */
int femgpu_csr_info(const femgpu_csr* a, size_t* n, size_t* nnz);
int femgpu_csr_download(const femgpu_csr* a, int64_t* ptr, uint32_t* idx, double* val);
/* A device matrix from host CSR arrays (the Rust `Csr` handed to Solver::new). */
int femgpu_csr_upload(size_t n, const int64_t* ptr, const uint32_t* idx, const double* val,
                      femgpu_csr** out);
/* Csr::diagonal (sparse.rs:88-93): the n diagonal entries (0 where a row has none). */
int femgpu_csr_diagonal(const femgpu_csr* a, double* d);

/* Rect (sparse.rs:196-293), a rectangular CSR matrix such as a prolongation, on the device:
 * y = P x (mul, sparse.rs:212-220) and y = P^T x (mul_transpose, :223-230), each output summed
 * in the reference's order (bit-identical), and the Galerkin product P^T A P (galerkin,
 * :233-292; its entries the reference's to rounding, its pattern the same). `ptr` starts at 0
 * and does not decrease; every column is below `cols`. */
typedef struct femgpu_rect femgpu_rect;
int femgpu_rect_upload(size_t rows, size_t cols, const int64_t* ptr, const uint32_t* idx,
                       const double* val, femgpu_rect** out);
int femgpu_rect_mul(femgpu_rect* r, const double* x, double* y);
int femgpu_rect_mul_transpose(femgpu_rect* r, const double* x, double* y);
int femgpu_rect_galerkin(const femgpu_rect* r, const femgpu_csr* a, femgpu_csr** out);
void femgpu_rect_free(femgpu_rect* r);

/* Csr::submatrix (sparse.rs:108-135): rows and columns `keep` (each index once). */
int femgpu_csr_submatrix(const femgpu_csr* a, const int64_t* keep, size_t nkeep,
                         femgpu_csr** out);
/* Csr::mul (sparse.rs:96-105): y = A x, host vectors. */
int femgpu_csr_mul(const femgpu_csr* a, const double* x, double* y);
/* heat::reduced_rhs (heat.rs:1219-1244, steady form): load - A t over the fixed columns, for
 * the free rows `free` (increasing). Host vectors; `out` holds nfree values. */
int femgpu_reduced_rhs(const femgpu_csr* a, const double* load, const double* t,
                       const int64_t* free, size_t nfree, double* out);
void femgpu_csr_free(femgpu_csr* a);

/* The largest matrix (rows) that femgpu_reduced_rhs_noalloc takes. */
#define FEMGPU_NOALLOC_MAX_ROWS 4194304

/* femgpu_reduced_rhs for callers that cannot allocate device memory. No counterpart in the
 * reference: it is this library's own addition.
 *
 * Some callers must not call cudaMalloc or cudaFree: code that shares the GPU with other work in
 * flight (a loop serving many solves on several streams) would be stalled by cudaFree, which
 * waits for the whole device, and code whose device memory is held by its own pool allocator
 * cannot count on a new allocation succeeding. This entry point allocates nothing: every pointer
 * is a device pointer owned by the caller (the CSR arrays of the n x n matrix: ptr n + 1, idx and
 * val ptr[n]; load and t n values; free nfree increasing rows; out nfree values), and its only
 * scratch, a row-to-place map, is a fixed array inside the library of FEMGPU_NOALLOC_MAX_ROWS
 * entries (16 MiB held on every GPU that loads the library until the process exits). A larger n
 * fails with FEMGPU_ERR_TOO_LARGE. The result is the allocating entry point's, bit for bit.
 *
 * `stream` is a cudaStream_t (null: the default stream). The call queues its work on `stream`,
 * then synchronizes `stream` to read its argument checks (free rows in 0..n, increasing, each
 * once; the column indices of the free rows in 0..n; else FEMGPU_ERR_INVALID), so `out` is
 * written when it returns, and it cannot be made while `stream` is being captured. The first
 * call on each device also looks up the scratch's device address. All calls share the scratch,
 * which keeps the last call's contents (each call clears what it uses); calls whose work
 * overlaps on the GPU race on it, so order them on one stream, or synchronize the previous
 * call's stream before calling on another. */
int femgpu_reduced_rhs_noalloc(size_t n, const int64_t* ptr, const uint32_t* idx,
                               const double* val, const double* load, const double* t,
                               const int64_t* free, size_t nfree, double* out, void* stream);

/* pmultigrid::prolongation (pmultigrid.rs:104-151): P from the free corner unknowns to the
 * free unknowns of a quadratic mesh. Two calls: with null outputs it writes the sizes
 * (`nnz`, `ncoarse`); then the CSR arrays of P (rows = nfree) and the coarse points (3 each). */
int femgpu_prolongation(size_t npoints, const double* points, size_t corners, size_t nedges,
                        const uint32_t* edges, size_t nfree, const int64_t* free, size_t* nnz,
                        size_t* ncoarse, int64_t* p_ptr, uint32_t* p_idx, double* p_val,
                        double* coarse_xyz);

/* ---------------------------------------------------------------- solver */

/* solve.rs:64-77 `Unknowns`. */
enum { FEMGPU_UNKNOWNS_GRID = 0, FEMGPU_UNKNOWNS_POINTS = 1, FEMGPU_UNKNOWNS_QUADRATIC = 2 };

typedef struct femgpu_unknowns {
    int kind;
    /* GRID (multigrid.rs:55-59 `Level`): the planes of each axis, and the grid point (3 values)
     * and component of each unknown. */
    const double* planes[3];
    size_t nplanes[3];
    const uint32_t* points;
    const uint8_t* comp;
    /* POINTS and QUADRATIC: the coordinates of each unknown (3 values each). */
    const double* xyz;
    /* QUADRATIC: the prolongation P (rows = unknowns, cols = coarse unknowns) and the point of
     * each coarse unknown; `coarse_comp` (optional, may be null) gives the component of each
     * coarse unknown, else it is inferred from the order of the unknowns at each point. */
    size_t p_cols;
    const int64_t* p_ptr;
    const uint32_t* p_idx;
    const double* p_val;
    const double* coarse_xyz;
    const uint8_t* coarse_comp;
} femgpu_unknowns;

/* solve.rs:28-39 `Crossover`: rule 0 = Unknowns(unknowns); 1 = Flops{flops, entries, flat} (the
 * sparse factor's figures of femgpu_symbolic_counts). A direct choice is solved directly: by a
 * dense inverse up to 4,096 unknowns, by the sparse multifrontal factor above. */
typedef struct femgpu_crossover {
    int rule;
    size_t unknowns;
    double flops;
    uint64_t entries;
    int flat;
} femgpu_crossover;

/* Options of this library (no reference counterpart; zeros pick the defaults). */
typedef struct femgpu_options {
    int precision;        /* FEMGPU_FP64 or FEMGPU_MIXED */
    int degree;           /* Chebyshev degree of each pre- and post-smoothing; 0 = autotuned:
                             1, 2 or 3 on every level, or 2 on the finest and 1 on the coarser
                             ones, by timed trial solves (device time per decade of residual
                             reduction), once per size class (the finest level's kind and
                             log2 rows, the level count, the precision) and kept for the process;
                             a batch takes 2 */
    double lower;         /* Chebyshev interval lower end as a fraction of lambda_max; 0 = default */
    int sell_c;           /* SELL chunk height (rows per slice; a warp reads 32 rows): 0 =
                             autotuned, 16, 32 or 64 by timing each level's product, once per
                             size class (log2 rows, entries per row, element size); or 8, 16,
                             32, 64 */
    int sell_sigma;       /* SELL sorting window in rows: 0 = autotuned */
    int coarsest;         /* the largest level that the dense coarse solve takes; 0 = 5000 (the
                             reference's COARSEST is 3000, multigrid.rs:94; the dense inverse
                             on the device takes 1 level more and the box grids measured
                             converge in 1 iteration less) */
    int max_levels;       /* 0 = 30 (multigrid.rs:94) */
    int graph;            /* 1 = replay each PCG iteration as a CUDA graph (default), 2 = off */
    int format;           /* 0 = a symmetric stencil for each level whose entries sit at a few
                             constant column offsets (box grids in grid order), SELL-C for the
                             others; 1 = SELL-C for every level */
    int tail;             /* > 0: the levels of at most this many rows, and the coarsest solve,
                             run as 1 cooperative kernel with a grid-wide barrier between steps;
                             0 (default) = every step its own launch (faster on B200 for the
                             box grids measured) */
    int launch;           /* 0 = each kernel of a PCG iteration may start while the one before
                             it drains, waiting on the device for its results (programmatic
                             dependent launch; default); 1 = plain stream-ordered launches */
    int values;           /* the mixed form's stencil levels: 0 = the default, 1 = FP32
                             coefficients, 2 = FP16 coefficients scaled by the level's largest
                             (the products read about 0.6 of the bytes; the V-cycle changes by
                             about 2^-11 relative); 3 = FP32 coefficients and the coarsest
                             level's dense inverse in FP16 scaled by its largest entry (its
                             product reads half the bytes, sums in FP32) */
    int tiles;            /* the mixed form's finest stencil level (K = 8): 0 = the autotuner
                             chooses by timing whether its smoothing steps and residuals stream
                             each tile's own arrays into shared memory by bulk copies or read
                             them directly; 1 = directly; 2 = bulk copies (the same bits) */
    int axes;             /* the axes that the grid coarsening halves (bit 0 x, 1 y, 2 z; 0 = all,
                             the reference's rule): 4 coarsens only z, for meshes extruded in
                             layers from an unstructured footprint, whose points are on z planes
                             but not on x or y planes (prism.rs) */
    int stencil;          /* the product kernel of the stencil levels (K = 8 or 14): 0 = the
                             autotuner's choice by timing, once per size class; 1 = K read at run
                             time, 2 = K known at compile time, 3 = 2 adjacent rows per thread,
                             4 = marching planes (every gather from shared memory). A kernel that
                             a level cannot take falls back to the next lower one. All give the
                             same bits. */
    int smoother;         /* the Chebyshev smoother's polynomial: 0 or 4 = the fourth kind on
                             [0, 1.1] lambda_max (Lottes 2023; the default), 1 = the first kind
                             on [lower, 1.1] lambda_max */
    int cluster;          /* the levels of at most 65,536 rows (stencil or SELL) after the first:
                             1 = each leg of the cycle there (the pre-smoothing steps, residual
                             and restriction; the prolongation and the post-smoothing steps) as 1
                             launch of 1 thread-block cluster with cluster barriers between
                             steps, where the device schedules clusters of 16 or 8 blocks;
                             0 (default) = a launch per step (the same bits; faster on B200 for
                             the box grids measured) */
    int l2;               /* 1 = keep the coarsest level's dense inverse resident in L2 (a
                             persisting access window on its product; the process's persisting
                             L2 limit is raised to the inverse's size, at most the device's
                             maximum); 0 (default) = plain loads */
    double upper;         /* the Chebyshev interval's upper end as a multiple of the power
                             method's lambda_max; 0 = 1.1 */
} femgpu_options;

/* solve.rs:81-86 `Stats`, plus the true residual |b - A x| / |b| computed in FP64 at the end
 * (the reference reports the recurrence residual for PCG and the true one for Cholesky). */
typedef struct femgpu_stats {
    size_t iterations;
    double residual;       /* the reference's definition for the method that ran */
    double true_residual;  /* |b - A x|_2 / |b|_2 in FP64 on the device */
    double seconds;        /* device time of the solve (CUDA events) */
    size_t launches;       /* kernels this library launched for the solve */
} femgpu_stats;

/* multigrid.rs:62-68 `Cells`: the box cells of a displacement model on grid unknowns, each by
 * its lowest grid point `origin` (3 values per cell) and its 24 x 24 matrix (row-major, unknown
 * 3 n + c for corner n in VTK order and component c), given by class: cell i has the matrix
 * matrices + 576 cls[i] (a per-cell table is cls[i] = i). The reference's `element` closure
 * gives Hex::new per cell (elastic.rs:499-521); femgpu_hex_elements makes the class matrices. */
typedef struct femgpu_cells {
    size_t count;
    const uint32_t* origin;
    const uint32_t* cls;
    const double* matrices;
    size_t nclass;
    /* femgpu_modes_cells only: the consistent mass of each class (576 values each, the same
     * classes; hex::mass, hex.rs:337-353), for the cells of K - shift M (modes.rs:394-401). */
    const double* mass;
} femgpu_cells;

/* Solver::new (solve.rs:92-183) with `cells` = None. The solver keeps a copy of `a` on the
 * device (the reference moves `a` in). `a` may be freed after the call. */
int femgpu_solver_new(const femgpu_csr* a, const femgpu_unknowns* unknowns, int method,
                      const femgpu_crossover* crossover, const femgpu_options* options,
                      femgpu_solver** out);
/* Solver::new with `cells` (may be null): grid unknowns whose multigrid coarse matrices come
 * from the cells (multigrid.rs:107-119, 458-608) instead of the Galerkin products. The cell
 * arrays may be freed after the call. */
int femgpu_solver_new_cells(const femgpu_csr* a, const femgpu_unknowns* unknowns, int method,
                            const femgpu_crossover* crossover, const femgpu_options* options,
                            const femgpu_cells* cells, femgpu_solver** out);
/* Hex::new (hex.rs:218-297) of `count` box cells on the device: `keys` holds 12 values per cell
 * (its 3 sides, then the 9 orthotropic constants of FEMGPU_P2_ELASTIC_ORTHO); `matrices` gets
 * the condensed 24 x 24 stiffness of each (576 values, row-major), bit-identical with the
 * reference's. */
int femgpu_hex_elements(size_t count, const double* keys, double* matrices);
/* hex::mass (hex.rs:337-353) of `count` box cells on the host: `sizes` 3 per cell, `density` 1
 * per cell; `out` gets 576 values per cell, bit-identical with the reference's. */
int femgpu_hex_mass(size_t count, const double* sizes, const double* density, double* out);
/* The entries (with the diagonal) and the floating point operations of the sparse Cholesky
 * factor of `a` in the nested dissection order of the unknowns' points (order.rs:19-198,
 * symbolic.rs:41-183): the figures Crossover::Flops compares (solve.rs:108-118, 160-172), which
 * femgpu_solver_new applies. No reference counterpart as an entry point: for checking the
 * crossover. */
int femgpu_symbolic_counts(const femgpu_csr* a, const femgpu_unknowns* unknowns,
                           uint64_t* entries, double* flops);
/* The matrix of multigrid level `level` (>= 1) that the solver of (a, unknowns, cells) forms
 * (cells may be null: the Galerkin products), `level` coarsenings regardless of the size limits.
 * The coarse unknowns are numbered in grid order (z, then y, then x, then the component); the
 * reference numbers the same unknowns in the order it first meets them (multigrid.rs:329-452).
 * `points` (3 plane indices per unknown) and `comp` (may be null) give each coarse unknown's
 * grid point and component. Two calls: with null arrays it writes n and nnz; then the CSR
 * arrays. No reference counterpart: for checking the hierarchy against the reference. */
int femgpu_coarse_matrix(const femgpu_csr* a, const femgpu_unknowns* unknowns,
                         const femgpu_cells* cells, int level, size_t* n, size_t* nnz,
                         int64_t* ptr, uint32_t* idx, double* val, uint32_t* points,
                         uint8_t* comp);
/* The polls of each bounded wait of the device (the mbarrier waits for the bulk copies of the
 * stencil tile kernels, femgpu_options.tiles) before the solve gives up with
 * FEMGPU_ERR_TIMEOUT; FEMGPU_WAIT_LIMIT_DEFAULT by default. A wait that runs out ends the solve
 * with the solver still usable. No reference counterpart: the failure-detection knob of this
 * library's device waits (0 makes every such wait run out at once, for testing that path). */
#define FEMGPU_WAIT_LIMIT_DEFAULT 4194304u
int femgpu_solver_set_wait_limit(femgpu_solver* s, uint32_t polls);
/* Solver::with_max_iter (solve.rs:187-189). */
int femgpu_solver_set_max_iter(femgpu_solver* s, size_t max_iter);
/* The relative residual of each PCG solve; PCG_TOL = 1e-10 (solve.rs:42) by default. */
int femgpu_solver_set_tol(femgpu_solver* s, double tol);
/* Solver::method (solve.rs:191-196). */
int femgpu_solver_method(const femgpu_solver* s);
/* The number of unknowns of each level (levels[0] = n); returns the level count. */
int femgpu_solver_levels(const femgpu_solver* s, size_t* sizes, int cap);
/* A text description of the solver (method, precision, and for each level its size, storage
 * format and the kernel variant the autotuner chose); returns the full length. No reference
 * counterpart. */
size_t femgpu_solver_describe(const femgpu_solver* s, char* buf, size_t len);
/* Runs 1 PCG iteration with its kernels launched one by one and a CUDA event after each, and
 * writes the device time of each kernel as text (1 line each); returns the full length. The
 * solver's vectors are overwritten; solve again afterwards. No reference counterpart. */
size_t femgpu_solver_breakdown(femgpu_solver* s, char* buf, size_t len);
/* Device memory held by the solver, in bytes. */
size_t femgpu_solver_bytes(const femgpu_solver* s);
/* Solver::solve (solve.rs:199-250): solve A x = b; `x` holds the start value and gets the
 * solution. `cancel` (may be null) is read before each PCG iteration, as the reference's
 * `cancelled` closure; a non-zero value ends the solve with FEMGPU_ERR_CANCELLED. */
int femgpu_solver_solve(femgpu_solver* s, const double* b, double* x, const volatile int* cancel,
                        femgpu_stats* stats);
int femgpu_solver_solve_device(femgpu_solver* s, const double* b, double* x,
                               const volatile int* cancel, femgpu_stats* stats);
/* femgpu_solver_solve from the start value x = 0, as every steady caller of the reference
 * passes it (heat.rs:672, elastic.rs:561, elastic_tet.rs:329, dc.rs:270): `x` is only written,
 * so its start value is not copied to the device. */
int femgpu_solver_solve_zero(femgpu_solver* s, const double* b, double* x,
                             const volatile int* cancel, femgpu_stats* stats);
/* z = M^-1 r: 1 application of the preconditioner (a V-cycle), device vectors. */
int femgpu_solver_precondition_device(femgpu_solver* s, const double* r, double* z);

/* multigrid::pcg (multigrid.rs:692-753), the reference's public conjugate gradients with the
 * caller's preconditioner z = M^-1 r: from the start value x to |b - A x| <= tol |b| (tested
 * before each step), FEMGPU_ERR_NOT_CONVERGED after max_iter iterations and
 * FEMGPU_ERR_CANCELLED when *cancel is nonzero, with the reference's texts; x holds the last
 * iterate either way. `precondition` NULL: z = r. The vectors live on the device; A p is summed
 * row by row in column order (Csr::mul), the dot products in fixed blocks. femgpu_pcg: host
 * vectors, a host preconditioner (r and z host arrays of n values). femgpu_pcg_device: device
 * vectors b and x on `stream` (a cudaStream_t, NULL for the legacy stream), a preconditioner on
 * device vectors: r is complete when it is called, and z must be complete on `stream` when it
 * returns (work queued on `stream`, or finished), e.g. femgpu_solver_precondition_device. */
typedef struct femgpu_convergence {
    size_t iterations;
    double residual; /* |b - A x| / |b| at the end (multigrid.rs:680-686) */
} femgpu_convergence;
typedef void (*femgpu_precondition_fn)(const double* r, double* z, size_t n, void* ctx);
typedef void (*femgpu_precondition_device_fn)(const double* r, double* z, size_t n, void* stream,
                                              void* ctx);
int femgpu_pcg(const femgpu_csr* a, const double* b, double* x, femgpu_precondition_fn precondition,
               void* ctx, double tol, size_t max_iter, const volatile int* cancel,
               femgpu_convergence* out);
int femgpu_pcg_device(const femgpu_csr* a, const double* b, double* x,
                      femgpu_precondition_device_fn precondition, void* ctx, double tol,
                      size_t max_iter, const volatile int* cancel, void* stream,
                      femgpu_convergence* out);
void femgpu_solver_free(femgpu_solver* s);

/* The CUDA stream (a cudaStream_t) on which the solver launches all its work, so that a caller
 * can order its own work and CUDA events with it. No reference counterpart. */
void* femgpu_solver_stream(const femgpu_solver* s);
/* Times `reps` back-to-back launches of 1 kernel of the solve on the solver's stream with CUDA
 * events and the solve's launch attributes: which = 0 the finest Chebyshev smoothing step (on a
 * stencil level alternately on the level and on a second copy of its operator and vectors, so
 * that each launch finds its data evicted from L2, as in a solve), 1 the FP64 operator product
 * of PCG (fused with p.q). Writes the mean device time of a launch (ms) and the algorithmic
 * bytes of 1 launch (values, indices and vectors, each read or written once). No reference
 * counterpart. */
int femgpu_solver_kernel_time(femgpu_solver* s, int which, int reps, double* ms, double* bytes);

/* ---------------------------------------------------------------- serving */

/* A server of solve requests. No reference counterpart: the reference's callers solve 1 model
 * at a time (heat.rs:661-676, elastic_tet.rs:293-337). `slots` host threads each run 1 solve at
 * a time on its solver's own CUDA stream, so up to `slots` requests are on the device together
 * and a request that arrives while others run starts when a slot is free. The resident solvers
 * (operators and hierarchies, keyed by the caller's 64-bit key, e.g. a mesh id) count against
 * `budget_bytes` of device memory; idle ones are freed least recently used first when room is
 * needed. 1 solver runs 1 request at a time; requests for 1 key run in submission order. */
typedef struct femgpu_server femgpu_server;
int femgpu_server_new(int slots, size_t budget_bytes, femgpu_server** out);
/* Frees idle resident solvers until `bytes` more fit; FEMGPU_ERR_TOO_LARGE if the busy ones
 * leave no room. Call it before building a solver that the server is to hold. */
int femgpu_server_reserve(femgpu_server* s, size_t bytes);
/* Hands `solver` to the server under `key`; the server owns it from then on (do not free it).
 * On an error the caller keeps it. */
int femgpu_server_put(femgpu_server* s, uint64_t key, femgpu_solver* solver);
/* 1 if a solver is resident under `key`. */
int femgpu_server_has(femgpu_server* s, uint64_t key);
/* Queues Solver::solve (solve.rs:199) of the solver under `key`: b and the start value x are
 * host arrays that must stay valid until the ticket is waited for; x gets the solution. */
int femgpu_server_submit(femgpu_server* s, uint64_t key, const double* b, double* x,
                         uint64_t* ticket);
/* Waits for a ticket: its status (the solve's), stats, and the seconds from submission to the
 * end of the solve. */
int femgpu_server_wait(femgpu_server* s, uint64_t ticket, femgpu_stats* stats, double* latency_s);
size_t femgpu_server_resident_bytes(femgpu_server* s);
size_t femgpu_server_resident_count(femgpu_server* s);
void femgpu_server_free(femgpu_server* s);

/* ---------------------------------------------------------------- batches */

/* Many small systems, each with `nrhs` right sides, solved together. No reference counterpart:
 * the reference's callers solve 1 model at a time; each (system, right side) pair, a segment,
 * is the reference's PCG with the multigrid V-cycle (multigrid.rs:692-753) with its own
 * scalars and stopping test. Each system keeps its own hierarchy (multigrid.rs:84-139, down to
 * `options->coarsest` unknowns, 1024 when 0) and the systems' levels are combined into
 * block-diagonal operators, so 1 launch of each kernel serves all systems; the loop is 1 CUDA
 * graph on the device. Vectors hold the right sides interleaved: value (row, k) of system s is
 * at (offsets[s] + row) * nrhs + k, offsets from femgpu_batch_systems. */
typedef struct femgpu_batch femgpu_batch;

typedef struct femgpu_batch_stats {
    size_t max_iterations;    /* the most iterations of a segment */
    double mean_iterations;
    double max_residual;      /* the largest recurrence residual |r| / |b| of a segment */
    double max_true_residual; /* the largest |b - A x| / |b| in FP64 of a segment */
    double seconds;           /* device time of the solve (CUDA events) */
    size_t launches;          /* kernels this library launched for the solve */
    size_t not_converged;     /* segments that hit the iteration limit or broke down */
    size_t restarts;          /* restarts from x of the segments whose true residual drifted */
} femgpu_batch_stats;

/* `count` systems with grid unknowns (FEMGPU_UNKNOWNS_GRID; else FEMGPU_ERR_NEEDS_GRID);
 * nrhs = 1, 4 or 16. Honours options->precision, degree, lower, coarsest and max_levels. */
int femgpu_batch_new(int count, const femgpu_csr* const* a, const femgpu_unknowns* unknowns,
                     int nrhs, const femgpu_options* options, femgpu_batch** out);
int femgpu_batch_set_tol(femgpu_batch* b, double tol);           /* default PCG_TOL, 1e-10 */
int femgpu_batch_set_max_iter(femgpu_batch* b, size_t max_iter); /* default PCG_MAX_ITER, 500 */
/* The number of systems; `offsets` (may be null) gets count + 1 row offsets. */
int femgpu_batch_systems(const femgpu_batch* b, size_t* offsets);
/* The number of levels; `sizes` (may be null) gets the combined unknowns of each. */
int femgpu_batch_levels(const femgpu_batch* b, size_t* sizes);
/* The batch's setup seconds by phase ("setup seconds: phase s; ..."), as much as fits in `len`
 * bytes with the terminating 0. No reference counterpart. */
int femgpu_batch_describe(const femgpu_batch* b, char* buf, size_t len);
/* Solves every segment from the start value in x (host arrays of rows * nrhs values). A segment
 * that hits the iteration limit or breaks down makes the call return FEMGPU_ERR_NOT_CONVERGED
 * naming the first such segment, with every x written; femgpu_batch_segments tells which. */
int femgpu_batch_solve(femgpu_batch* b, const double* rhs, double* x, const volatile int* cancel,
                       femgpu_batch_stats* stats);
/* As femgpu_batch_solve on device arrays, on the batch's stream. */
int femgpu_batch_solve_device(femgpu_batch* b, const double* rhs, double* x,
                              const volatile int* cancel, femgpu_batch_stats* stats);
/* Per segment (system s, right side k at s * nrhs + k) of the last solve: iterations, true and
 * recurrence residuals, status (0 converged, 1 iteration limit, 2 broke down). Any may be null. */
int femgpu_batch_segments(const femgpu_batch* b, size_t* iterations, double* true_residual,
                          double* residual, int* status);
/* Times `reps` back-to-back launches of the finest level's Chebyshev step over all right sides
 * on the batch's stream (CUDA events); writes the mean device time of a launch (ms) and its
 * algorithmic bytes (values and indices once; b, x, d read, d, x written per right side). The
 * level's work vectors are overwritten. No reference counterpart. */
int femgpu_batch_kernel_time(femgpu_batch* b, int reps, double* ms, double* bytes);
size_t femgpu_batch_bytes(const femgpu_batch* b);
void* femgpu_batch_stream(const femgpu_batch* b);
void femgpu_batch_free(femgpu_batch* b);

/* Continuous batching over a batch's systems. No reference counterpart: the reference's
 * callers solve 1 model at a time; serving many requests for resident meshes is this library's.
 * femgpu_stream_new turns a batch into a server of single right sides: each system has `nrhs`
 * slots; a request (1 right side of 1 system, x from 0) waits until a slot of its system is
 * free and is then admitted by the running device loop at its next PCG iteration, while the
 * other slots' solves go on; a finished slot's solution (after its true residual, and restarts
 * from x for the mixed form as in femgpu_batch_solve) is written back and the slot takes the
 * next request at once. The loop is the batch's CUDA-graph-captured PCG with the multigrid
 * V-cycle, 1 launch that runs while any slot is busy; its right sides come in and its solutions
 * go out through pinned, mapped host memory. Every request's result is the same bit for bit
 * whatever else is in the loop (each slot's arithmetic reads only its own data), and equals
 * femgpu_batch_solve's for the same right side from x = 0. While a stream is open, the batch's
 * own solves refuse; a batch serves 1 stream in its life. rhs and x hold the system's rows in
 * its own order (femgpu_batch_systems). */
typedef struct femgpu_stream femgpu_stream;
typedef struct femgpu_stream_result {
    size_t iterations;
    double residual;       /* |r| / |b| of the recurrence */
    double true_residual;  /* |b - A x| / |b| in FP64 */
    int status;            /* 0 converged, 1 iteration limit, 2 broke down */
    double latency_s;      /* from submission to the solution's arrival on the host */
} femgpu_stream_result;
int femgpu_stream_new(femgpu_batch* b, femgpu_stream** out);
int femgpu_stream_submit(femgpu_stream* s, int system, const double* rhs, uint64_t* ticket);
/* Waits for a request: x gets its solution; the reference's texts for the iteration limit. */
int femgpu_stream_wait(femgpu_stream* s, uint64_t ticket, double* x, femgpu_stream_result* result);
/* The device loop's iterations so far, and the slots they served summed over them (their ratio
 * is the mean number of requests packed into 1 iteration). */
int femgpu_stream_counts(femgpu_stream* s, size_t* loops, size_t* served_iterations);
void femgpu_stream_free(femgpu_stream* s);

/* ---------------------------------------------------------------- transient heat */

/* The backward-Euler loop of a transient heat model with lumped capacity (heat.rs:686-733): 1
 * operator, K + C/dt on the free points, solved once per time step from the last temperatures.
 * The matrix, its solver and the vectors stay on the device for the whole run. */
typedef struct femgpu_transient femgpu_transient;

/* The energy terms of heat.rs:535-547 that the loop forms, for a step with no radiation:
 * stored = sum of the rates C (T - T_prev) / dt; fixed = sum over the fixed points of
 * q = (K T)_i + rate_i - load_i; gross = sum of |rate| and |q|. The caller adds its own source,
 * flux and convection terms. Summed on the device in a fixed order (deterministic; not the
 * reference's point order, so they agree to rounding). */
typedef struct femgpu_energy {
    double stored;
    double fixed;
    double gross;
} femgpu_energy;

/* heat.rs:688-703: `k` the full conductivity matrix (femgpu_assemble, P1 heat), `capacity` the
 * lumped capacity of each point, `dt` the step, `free` the free points (increasing) and
 * `unknowns` their grid level, as for femgpu_solver_new (whose method, crossover and options
 * these are). A NULL crossover is Unknowns(40000), the reference's TRANSIENT_DIRECT_LIMIT
 * (solve.rs:24). */
int femgpu_transient_new(const femgpu_csr* k, const double* capacity, double dt,
                         const int64_t* free, size_t nfree, const femgpu_unknowns* unknowns,
                         int method, const femgpu_crossover* crossover,
                         const femgpu_options* options, femgpu_transient** out);
/* The solver of the loop, for femgpu_solver_set_tol / _set_max_iter / _describe. It belongs to
 * the transient handle. */
femgpu_solver* femgpu_transient_solver(femgpu_transient* t);
/* heat.rs:709-733 for `steps` steps: `temperature` (n) holds the start values (the fixed points
 * keep theirs) and gets the last step's; `load` (n) is the constant load of each point. The
 * steps s with s % output_every == 0 or s == steps write their temperatures to `frames`
 * (n each, in order; NULL skips them) and their energies to `energies` (NULL skips them).
 * "cancelled" between steps and between PCG iterations, as the reference. `stats` sums the
 * iterations, device seconds and launches of all steps. Host pointers. */
int femgpu_transient_run(femgpu_transient* t, size_t steps, const double* load,
                         double* temperature, size_t output_every, double* frames,
                         femgpu_energy* energies, const volatile int* cancel,
                         femgpu_stats* stats);
void femgpu_transient_free(femgpu_transient* t);

/* ---------------------------------------------------------------- modes */

/* The lowest eigenpairs of K x = lambda M x of an elastic model by shift-invert subspace
 * iteration with Rayleigh-Ritz (eigen.rs:81-177) as modes.rs:180-216 runs it: K - shift M is
 * formed on the device and solved by this library's solver (the dense factor or PCG with
 * multigrid, resident for all the solves); the p = max(2 count, count + 8) subspace vectors and
 * their images stay on the device, and so does the p x p Rayleigh-Ritz problem
 * (femgpu_dense_generalized's solver). */
typedef struct femgpu_modes_stats {
    size_t iterations;      /* subspace iterations */
    size_t solves;          /* solves of (K - shift M) x = M y */
    size_t pcg_iterations;  /* summed over the solves (0 with the direct method) */
    double shift;           /* the shift used */
    double seconds;         /* device time of the solves */
} femgpu_modes_stats;

/* eigen.rs:81-177. `k` and `m` are the free-unknown submatrices of the stiffness and the mass
 * (the same pattern, as modes.rs:183-185 forms them; femgpu_assemble with FEMGPU_P2_ELASTIC and
 * FEMGPU_P2_MASS, then femgpu_csr_submatrix); `shift` NaN takes modes.rs:186-191's
 * -1e-8 mean(K_ii / M_ii). `unknowns`, `method`, `crossover` (NULL: Unknowns(16384); the
 * reference's modes pass Flops{infinity, 2.5e8, flat}, modes.rs:101-107) and
 * `options` are those of femgpu_solver_new for K - shift M. `values` gets `count` eigenvalues
 * ascending, `vectors` (NULL skips them) count x n M-orthonormal vectors. At most 64 modes; the
 * reference's texts for too many modes, non-convergence in 120 iterations and "cancelled"
 * (between iterations and between PCG iterations). Host pointers. */
int femgpu_modes(const femgpu_csr* k, const femgpu_csr* m, size_t count, double shift,
                 const femgpu_unknowns* unknowns, int method, const femgpu_crossover* crossover,
                 const femgpu_options* options, const volatile int* cancel, double* values,
                 double* vectors, femgpu_modes_stats* stats);
/* modes.rs:355-420 for the box grid: femgpu_modes with `cells` (their `mass` set), whose
 * solver of K - shift M takes its coarse matrices from the cells' K_e - shift M_e. */
int femgpu_modes_cells(const femgpu_csr* k, const femgpu_csr* m, size_t count, double shift,
                       const femgpu_unknowns* unknowns, int method,
                       const femgpu_crossover* crossover, const femgpu_options* options,
                       const femgpu_cells* cells, const volatile int* cancel, double* values,
                       double* vectors, femgpu_modes_stats* stats);
/* The step of eigen.rs:183-269 on the device: K q = lambda M q for dense symmetric row-major
 * n x n host matrices, M positive definite, n <= 1024; the eigenvalues ascending and the vectors
 * as the columns of q with Q^T M Q = I. The scaled Cholesky reduction of the reference, then the
 * parallel (round-robin) Jacobi method in place of its cyclic one: the reference's results to
 * rounding, and its texts for an M that is not positive definite or has dependent columns. */
int femgpu_dense_generalized(const double* k, const double* m, size_t n, double* values,
                             double* q);

/* ---------------------------------------------------------------- post-solve recovery */

/* The strain and the stress of a solved P2 elasticity model at the 10 points of each cell,
 * the mean at each point, and the peak of each part: the loop of elastic_tet.rs:367-427 with
 * Tet10::strain_stress (tet10.rs:142-169), and the von Mises and principal stresses of the
 * means (elastic_tet.rs:482-483; elastic.rs:977-1002). Materials are isotropic, E and nu per
 * cell as in femgpu_assemble. Stress order xx, yy, zz, xy, yz, xz (elastic.rs:967-970); strain
 * as tensor components in the same order (elastic.rs:972-975). The sums at each point run in
 * increasing cell order, so stress, strain, mises and the peaks are bit-identical with the
 * reference; the principal stresses call acos and cos and agree to a few ulp. */
typedef struct femgpu_recovery femgpu_recovery;

/* The reference's `Peak` of 1 part (elastic.rs:186-195, set by elastic_tet.rs:405-416): the
 * largest von Mises stress over the 10 points of the part's cells, first in (cell, point) order
 * on ties, and the same over the regular points (neither the point nor a corner of its cell
 * singular). A part with no cell keeps mises -inf and element -1; regular_element -1 is the
 * reference's `None`. */
typedef struct femgpu_peak {
    double mises;
    int64_t element;         /* the cell */
    int32_t local;           /* which of its 10 points (tet10.rs:216-228 order) */
    uint32_t point;          /* that point's number */
    int32_t singular;        /* 1: the point or a corner of the cell is singular (`why`) */
    int32_t pad;
    double regular_mises;
    int64_t regular_element;
    int32_t regular_local;
    uint32_t regular_point;
} femgpu_peak;

/* The mesh side of the loop, kept on the device: points (3 coordinates each), the 10 points of
 * each cell (corners first, as Quadratic, tet10.rs:232-272), E and nu per cell, the thermal
 * expansion alpha_x, alpha_y, alpha_z per cell (NULL: none; D alpha as elastic_tet.rs:164-170),
 * the part of each cell (NULL: all in part 0; nparts >= 1, at most 2048) and the singular mask
 * of each point (NULL: none; the reference's `singular_points`). */
int femgpu_recovery_new(size_t npoints, const double* xyz, size_t nel, const uint32_t* tets10,
                        const double* coef, const double* expansion, const uint32_t* part,
                        size_t nparts, const uint8_t* singular, femgpu_recovery** out);
/* The forces of the box cells' loop (elastic.rs:386-405): for each cell in increasing order and
 * each of its 24 unknowns, the load of its corner temperature changes (Hex::load, hex.rs:283-289:
 * D alpha through the 8 corners, the modes condensed) plus `accel` (3 per cell: the density
 * times gravity plus the body force per unit volume, as the reference sums them) times the
 * volume / 8, summed into `force` (3 per point, written whole) in the reference's order. `coef`
 * and `expansion` as femgpu_recovery_new_hex; `accel` and `dtemp` (1 per point) may be null: 0.
 * The reference's `gross` force scale is not formed. */
int femgpu_hex_loads(size_t npoints, const double* xyz, size_t nel, const uint32_t* hexes,
                     const double* coef, const double* expansion, const double* accel,
                     const double* dtemp, double* force);
/* The box grid's loop (elastic.rs:615-660 and 709-710): the strain and the stress at the 8
 * corners of each box cell (Hex::strain_stress, hex.rs:311-335, with the cell's incompatible
 * modes recovered from its corners), their mean at each point and the peaks of each part. The 8
 * corners of each cell in VTK order, the sides corner 6 minus corner 0; `coef` holds the 9
 * orthotropic constants per cell (as FEMGPU_HEX8_ELASTIC), `expansion` alpha_x, alpha_y, alpha_z
 * per cell (NULL: none; D alpha as hex.rs:222-223); `part` and `singular` as above. The peaks'
 * `local` is the corner (0-7). femgpu_recovery_run then serves both kinds of cells. */
int femgpu_recovery_new_hex(size_t npoints, const double* xyz, size_t nel, const uint32_t* hexes,
                            const double* coef, const double* expansion, const uint32_t* part,
                            size_t nparts, const uint8_t* singular, femgpu_recovery** out);
/* One recovery from the full displacement `u` (3 per point; the solution at the free unknowns
 * and the prescribed values elsewhere, elastic_tet.rs:349-351) and the temperature change of
 * each point (NULL: none; only corners are read). Outputs may be NULL to skip them: stress and
 * strain 6 per point, mises 1, principal 3 (largest first), peaks nparts. Host pointers. */
int femgpu_recovery_run(femgpu_recovery* r, const double* u, const double* dtemp, double* stress,
                        double* strain, double* mises, double* principal, femgpu_peak* peaks);
/* The same with u, dtemp, stress, strain, mises and principal in device memory (stress and
 * strain required); peaks stays a host array. Returns when the results are written. */
int femgpu_recovery_run_device(femgpu_recovery* r, const double* u, const double* dtemp,
                               double* stress, double* strain, double* mises, double* principal,
                               femgpu_peak* peaks);
/* The probes of a P2 model (elastic_tet.rs:428-467): for each point (3 coordinates each), the
 * cells whose volume coordinates of the point are all >= -1e-9 (cells_at, elastic_tet.rs:538-553),
 * each taking the share 1 / hits of the displacement (the 10 functions of tet10.rs:51-60), the
 * stress (Tet10::strain_stress with `dtemp`) and the temperature (the 4 corners of `temperature`,
 * the absolute corner temperatures; NULL: 0), summed in increasing cell order as the reference;
 * `mises` of the mean stress. Outputs: displacement 3, stress 6 (xx, yy, zz, xy, yz, xz), mises 1,
 * temp 1 per probe; `hits` (may be NULL) the cells of each. A probe in no cell fails with the
 * reference's text "probe NAME at (x, y, z) is in no part" (names may be NULL: the index), the
 * coordinates as Rust's {} writes them. Bit-identical with the reference. Host pointers. */
int femgpu_recovery_probes(femgpu_recovery* r, const double* u, const double* dtemp,
                           const double* temperature, size_t nprobes, const double* points,
                           const char* const* names, double* displacement, double* stress,
                           double* mises, double* temp, int64_t* hits);
/* The device time of the recovery kernels of the last run in ms (CUDA events), and the
 * algorithmic bytes they move: the cell records, the incidence and u once, the outputs once. */
int femgpu_recovery_last_time(const femgpu_recovery* r, double* ms, double* bytes);
size_t femgpu_recovery_bytes(const femgpu_recovery* r);
void* femgpu_recovery_stream(const femgpu_recovery* r);
void femgpu_recovery_free(femgpu_recovery* r);

/* ---------------------------------------------------------------- reactions */

/* elastic::reactions (elastic.rs:772-839), as elastic.rs:585 and elastic_tet.rs:352 call it
 * after the solve: r = K u - f at each fixed unknown i, in increasing i, summed into
 * `load_force` (3 per load: the components of the reactions of load owner[i]; for a fixed face
 * set that is the reference's Reaction::force, for a point support its point_force, whose
 * warning is |component| > 1e-6 `gross_out`), into `total` (applied + the reactions, per
 * component) and into `gross_out` (`gross` + |r|); `imbalance` = max |total| / gross_out, 0 when
 * gross_out is 0 (the reference warns above IMBALANCE = 1e-6, elastic.rs:278). `k` is the full
 * stiffness (3 unknowns per point, femgpu_assemble); `u` the full displacement and `force` the
 * full force (3 per point); `fixed` 1 byte per unknown (nonzero: fixed); `owner` the load that
 * fixed each unknown (values >= nloads are skipped, as the reference's `None`); `applied` the 3
 * sums of the applied forces. Every sum is in the reference's order: bit-identical. Host
 * pointers. */
int femgpu_reactions(const femgpu_csr* k, const double* u, const double* force,
                     const uint8_t* fixed, const uint32_t* owner, size_t nloads,
                     const double* applied, double gross, double* load_force, double* total,
                     double* gross_out, double* imbalance);

/* ---------------------------------------------------------------- prism meshes */

/* prism.rs:29-37 Outline: a polygon (`ncorners` corners, 2 coordinates each across the axis, in
 * either direction) or a circle (`centre`, `radius`). */
typedef struct femgpu_outline {
    int circle;
    size_t ncorners;
    const double* corners;
    double centre[2];
    double radius;
} femgpu_outline;

/* grid.rs:22-35 Part: a box [lo, hi] of material `material`; where parts overlap the higher
 * `priority` holds the space. With `has_footprint` the part is the prism of the footprint
 * (prism.rs:40-44: `outline` and `nholes` holes) between lo and hi on the extrusion axis. */
typedef struct femgpu_part {
    const char* name;
    size_t material;
    int64_t priority;
    double lo[3], hi[3];
    int has_footprint;
    femgpu_outline outline;
    size_t nholes;
    const femgpu_outline* holes;
} femgpu_part;

/* grid.rs:37-46 Spacing. */
typedef struct femgpu_spacing {
    double max_cell;
    double max_growth;
    size_t min_cells;
} femgpu_spacing;

typedef struct femgpu_tetmesh femgpu_tetmesh; /* prism.rs:117-132 TetMesh */
typedef struct femgpu_tetmesh_counts {
    size_t points, tets, faces, face_circles, circles, triangles, planes;
} femgpu_tetmesh_counts;

/* prism::mesh_hollow (prism.rs:185-380; prism::mesh, prism.rs:170-181, with no hollow part), as
 * heat.rs:898, elastic_tet.rs:98 and modes.rs:432 call it: the footprints of all parts meshed in
 * 1 quality triangle mesh on the host (mesh2d.rs), extruded through the graded planes of `axis`
 * (grid.rs:418) and cut into 3 tetrahedra per prism on the device. `hollow[k]` nonzero: part k
 * keeps its space but no tetrahedra (missing items: 0). More than `max_points` points ends with
 * FEMGPU_ERR_TOO_LARGE and the text `refusal`; the reference's other errors come with their texts
 * (FEMGPU_ERR_INVALID). The points and tetrahedra stay on the device for femgpu_assemble_device
 * (femgpu_tetmesh_device) and are copied to the host (femgpu_tetmesh_copy). Host pointers. */
int femgpu_prism_mesh(const femgpu_part* parts, size_t nparts, int axis,
                      const femgpu_spacing* spacing, size_t max_points, const char* refusal,
                      int periodic, const uint8_t* hollow, size_t nhollow, femgpu_tetmesh** out);
int femgpu_tetmesh_sizes(const femgpu_tetmesh* m, femgpu_tetmesh_counts* sizes);
/* Any pointer may be null (skipped). points 3 per point; tets 4 per tetrahedron (positive
 * volume); part 1 per tetrahedron; the boundary faces sorted by (tet, nodes): face_nodes 3 per
 * face (counterclockwise from outside), face_tet, face_beyond (the hollow part beyond, or
 * 0xffffffff), face_circle_start (faces + 1 offsets into face_circles: the circles whose outline
 * holds the face); circles 3 per circle (centre, radius). */
int femgpu_tetmesh_copy(const femgpu_tetmesh* m, double* points, uint32_t* tets, uint32_t* part,
                        uint32_t* face_nodes, uint32_t* face_tet, uint32_t* face_beyond,
                        uint64_t* face_circle_start, uint32_t* face_circles, double* circles);
/* The device copies of the points, tetrahedra and parts (owned by the mesh). */
int femgpu_tetmesh_device(const femgpu_tetmesh* m, const double** points, const uint32_t** tets,
                          const uint32_t** part);
void femgpu_tetmesh_free(femgpu_tetmesh* m);

/* grid::axis_planes (grid.rs:418-484): the graded planes of axis `axis` for the parts and the
 * `extra` key planes; `count` is set to their number and up to `cap` are written. Host only (no
 * device work). */
int femgpu_axis_planes(const femgpu_part* parts, size_t nparts, int axis,
                       const femgpu_spacing* spacing, const double* extra, size_t nextra,
                       double* planes, size_t cap, size_t* count);

/* mesh2d::mesh / periodic_mesh (mesh2d.rs:87-110): the quality triangle mesh of `points` (2
 * coordinates each) and `segments` (2 point numbers each); `classify(point, ctx)` labels a point
 * inside a region, or returns 0xffffffff (outside). Host only (no device work). */
typedef uint32_t (*femgpu_classify_fn)(const double* point, void* ctx);
typedef struct femgpu_mesh2 femgpu_mesh2; /* mesh2d.rs:72-82 Mesh2 */
int femgpu_mesh2d(const double* points, size_t npoints, const uint32_t* segments,
                  size_t nsegments, double max_size, double max_growth, int periodic,
                  femgpu_classify_fn classify, void* ctx, femgpu_mesh2** out);
int femgpu_mesh2_sizes(const femgpu_mesh2* m, size_t* points, size_t* triangles,
                       size_t* segment_edges, size_t* segment_origins);
/* Any pointer may be null. points 2 per point; triangles 3 per triangle (counterclockwise);
 * label 1 per triangle; across 3 per triangle (the triangle across the edge opposite each point,
 * or 0xffffffff); the edges on segments (2 points each, smaller first, in increasing order) with
 * their input segments: origin_start (edges + 1 offsets) into origins. */
int femgpu_mesh2_copy(const femgpu_mesh2* m, double* points, uint32_t* triangles, uint32_t* label,
                      uint32_t* across, uint32_t* edges, uint64_t* origin_start,
                      uint32_t* origins);
void femgpu_mesh2_free(femgpu_mesh2* m);

/* grid::Grid::build (grid.rs:116-158, the cells' parts by grid.rs:292-330) and the hex mesh of
 * its cells (heat.rs:1165-1210 `number`), as heat.rs:755-800 and elastic.rs call them through
 * build_grid: the graded planes of each axis (with the `nextra[d]` extra key planes `extra[d]`,
 * for example a plane of symmetry), each cell's part (the highest priority holding its centre;
 * the footprints of the parts are not read), the mesh points numbered in first use over the cells
 * of the parts (cell order i + nx (j + ny k), corners in VTK order) and the model's faces (sides
 * with no cell of a part beyond, grid.rs:234-254). More than `max_points` mesh points ends with
 * FEMGPU_ERR_TOO_LARGE and the text `refusal`; the reference's other errors come with their texts.
 * The mesh points and cells stay on the device (femgpu_boxgrid_device). Host pointers. */
typedef struct femgpu_boxgrid femgpu_boxgrid;
typedef struct femgpu_boxgrid_counts {
    size_t planes[3], grid_cells, points, cells, faces;
} femgpu_boxgrid_counts;
int femgpu_box_grid(const femgpu_part* parts, size_t nparts, const femgpu_spacing* spacing,
                    const double* const* extra, const size_t* nextra, size_t max_points,
                    const char* refusal, femgpu_boxgrid** out);
int femgpu_boxgrid_sizes(const femgpu_boxgrid* g, femgpu_boxgrid_counts* counts);
/* Any pointer may be null. planes: 3 arrays; part per grid cell (0xffffffff: void); points 3 per
 * mesh point and ijk its grid point; cells 8 per mesh cell; cell_of its grid cell; mesh_part its
 * part; the faces as (grid cell, side in x-, x+, y-, y+, z-, z+ order). */
int femgpu_boxgrid_copy(const femgpu_boxgrid* g, double* const* planes, uint32_t* part,
                        double* points, uint32_t* ijk, uint32_t* cells, uint64_t* cell_of,
                        uint32_t* mesh_part, uint64_t* face_cell, uint8_t* face_side);
int femgpu_boxgrid_device(const femgpu_boxgrid* g, const double** points, const uint32_t** cells);
void femgpu_boxgrid_free(femgpu_boxgrid* g);

/* prism::split_prism (prism.rs:144-154): the 3 tetrahedra (12 local corners) of a prism whose
 * corners (bottom 0 1 2, top 3 4 5, 3 above 0) have the global numbers g[6]. */
int femgpu_split_prism(const uint64_t* g, int32_t* out);

#ifdef __cplusplus
}
#endif
#endif /* FEMGPU_H */
