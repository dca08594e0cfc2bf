/*
 * mfs_b200.h -- C ABI of the B200 numeric path for MeshFEMSparse-style
 * block-CSC Hessians: element assembly, supernodal Cholesky and multi-RHS
 * triangular solves on one GPU.
 *
 * Plain pointers and sizes only. Every entry point returns an mfs_status and
 * never throws; mfs_last_error() returns the message of the last failure on a
 * handle. A handle is bound to one CUDA device and one stream and is not
 * re-entrant (one handle per stream), like the reference factorizer, whose
 * solve scratch is mutable state (Solvers/CholeskyFactorizerBase.hh:396-397).
 *
 * Matrix format (the reference's BlockCSCHessian<..., ContiguousBlocks=true>,
 * BlockCSCHessian.hh:560-571, 862-875): upper-triangular block CSC over
 * n_blocks block variables of size bs; Ap (n_blocks+1) and Ai (nnz_b) are the
 * *block* pattern with rows sorted per column; Ax holds bs*bs scalars per block,
 * each block column-major and contiguous, at Ax[bs*bs*k]; diagonal blocks are
 * stored in full but only their upper triangle is read.
 * Pins are scalar variable indices (x[pins] = 0), as in
 * CholeskyFactorizerBase::factorizeSymbolic(mat, pinnedVars).
 */
#ifndef MFS_B200_H
#define MFS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    MFS_OK = 0,
    MFS_NOT_POSDEF = 1,     /* numeric factorization hit a non-positive pivot */
    MFS_INVALID_ARG = 2,
    MFS_SIZE_MISMATCH = 3,
    MFS_NO_FACTOR = 4,      /* the requested factorization does not exist */
    MFS_OOM = 5,
    MFS_TIMEOUT = 6,
    MFS_CUDA_ERROR = 7,
    MFS_INTERNAL = 8
} mfs_status;

typedef enum {
    MFS_PREC_FP64 = 0,      /* FP64 factor and solves (the drop-in plain path) */
    MFS_PREC_FP32 = 1       /* FP32 factor (tensor-core Schur updates), FP64 vectors */
} mfs_precision;

typedef enum {
    MFS_ORDER_ND = 0,       /* nested dissection (CatamariFactorizer::OrderingMethod::CholmodNesdisParallel) */
    MFS_ORDER_NATIVE = 1,   /* input order kept (OrderingMethod::Native) */
    MFS_ORDER_MD = 2,       /* minimum degree (OrderingMethod::AMD) */
    MFS_ORDER_USER = 3      /* caller-supplied permutation (replay of a recorded ordering) */
} mfs_ordering;

/* Solve flags */
#define MFS_SOLVE_FULL 0            /* B, X have n_full rows; pinned rows of X are 0 (CholeskyFactorizerBase::solve) */
#define MFS_SOLVE_REDUCED 1         /* n_reduced rows, unpermuted (solveRawReduced, alreadyPermuted=false) */
#define MFS_SOLVE_REDUCED_PERMUTED 2 /* n_reduced rows, already permuted (alreadyPermuted=true) */
#define MFS_DEVICE_POINTERS 16      /* B/X (or Ax, Ke) are device pointers */

typedef struct {
    int32_t precision;          /* mfs_precision */
    int32_t ordering;           /* mfs_ordering */
    int32_t relax;              /* relax_supernodes (CatamariFactorizer.cc:105), default 1 */
    int32_t device;             /* CUDA device ordinal */
    int64_t relax_zeros;        /* allowable explicit zeros per relaxed supernode (128) */
    double relax_ratio;         /* alternative allowance as zero ratio (0.01) */
    int64_t nd_leaf_size;       /* nested-dissection leaf size (vertices) */
    uint64_t seed;              /* ordering seed */
    void *stream;               /* cudaStream_t, NULL = a stream owned by the handle */
    int32_t small_front_max;    /* fronts up to this size are factored in shared memory (0 = default) */
    int32_t refine;             /* FP32 solves: FP64 preconditioned-CG refinement on (1) / off (0) */
    double refine_tol;          /* relative residual target ||b - Hx|| / ||b|| (1e-10) */
    int32_t refine_maxit;       /* iteration cap (50) */
    int32_t use_graphs;         /* capture the factorization / solve launch sequence in CUDA graphs */
    int32_t tensor_cores;       /* FP32 Schur updates: 0 auto (6 with refinement, else split 3xTF32),
                                   1 TF32 on tcgen05, 2 split 3xTF32 (FP32-level products, mma.sync),
                                   3 TF32 on mma.sync (the pre-Blackwell tensor-core path),
                                   4 TF32 on tcgen05 with TMA-fed operands for the Schur updates,
                                   5 FP16 operands on tcgen05 (kind::f16, TMA-fed): the row solves
                                     write a copy of the panels scaled by a power of two per front;
                                     needs refine = 1 (without it: as 2),
                                   6 split FP16 on tcgen05: hi and 2^11-scaled lo half copies, three
                                     MMAs per k slice into two TMEM accumulators (FP32-level products),
                                     split-TF32 row solves; needs refine = 1 (without it: as 2) */
    int32_t time_kernels;       /* 1: mfs_numeric times each tensor-core GEMM launch with CUDA events on its
                                   stream (mfs_stats.gemm_ms / gemm_flops); adds event records, off by default */
    int32_t nd_reuse_period;    /* > 0: a nested-dissection analysis of a changed pattern on the same variables
                                   reuses the previous separator tree, re-dissecting only the subtrees that a
                                   new edge violates (PARTH-style temporal reuse, ParallelNestedDissection/
                                   README.md:86-127); a full dissection every nd_reuse_period analyses */
    int32_t solve_chain;        /* diagonal-block solves of the fronts above the subtree cut: 0 through the
                                   inverses of 256-row superblocks of L11 (one CTA per superblock),
                                   1 through chains of 64-row blocks (one CTA per pair of blocks) */
    int32_t factor_group;       /* large fronts: column blocks per group of the blocked factorization (inside a
                                   group left-looking, after it one update of the rest of the front);
                                   0: default (4); read at the symbolic analysis */
    int32_t solve_subtrees;     /* solves: the levels below the highest level with at least this many subtrees
                                   (fronts of at most 2048 rows) are solved one subtree per CTA, the levels above
                                   by level kernels; 0: default (the larger of 2368 and 48 per tree of the
                                   assembly forest); read at the symbolic analysis */
    int32_t reserved[2];
} mfs_options;

typedef struct mfs_handle mfs_handle;

/* Defaults matching the reference's CatamariFactorizer configuration. */
mfs_status mfs_default_options(mfs_options *opt);

/* Replaces: make_cholesky_factorizer(CholeskyProvider, singlePrecision)
 *           (Solvers/make_cholesky_factorizer.cc:54-123) */
mfs_status mfs_create(mfs_handle **h, const mfs_options *opt);
/* Updates the options that take effect at the next symbolic analysis or solve
 * (ordering, relaxation, refinement, tensor cores, graphs); precision, device
 * and stream are fixed per handle. Mirrors setting CatamariFactorizer::orderingMethod
 * (CatamariFactorizer.hh:149-154), which also applies at the next factorizeSymbolic. */
mfs_status mfs_set_options(mfs_handle *h, const mfs_options *opt);
mfs_status mfs_destroy(mfs_handle *h);
/* Copies the last error message (NUL-terminated, truncated to len). */
mfs_status mfs_last_error(const mfs_handle *h, char *buf, size_t len);

/* Replaces: SystemAssembler<N>::blockSparsityPattern(numElems, elemGetter)
 *           (SystemAssembler.hh:252-465). Two-phase: with Ai == NULL only
 *           Ap (nvars+1) and *nnz are produced; call again with Ai of size *nnz. */
mfs_status mfs_build_pattern(int64_t nvars, int64_t nelem, int32_t npe, const int64_t *conn, int64_t *Ap,
                             int64_t *Ai, int64_t *nnz);
/* Replaces: SystemAssembler<N>::blockSparsityPattern (SystemAssembler.hh:252-465),
 *           built on the GPU: conn (nelem x npe, npe <= 32), Ap (nvars+1) and Ai are
 *           device pointers on `device`, stream a cudaStream_t (NULL: the legacy
 *           stream); *nnz is host memory. Same two-phase protocol and the same
 *           result, entry for entry, as mfs_build_pattern. Synchronizes the stream. */
mfs_status mfs_build_pattern_device(int32_t device, int64_t nvars, int64_t nelem, int32_t npe,
                                    const int64_t *conn, int64_t *Ap, int64_t *Ai, int64_t *nnz, void *stream);

/* Replaces: CatamariFactorizer::factorizeSymbolic(const BlockCSCHessianBase&, pinnedVars)
 *           (Solvers/CatamariFactorizer.cc:136-161, 177-616).
 * user_perm (MFS_ORDER_USER only): new->old over reduced block variables.
 * supernode_sizes (optional, NATIVE / USER orderings): a supernode partition in reduced
 * block variables to use verbatim instead of fundamental + relaxed supernodes, as the
 * reference's SymmetricOrdering::supernode_sizes (CatamariFactorizer.cc:311-324);
 * every supernode must be a chain of the elimination tree. */
mfs_status mfs_symbolic(mfs_handle *h, int64_t n_blocks, const int64_t *Ap, const int64_t *Ai, int32_t block_size,
                        const int64_t *pinned, int64_t n_pinned, const int64_t *user_perm,
                        const int64_t *supernode_sizes, int64_t num_supernodes);

/* Replaces: CatamariFactorizer::factorizeNumeric / factorizeNumericWithShift(A, sigma[, B])
 *           (Solvers/CatamariFactorizer.cc:618-714, CatamariFactorizer.hh:52-63).
 * Factors A + sigma*I (Bx == NULL) or A + sigma*B (B shares A's pattern and layout).
 * Ax == NULL uses the values produced by the last mfs_assemble on this handle.
 * On a non-positive pivot returns MFS_NOT_POSDEF and the numeric factor is invalidated
 * (CatamariFactorizer.cc:701-705). */
mfs_status mfs_numeric(mfs_handle *h, const double *Ax, const double *Bx, double sigma, int32_t flags);

/* Replaces: CholeskyFactorizerBase::solve / solveMultiRHS / solveRawReduced[InPlace]
 *           (CholeskyFactorizerBase.hh:263-363, CatamariFactorizer.cc:788-907).
 * Column-major B and X (ld = ldb), nrhs columns; X may alias B. */
mfs_status mfs_solve(mfs_handle *h, const double *B, double *X, int64_t nrhs, int64_t ldb, int32_t flags);

/* Assembly (SystemAssembler::assembleHessianBlockAccelerated, SystemAssembler.hh:524-577):
 * set the element stencils once per pattern, then assemble Ax = sum_e Ke_e into the
 * pattern passed to mfs_symbolic. Ke is [nelem][12][12] row-major FP64 (bs = 3, 4 nodes).
 * The result stays resident on the device for mfs_numeric(h, NULL, ...). */
mfs_status mfs_assembly_setup(mfs_handle *h, int64_t nelem, const int64_t *conn);
mfs_status mfs_assemble(mfs_handle *h, const double *Ke, double *Ax_out, int32_t flags);

/* y = H x on the reduced system (BlockCSCHessianBase::apply restricted to free
 * variables; BlockCSCHessian.hh:723-732). flags: MFS_SOLVE_FULL / REDUCED / REDUCED_PERMUTED
 * select the vector layout as for mfs_solve; pinned rows of a full y are 0. */
mfs_status mfs_apply(mfs_handle *h, const double *x, double *y, int64_t nrhs, int64_t ld, int32_t flags);
/* No counterpart in the reference. mfs_apply for callers that cannot allocate
 * device memory at the point where they apply H: a process whose caching
 * allocator has already reserved the device, or a loop where the device-wide
 * synchronisation of cudaMalloc / cudaFree is not acceptable. x and y must be
 * device pointers (flags must include MFS_DEVICE_POINTERS); the vector layouts
 * are those of mfs_apply. Temporaries live in one fixed device array of
 * 2 x 2^20 doubles (16 MiB, on every GPU that loads the library, until exit),
 * so (free variables) x nrhs may not exceed 1048576 (MFS_SIZE_MISMATCH
 * otherwise). The first call on a device looks up that array's address; make
 * it before any stream capture. All calls on a device share the array: calls
 * that overlap on the GPU (other handles, other streams) race and must be
 * serialised by the caller. Returns after the result is written. */
mfs_status mfs_apply_noalloc(mfs_handle *h, const double *x, double *y, int64_t nrhs, int64_t ld, int32_t flags);

/* ---- Learned preconditioner (no counterpart in the reference). A 4-layer
 * message-passing network (hidden 64, BF16 weights, FP32 accumulation) reads the
 * Jacobi-scaled 3 x 3 blocks of H and emits a lower block-triangular G on H's
 * pattern; mfs_pcg_solve runs PCG with M^{-1} = D^{-1/2} G^T G D^{-1/2}
 * (D = diag H) and falls back to the Cholesky factor (mfs_numeric + mfs_solve on
 * the same values) when PCG misses `tol` within `maxit` iterations. Needs a 3 x 3
 * block analysis (block size 3, whole-block pins). A network lives on one device
 * and may serve many handles on that device; it is not re-entrant. */
typedef struct mfs_lpc mfs_lpc;
mfs_status mfs_lpc_param_count(int64_t *count);
/* Weights drawn from `seed`; the output head starts at zero, so G = I (Jacobi). */
mfs_status mfs_lpc_create(mfs_lpc **net, int32_t device, uint64_t seed);
mfs_status mfs_lpc_destroy(mfs_lpc *net);
/* FP32 master weights (host arrays of mfs_lpc_param_count floats); setting them
 * resets the optimizer state. */
mfs_status mfs_lpc_get_weights(const mfs_lpc *net, float *w, int64_t count);
mfs_status mfs_lpc_set_weights(mfs_lpc *net, const float *w, int64_t count);
/* Loss mean_r ||M^{-1} b_r - x_r||_H^2 / (x_r^T b_r) of pairs (B, X = H^{-1} B) and
 * its gradient (host, param_count floats; NULL to skip). Ax: matrix values in the
 * caller's block-CSC layout, NULL = the last mfs_assemble; flags as mfs_solve
 * (vector order | MFS_DEVICE_POINTERS, which also covers Ax). nrhs <= 64. */
mfs_status mfs_lpc_loss_grad(mfs_handle *h, mfs_lpc *net, const double *Ax, const double *B, const double *X,
                             int64_t nrhs, int64_t ld, int32_t flags, double *loss, float *grad);
/* One Adam step (beta 0.9 / 0.999) of the loss above at learning rate lr. */
mfs_status mfs_lpc_train_step(mfs_handle *h, mfs_lpc *net, const double *Ax, const double *B, const double *X,
                              int64_t nrhs, int64_t ld, int32_t flags, float lr, double *loss);
/* X = H^{-1} B by PCG to relative residual tol (per column) within maxit
 * iterations (<= 0: 200); net NULL = Jacobi. On a miss the handle factors Ax and
 * solves (its own precision and refinement options); mfs_stats.pcg_fallback says
 * which ran. *iterations = PCG iterations taken. */
mfs_status mfs_pcg_solve(mfs_handle *h, mfs_lpc *net, const double *Ax, const double *B, double *X, int64_t nrhs,
                         int64_t ld, int32_t flags, int32_t maxit, double tol, int32_t *iterations);
/* Conversion-plan entries are exported as 4 int64 each: (dst, src, ld, flags);
 * flags bit0 = source block transposed, bit1 = diagonal block (lower part only). */

/* Introspection: CatamariFactorizer::getFactorNNZ / getFlopEstimate / n_reduced /
 * getInversePermutation (CatamariFactorizer.cc:716-732). */
mfs_status mfs_info(const mfs_handle *h, int64_t *n_full, int64_t *n_reduced, int64_t *factor_nnz,
                    double *flops, int64_t *num_supernodes, int32_t *factorization_type);
mfs_status mfs_inverse_permutation(const mfs_handle *h, int64_t *iperm_out /* n_reduced */);
/* NDOrdering snapshot (CholeskyFactorizerBase.hh:55-59): sizes first with NULL outputs. */
mfs_status mfs_nd_ordering(const mfs_handle *h, int64_t *ncomp, int64_t *nmember, int64_t *cparent,
                           int64_t *cmember);
/* Supernode partition: sn_start (nsn+1, analysis-variable columns), parent (nsn),
 * struct_ptr (nsn+1), struct_rows, rel (per struct entry, child_rel_indices),
 * analysis block size. Sizes first with NULL outputs. */
mfs_status mfs_supernodes(const mfs_handle *h, int64_t *nsn, int64_t *nstruct, int32_t *vb, int64_t *sn_start,
                          int64_t *parent, int64_t *struct_ptr, int64_t *struct_rows, int64_t *rel);
/* Conversion plan (CatamariConversionPlan.hh:402-541): column_offsets (2*nv+1) and
 * entries (4 int64 each, see above). Sizes first with NULL outputs. */
mfs_status mfs_conversion_plan(const mfs_handle *h, int64_t *nv, int64_t *nentries, int64_t *column_offsets,
                               int64_t *entries);
/* The same conversion plan as built on the GPU for the numeric factorization
 * (CatamariConversionPlan.hh:402-541, catamari layout), copied to host memory in
 * the format of mfs_conversion_plan; equal to it entry for entry. */
mfs_status mfs_conversion_plan_device(const mfs_handle *h, int64_t *nv, int64_t *nentries, int64_t *column_offsets,
                                      int64_t *entries);
/* Copies the factor values (factor_size entries as double) to host memory. */
mfs_status mfs_factor_values(const mfs_handle *h, int64_t *factor_size, double *out);

/* Stash / swap / clear (CatamariFactorizer.cc:925-948) and clearFactors (:111-114). */
mfs_status mfs_stash(mfs_handle *h);
mfs_status mfs_swap_stash(mfs_handle *h);
mfs_status mfs_clear_stash(mfs_handle *h);
mfs_status mfs_has_stash(const mfs_handle *h, int32_t *has);
mfs_status mfs_clear_factors(mfs_handle *h);

/* Statistics of the last numeric factorization / refined solve. */
typedef struct {
    double factor_ms;            /* device time of the last mfs_numeric (CUDA events) */
    double solve_ms;             /* device time of the last mfs_solve */
    double assemble_ms;          /* device time of the last mfs_assemble */
    int32_t refine_iterations;   /* PCG iterations of the last refined solve (max over RHS) */
    int32_t failed_column;       /* first non-positive pivot column, -1 if none */
    double residual;             /* max relative residual of the last refined solve */
    int64_t device_bytes;        /* device memory held by the handle */
    int32_t num_levels;          /* levels of the assembly tree */
    int32_t num_large;           /* supernodes on the tiled large-front path */
    int64_t kernel_launches;     /* kernels launched by the library since it was loaded */
    int32_t perturbed_pivots;    /* FP32 factor under refinement: non-positive pivots (after the FP64
                                    re-factor, for large fronts) replaced by a floor relative to the
                                    injected diagonal (last numeric) */
    int32_t pcg_iterations;      /* iterations of the last mfs_pcg_solve (max over RHS) */
    int32_t pcg_fallback;        /* 1: the last mfs_pcg_solve missed the tolerance and used the factor */
    int32_t nd_reused;           /* 1: the last symbolic analysis reused the previous separator tree */
    double pcg_ms;               /* device time of the last converged mfs_pcg_solve (inference + PCG) */
    double gemm_ms;              /* time_kernels: summed device time of the last mfs_numeric's GEMM launches */
    double gemm_flops;           /* algorithmic flops of those launches (2mnk, triangle-aware; m n k per row solve) */
    int64_t gemm_launches;       /* GEMM launches timed */
    int64_t nd_rebuilt_vertices; /* nd_reused: analysis variables re-dissected */
    int32_t refactored_blocks;   /* FP32 factor under refinement: large-front diagonal blocks whose FP32
                                    factorization met a pivot <= 1e-5 x the injected diagonal and were
                                    factored again in FP64 (last numeric) */
    int32_t split_escalations;   /* FP32 under refinement: times a single-pass TF32 / FP16 factorization was
                                    redone with split FP16 (FP32-level, tensor_cores 6) products because it perturbed a
                                    pivot or its refinement stalled; the handle then keeps the split
                                    products until the next symbolic analysis or mfs_set_options
                                    (cumulative) */
} mfs_stats;
mfs_status mfs_get_stats(const mfs_handle *h, mfs_stats *st);

#ifdef __cplusplus
}
#endif
#endif /* MFS_B200_H */
