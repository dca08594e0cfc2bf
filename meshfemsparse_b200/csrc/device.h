// Device-side data layout and kernel launchers shared by the CUDA sources.
//
// Storage in HBM (all column-major):
//   factor values  : one panel per supernode, (w+d) x w with ld = w+d rounded up to a
//                    multiple of 8 (16-byte aligned columns for the tensor-core
//                    GEMM loads, FP32 and FP16), panels back to back; the catamari layout
//                    (CatamariConversionPlan.hh:366, ld = w+d) is produced on export;
//                    followed by the
//                    64 x 64 inverses of the diagonal blocks of every large front's L11
//                    (written by the panel kernel) and the inverses of the 256-row
//                    superblocks of L11 of the fronts above the solve cut (written
//                    after the factorization, read by the triangular solves)
//   update arena   : U_s (d x d, ld d) of the multifrontal assembly tree; offsets from
//                    the static level-lifetime plan built on the host
//   solve arena    : u_s (d x nrhs, ld d) forward-substitution update vectors; offsets
//                    are the same plan computed with unit size d, scaled by nrhs
//   right-hand sides: permuted reduced order, n x nrhs, ld = n
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include <mutex>
#include <utility>

namespace mfs {

// One-time host set-up per device. Kernel attributes (the dynamic shared-memory
// opt-in) and occupancy figures belong to the device that is current when they
// are set or measured, so every such set-up is keyed by the current device.
constexpr int kMaxDevices = 64;
int current_device();                   // the calling thread's current device (0 if the query fails)
int device_sm_count();                  // SM count of the current device (cached per device)
struct PerDeviceOnce {
    std::once_flag flag[kMaxDevices];
    template <typename F>
    void operator()(F &&fn) {
        const int d = current_device();
        if (d < 0 || d >= kMaxDevices) {
            fn();
            return;
        }
        std::call_once(flag[d], std::forward<F>(fn));
    }
};

// Kernels launched by this library since load (every launcher increments it).
extern long long g_kernel_launches;

struct SnDev {
    const int32_t *w, *d, *f;           // scalar width / degree / front size
    const int32_t *ld;                  // panel leading dimension: f rounded up to a multiple of 8
    const int32_t *col0;                // first scalar column of the supernode
    const int64_t *pan_off;             // panel offset in the factor array (a multiple of 8)
    const int64_t *upd_off;             // U_s offset in the update arena (-1: none)
    const int64_t *sol_off;             // u_s offset (units of one RHS) in the solve arena
    const int64_t *inv_off;             // factor-array offset of the 64 x 64 inverses of L11's
                                        // diagonal blocks, ceil(w/64) blocks (-1: not stored)
    const int32_t *child_ptr, *child_list;
    const int64_t *struct_ptr;          // per supernode, into struct_rows / rel
    const int32_t *struct_rows;         // analysis-variable rows (permuted)
    const int32_t *rel;                 // per struct entry: scalar row in the parent's front
    int vb;                             // analysis block size
};

// Pivot handling of the factorization kernels: smallest failing column, count
// of perturbed pivots, and (perturbation mode only) the injected diagonal.
struct PivotCtl {
    int *fail_col;
    int *perturbed;
    const double *dorig;                // nullptr: no perturbation, failures are reported
    int *refactored;                    // FP32 panels under refinement: a diagonal block with a
                                        // pivot <= kRefactorTiny * injected diagonal is factored
                                        // again in FP64 (count of such blocks); nullptr: off
};
constexpr double kRefactorTiny = 1e-5;

// Plan entry mirror of host_symbolic.h PlanEntry.
struct PlanEntryDev {
    int64_t dst;
    int64_t src;
    int32_t ld;
    int32_t flags;
};

// C(i,j) -= sum_k A(i,k) B(j,k)  (mode 0)  or  C(i,j) = sum_k A(i,k) B(j,k)  (mode 1)
// for i < m, j < n over a grid of tiles_m x tiles_n CTA tiles; A, B, C are
// column-major blocks at the given offsets of the launch's three base arrays.
struct GemmTask {
    int64_t a_off, b_off, c_off;
    int32_t lda, ldb, ldc;
    int32_t m, n, k;
    int32_t tiles_m, tiles_n;
    int32_t tile_base;                  // prefix over tasks of tiles_m*tiles_n
    int32_t lower;                      // 1: only i >= j is touched
    int32_t mode;
    int32_t shift;                      // FP32: tiles start da = shift & 255 rows before A and
                                        // db = shift >> 8 rows before B (8-element aligned starts);
                                        // tiles_m / tiles_n cover m + da / n + db
    // TMA-fed kernel (mode 0): tensor maps of A and B (indices into the launch's map
    // array) and the map coordinates (row, column) of the shifted operand starts
    // (A(-da, 0) and B(-db, 0)); C -= 2^scale_exp * A B^T.
    int32_t amap, bmap;
    int32_t ax, ay, bx, by;
    int32_t scale_exp;
    int32_t sn;                         // front of the task (-1: none); FP16 operands of a front
                                        // are scaled by 2^-sexp[sn]
};
constexpr int kTensorMapBytes = 128;    // CUtensorMap (64-byte aligned in device memory)
struct alignas(64) TensorMapBlob {
    unsigned char bytes[kTensorMapBytes];
};

// One column block of a large front: factor its nb x nb diagonal block in
// place, store inv(L) of the block (nb x nb, ld ldi) at `inv_full` of the
// inverse scratch for the row solve X := X inv(L)^T that follows as a GEMM,
// and store the 64 x 64 diagonal blocks of inv(L) at `inv_out` of the factor
// array (-1: not stored), which the triangular solves apply as small GEMVs.
struct PanelTask {
    int64_t off;                        // offset of the diagonal block's (0,0) entry
    int64_t inv_full;                   // scratch offset of inv(L) of the block
    int64_t inv_out;                    // factor-array offset of the 64 x 64 inverse blocks
    int32_t ld, nb;
    int32_t col;                        // global scalar column of the block's first pivot
    int32_t ldi;                        // leading dimension of inv(L) in scratch (nb rounded up to 4)
};

// Extend-add of all children of a large supernode, split by front columns.
struct AssembleTask {
    int32_t sn;
    int32_t tile_base;                  // prefix over tasks of column chunks
};

// Solve tasks: one 64-row block of a front (blk < ceil(w/64): diagonal block,
// otherwise structure block blk - ceil(w/64)); flag_base indexes the front's
// first diagonal-block flag.
struct SolveTask {
    int32_t sn, blk, flag_base, pad;
};
// Forward extend-add of children's update vectors, split by front rows.
struct SolveAsmTask {
    int32_t sn;
    int32_t tile_base;
};
// Structure part of a solve level: one 64-row (forward) or 64-column (backward)
// slab `idx` of L21 times one kStrChunk-wide chunk of the other dimension.
struct StrTask {
    int32_t sn, idx, chunk, pad;
};
// Fixed-order reduction of the chunk partials [first, first + nchunks) of a slab.
struct StrReduce {
    int32_t sn, idx, first, nchunks;
};
// One superblock K of a front's L11 in the diagonal-block solves: a CTA task of the
// inverse kernel (part 0), or of the forward / backward chains for its 64-row part
// `pad`. inv: factor-array offset of inv(L_KK) (nrp x nrp column-major, nrp = 64 *
// ceil(rows / 64)); flag0: the front's first count (two per superblock: parts
// solved, parts whose accumulated right-hand side is in the scratch vector);
// pmap / imap: the first of the two tensor maps (forward box, backward box) of the
// front's L11 / of inv(L_KK) in the solve's map array.
struct SbTask {
    int32_t sn, K, flag0, pad;
    int64_t inv;
    int32_t pmap, imap;
};
constexpr int kSuperBlock = 256;        // rows per superblock
// structure part of the solves: forward tasks are kStrRows rows x kStrCols columns
// of L21, backward tasks kStrBCols columns x str_bwd_rows rows
constexpr int kStrRows = 1024;
constexpr int kStrCols = 256;
constexpr int kStrBCols = 64;
__host__ __device__ constexpr int str_bwd_rows(bool fp64) { return fp64 ? 1024 : 2048; }
constexpr int kSolveAsmRows = 256;      // front rows per forward extend-add CTA
constexpr int kMaxSolveRhs = 16;        // right-hand sides per solve pass (more are chunked)
constexpr int kSbMaxRhs = 8;            // right-hand sides per pass of the superblock solves

constexpr int kAsmCols = 32;            // front columns per assemble CTA
constexpr int kMaxSmemOptin = 232448;   // opt-in dynamic shared memory per CTA (227 KB)

// ---------------------------------------------------------------- launchers
template <typename T>
void launch_zero(T *p, int64_t n, cudaStream_t st);
template <typename T>
void launch_inject(const PlanEntryDev *plan, int64_t nplan, int vb, int src_ld, const double *Ax,
                   const double *Bx, double sigma_b, T *factor, cudaStream_t st);
template <typename T>
void launch_diag_shift(const int64_t *diag_off, int64_t n, double sigma, T *factor, cudaStream_t st);
template <typename T>
void launch_extract_diag(const int64_t *diag_off, int64_t n, const T *factor, double *out, cudaStream_t st);
template <typename T>
void launch_small_factor(const int32_t *list, int count, int max_front, SnDev sd, T *factor, T *upd,
                         PivotCtl pv, cudaStream_t st);
template <typename T>
void launch_assemble_large(const AssembleTask *tasks, int ntasks, int ntiles, SnDev sd, T *factor, T *upd,
                           cudaStream_t st);
template <typename T>
void launch_panel(const PanelTask *tasks, int ntasks, int max_nb, T *factor, T *inv_scratch, PivotCtl pv,
                  bool round_inv, cudaStream_t st);
// Tensor-core tile GEMM. float: split 1 = single-pass TF32 on tcgen05, 3 = split
// 3xTF32 on mma.sync, 0 = single-pass TF32 on mma.sync; double: DMMA. A wait of
// the tcgen05 pipeline that times out sets *err.
template <typename T>
void launch_gemm(const GemmTask *tasks, int ntasks, int ntiles, const T *A, const T *B, T *C, int split, int *err,
                 cudaStream_t st);
// h16 (row solves, mode 1): also store each result as FP16 scaled by 2^-sexp[task.sn]
// at the same offset of the half-precision copy, and store the FP32 result as that
// FP16 value scaled back (nullptr: the result is stored rounded to TF32).
// With h16lo as well (split-FP16 mode, mode-1 tasks): A and B are split into TF32 hi
// + lo in shared memory (FP32-level products), the FP32 result is stored as is, and
// the half copies get hi = rn16(2^-e v) and lo = rn16(2^11 (2^-e v - hi)).
void launch_gemm_tc(const GemmTask *tasks, int ntasks, int ntiles, const float *A, const float *B, float *C, int *err,
                    cudaStream_t st, void *h16 = nullptr, const int32_t *sexp = nullptr, void *h16lo = nullptr);
// TMA-fed tcgen05 GEMM (mode 0 tasks only). operands: 0 FP32 read as TF32, 1 FP16
// (kind::f16), 2 split FP16 (hi + 2^-11 lo, three MMAs per k slice into two TMEM
// accumulators; the lo operands' tensor maps are lo_maps entries after the hi ones).
// C -= 2^e A B^T with e = 2 sexp[task.amap] when sexp is given (the operands of a
// front's panel carry the front's scale), else e = task.scale_exp.
void launch_gemm_tma(int operands, const GemmTask *tasks, int ntasks, int ntiles, const void *maps, float *C,
                     const int32_t *sexp, int *err, cudaStream_t st, int lo_maps = 0);
// Tensor map of a column-major operand (rows x cols, leading dimension ld elements,
// base 16-byte aligned, ld * element size a multiple of 16) in the box and swizzle
// form that launch_gemm_tma's `operands` variant (0, 1 or 2; both the hi and the lo
// maps for 2) stages; false if the driver refuses it.
bool encode_operand_map(void *out, const void *base, int operands, uint64_t rows, uint64_t cols, uint64_t ld);
// Plain (unswizzled) 2D tensor map of a column-major FP32 / FP64 matrix (rows x cols,
// leading dimension ld elements), box box_rows x box_cols; reads outside the matrix
// are zero.
bool encode_plain_map(void *out, const void *base, int esize, uint64_t rows, uint64_t cols, uint64_t ld,
                      uint32_t box_rows, uint32_t box_cols);
// Power-of-two scale exponent of each listed front's FP16 operand copy, from the
// injected diagonal d: sexp[s] = e with max over the front's rows of sqrt(d) < 2^(e + 12),
// so |L| 2^-e < 2^12 (|L(i, j)| <= sqrt(A(i, i)) for a Cholesky factor).
void launch_front_scale(const int32_t *fronts, int nfronts, SnDev sd, const double *diag, int32_t *sexp,
                        cudaStream_t st);
int gemm_tile_m(bool fp64);
int gemm_tile_n(bool fp64);

// Solves (the factor type T may be float while vectors stay double).
void launch_fwd_asm(const SolveAsmTask *tasks, int ntasks, int ntiles, SnDev sd, double *X, int64_t ldx, int nrhs,
                    double *sol, cudaStream_t st);
template <typename T>
cudaError_t launch_diag(bool forward, const SolveTask *tasks, int ntasks, SnDev sd, const T *factor, double *X,
                        int64_t ldx, int nrhs, int *flags, int *err, cudaStream_t st);
template <typename T>
void launch_str(bool forward, const StrTask *tasks, int ntasks, const StrReduce *red, int nred, SnDev sd,
                const T *factor, double *X, int64_t ldx, int nrhs, double *sol, double *P, cudaStream_t st);
// Superblock diagonal solves (cooperative launch) and the superblock inverses they apply.
template <typename T>
cudaError_t launch_sb_solve(bool forward, const SbTask *tasks, int ntasks, SnDev sd, const T *factor,
                            const void *maps, double *X, int64_t ldx, int nrhs, double *scratch, int *flags, int *err,
                            cudaStream_t st);
template <typename T>
void launch_sb_inverse(const SbTask *tasks, int ntasks, SnDev sd, T *factor, cudaStream_t st);
int solve_rows_per_task();
int diag_blocks_per_task();             // 64-row blocks per diagonal-chain task (one flag each)
// Forward / backward solve of whole subtrees (subs[k] = postorder range [x, y]),
// one CTA per subtree, fronts of at most fmax rows.
template <typename T>
void launch_subtree_solve(bool forward, const int2 *subs, int nsub, int fmax, SnDev sd, const T *factor, double *X,
                          int64_t ldx, int nrhs, double *sol, cudaStream_t st);

// Symmetric block SpMV over permuted reduced rows: Y = A X (both ld = n).
void launch_spmv(const int64_t *ptr, const int64_t *src, const int32_t *col, const int32_t *flag, int64_t nrows,
                 int vb, int src_ld, const double *Ax, const double *X, double *Y, int64_t ld, int nrhs,
                 cudaStream_t st);

// Gather/scatter between the caller's (full or reduced) order and the permuted reduced order.
void launch_gather_rows(const int64_t *map, int64_t n_in, const double *in, int64_t ld_in, double *out,
                        int64_t ld_out, int nrhs, cudaStream_t st);
void launch_scatter_rows(const int64_t *map, int64_t n_out, const double *in, int64_t ld_in, double *out,
                         int64_t ld_out, int nrhs, cudaStream_t st);

// Assembly (K1): Ax[slot*9 + c*3 + r] = sum of contributions in element order.
void launch_assemble_elements(const int64_t *slot_ptr, const int64_t *contrib, int64_t nslots, const double *Ke,
                              double *Ax, cudaStream_t st);

// Refinement / PCG vector kernels (column-wise over nrhs columns, ld = n).
void launch_residual(const double *B, const double *AX, double *R, int64_t n, int nrhs, cudaStream_t st);
void launch_colnorm2(const double *X, int64_t n, int nrhs, double *partials, double *out, cudaStream_t st);
void launch_coldot(const double *X, const double *Y, int64_t n, int nrhs, double *partials, double *out,
                   cudaStream_t st);
void launch_pcg_update_x_r(double *X, double *R, const double *P, const double *AP, const double *rz,
                           const double *pap, const int *active, int64_t n, int nrhs, cudaStream_t st);
void launch_pcg_update_p(double *P, const double *Z, const double *rz_new, const double *rz_old, const int *active,
                         int64_t n, int nrhs, cudaStream_t st);
void launch_copy(double *dst, const double *src, int64_t count, cudaStream_t st);
void launch_axpy(double *y, const double *x, double alpha, int64_t count, cudaStream_t st);

int reduce_partials_count();

}  // namespace mfs
