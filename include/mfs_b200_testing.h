/* Test hooks of libmfs_b200.so.
 *
 * These entry points have no counterpart in the reference: they expose single
 * kernels of the numeric factorization so that tests can check them against a
 * host computation on crafted inputs (edge tiles, operand alignment shifts,
 * lower-triangle masks), the way tests/test_catamari_solve_kernels.cc checks
 * catamari's dense kernels against dense references. They are not part of the
 * factorizer interface and are not needed by callers of it.
 */
#ifndef MFS_B200_TESTING_H
#define MFS_B200_TESTING_H

#include "mfs_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Fields of one Schur-update GEMM task, in this order (int64 each). */
#define MFS_GEMM_TASK_FIELDS 12
/* a_off, b_off, c_off, lda, ldb, ldc, m, n, k, lower, mode, scale_exp:
 *   mode 0:  C(i,j) -= 2^scale_exp sum_k A(i,k) B(j,k)     mode 1:  C(i,j) = sum_k A(i,k) B(j,k)
 *   for i < m, j < n (lower = 1: only i >= j), A, B, C column-major at the given
 *   offsets (elements) of the arrays A, B, C of a_len, b_len, c_len elements.
 *
 * Runs one launch of the factorization's GEMM kernel over all tasks on `device`
 * (device pointers; the call synchronizes the device). precision MFS_PREC_FP32:
 * float arrays, `kernel` 1 = single-pass TF32 on the 5th-generation tensor cores
 * (tcgen05), 4 = the same with TMA-fed operands (mode 0 only; arrays 16-byte
 * aligned), 5 = FP16 A and B (IEEE half arrays, leading dimensions multiples of 8)
 * with FP32 C on tcgen05 with TMA (mode 0 only; scale_exp is used by kernels 5 and
 * 6 only), 6 = split FP16: A and B each hold an FP16 hi array of a_len / 2 (b_len / 2)
 * elements followed by the lo array (A ~ hi + 2^-11 lo), offsets index either half;
 * three MMAs per k slice (mode 0 only), 7 = split TF32 on tcgen05 (float arrays, hi /
 * lo split in shared memory, the row-solve kernel of tensor_cores 6; mode 1 writes
 * its half copies to scratch), 3 = split 3xTF32 (mma.sync), 0 = single-pass TF32
 * (mma.sync);
 * MFS_PREC_FP64: double arrays on the FP64 tensor cores (kernel ignored).
 * FP32 leading dimensions must be multiples of 4 (16-byte aligned columns, as
 * the factor's panels are). Every access is checked against the array lengths
 * (elements of each array's type) before the launch (MFS_INVALID_ARG otherwise). */
mfs_status mfs_debug_gemm(int32_t device, int32_t precision, int32_t kernel, int64_t ntasks,
                          const int64_t *tasks, const void *A, int64_t a_len, const void *B, int64_t b_len,
                          void *C, int64_t c_len, char *err_buf, size_t err_len);

/* Per-launch record of the last numeric factorization run with time_kernels = 1:
 * for each tensor-core GEMM launch (in launch order) out[5 i .. 5 i + 4] = {CUDA-event
 * ms, algorithmic flops, CTA tiles, tasks, kind}; kind 0 = left-looking update inside
 * a column-block group, 1 = row solve, 2 = update of the next group's columns, 3 =
 * trailing update of the columns after it, 4 = the level's Schur-complement SYRK.
 * *count receives the number of launches; at most max_launches are written. */
mfs_status mfs_debug_gemm_launches(const mfs_handle *h, int64_t max_launches, double *out, int64_t *count);

/* The temporal nested-dissection reuse rule on its own (host only, no device): for a
 * previous separator forest (ncomp components, cparent postordered with -1 for roots,
 * cmember[v] the component of vertex v) and a new symmetric graph on the same n
 * vertices (CSR xadj / adj, self loops allowed), *full_rebuild = 1 when a full
 * dissection is needed, else the violated subtree roots go to roots[0 .. *nroots)
 * (ascending; roots holds ncomp entries). Replaces no reference entry point: it
 * exposes PersistentSeparatorTree::dirty_subtrees
 * (ParallelNestedDissection/persistent_separator_tree.hh:81-118) for its tests. */
mfs_status mfs_debug_dirty_subtrees(int64_t n, const int64_t *xadj, const int64_t *adj, int64_t ncomp,
                                    const int64_t *cparent, const int64_t *cmember, int32_t *full_rebuild,
                                    int64_t *roots, int64_t *nroots);

/* The hierarchical constrained-minimum-degree final order on its own (host only): for a
 * symmetric graph (CSR, n vertices) and a separator forest (ncomp components, cparent
 * postordered, cmember per vertex), the order at cut_depth (clamped to the forest's
 * depth) into perm[0 .. n) (new -> old) and stats[4] = {effective cut depth, subtree
 * problems, vertices above the cut, boundary cliques passed to the upper problem}.
 * MFS_INVALID_ARG when the forest does not fit the graph (an edge between two subtrees
 * of the cut, or between components that are not ancestor and descendant). Replaces no
 * reference entry point: it exposes the stage hierarchical_camd
 * (ParallelNestedDissection/hierarchical_camd.cc:165-333) stands for, for its tests. */
mfs_status mfs_debug_hierarchical_order(int64_t n, const int64_t *xadj, const int64_t *adj, int64_t ncomp,
                                        const int64_t *cparent, const int64_t *cmember, int32_t cut_depth,
                                        int64_t *perm, int64_t *stats);

#ifdef __cplusplus
}
#endif

#endif /* MFS_B200_TESTING_H */
