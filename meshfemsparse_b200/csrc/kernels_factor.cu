// Numeric factorization kernels (K2 value injection, K3 POTRF, K4 TRSM,
// K5 Schur update + extend-add) for the multifrontal, level-scheduled
// supernodal Cholesky factorization.
//
// The reference delegates this stage to BlockCatamari's
// SparseLDL::RefactorWithFixedSparsityPattern (called at
// Solvers/CatamariFactorizer.cc:660): inject A (+ sigma I or sigma B) through
// the conversion plan, then a right-looking supernodal Cholesky where every
// supernode's Schur complement is merged into its parent through
// child_rel_indices. The GPU restatement keeps that structure:
//   * one injection pass over the plan (CatamariConversionPlan.hh:524-525);
//   * per elimination-tree level, small fronts are factored by one CTA each in
//     shared memory; large fronts run as tiled POTRF / TRSM / update kernels
//     whose task lists cover every large front of the level at once;
//   * a parent pulls its children's update matrices in child order
//     (deterministic, no atomics), so results are bit-identical run to run.
// Pivot failures never trap: the smallest failing column is recorded and the
// pivot replaced by 1 so the launch completes; the host turns it into
// the reference's "pivots successful" error (CatamariFactorizer.cc:701-705).
#include "device.h"

#include <cstdio>

namespace mfs {

namespace {

template <typename T>
__device__ __forceinline__ T dev_sqrt(T x);
template <>
__device__ __forceinline__ double dev_sqrt<double>(double x) { return sqrt(x); }
template <>
__device__ __forceinline__ float dev_sqrt<float>(float x) { return sqrtf(x); }

template <typename T>
__global__ void zero_kernel(T *p, int64_t n) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        p[i] = T(0);
}

// K2: one thread per (plan entry, block component).
template <typename T>
__global__ void inject_kernel(const PlanEntryDev *__restrict__ plan, int64_t nplan, int vb, int src_ld,
                              const double *__restrict__ Ax, const double *__restrict__ Bx, double sigma_b,
                              T *__restrict__ factor) {
    const int vb2 = vb * vb;
    const int64_t total = nplan * vb2;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t e = t / vb2;
        const int comp = int(t - e * vb2);
        const int r = comp % vb, c = comp / vb;
        const PlanEntryDev pe = plan[e];
        if ((pe.flags & 2) && r < c) continue;   // diagonal block: lower part only
        const int64_t so = (pe.flags & 1) ? pe.src + int64_t(r) * src_ld + c : pe.src + int64_t(c) * src_ld + r;
        double v = Ax[so];
        if (Bx) v += sigma_b * Bx[so];
        factor[pe.dst + int64_t(c) * pe.ld + r] = T(v);
    }
}

template <typename T>
__global__ void diag_shift_kernel(const int64_t *__restrict__ diag_off, int64_t n, double sigma, T *factor) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        factor[diag_off[i]] = T(double(factor[diag_off[i]]) + sigma);
}

__device__ __forceinline__ int child_rel(const int32_t *rel, int i, int vb) { return rel[i / vb] + i % vb; }

// Small fronts: the whole (w+d)^2 front lives in shared memory.
template <typename T>
__global__ void __launch_bounds__(256) small_factor_kernel(const int32_t *__restrict__ list, SnDev sd,
                                                           T *__restrict__ factor, T *__restrict__ upd,
                                                           int *__restrict__ fail_col) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *F = reinterpret_cast<T *>(smem_raw);
    const int s = list[blockIdx.x];
    const int w = sd.w[s], d = sd.d[s], f = w + d;
    const int tid = threadIdx.x, nt = blockDim.x;
    T *pan = factor + sd.pan_off[s];
    const int fw = f * w;
    for (int k = tid; k < f * f; k += nt) F[k] = k < fw ? pan[k] : T(0);
    __syncthreads();
    const int vb = sd.vb;
    for (int ci = sd.child_ptr[s]; ci < sd.child_ptr[s + 1]; ++ci) {
        const int c = sd.child_list[ci];
        const int dc = sd.d[c];
        const T *U = upd + sd.upd_off[c];
        const int32_t *rel = sd.rel + sd.struct_ptr[c];
        for (int k = tid; k < dc * dc; k += nt) {
            const int j = k / dc, i = k - j * dc;
            if (i < j) continue;
            F[child_rel(rel, j, vb) * f + child_rel(rel, i, vb)] += U[k];
        }
        __syncthreads();
    }
    for (int k = 0; k < w; ++k) {
        T *colk = F + k * f;
        if (tid == 0) {
            T a = colk[k];
            if (!(a > T(0))) { atomicMin(fail_col, sd.col0[s] + k); a = T(1); }
            colk[k] = dev_sqrt(a);
        }
        __syncthreads();
        const T piv = colk[k];
        for (int i = k + 1 + tid; i < f; i += nt) colk[i] = colk[i] / piv;
        __syncthreads();
        const int m = f - k - 1;
        for (int t = tid; t < m * m; t += nt) {
            const int jj = t / m, ii = t - jj * m;
            if (ii < jj) continue;
            const int j = k + 1 + jj, i = k + 1 + ii;
            F[j * f + i] -= colk[i] * colk[j];
        }
        __syncthreads();
    }
    for (int k = tid; k < fw; k += nt) pan[k] = F[k];
    if (d > 0 && sd.upd_off[s] >= 0) {
        T *U = upd + sd.upd_off[s];
        for (int k = tid; k < d * d; k += nt) {
            const int j = k / d, i = k - j * d;
            U[k] = F[(w + j) * f + (w + i)];
        }
    }
}

// Large fronts: zero U_s and extend-add every child into the columns
// [c0, c0 + kAsmCols) of the front (panel part or U_s part).
template <typename T>
__global__ void __launch_bounds__(256) assemble_large_kernel(const AssembleTask *__restrict__ tasks, int ntasks,
                                                             SnDev sd, T *__restrict__ factor,
                                                             T *__restrict__ upd) {
    const int t = blockIdx.x;
    int lo = 0, hi = ntasks - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (tasks[mid].tile_base <= t) lo = mid; else hi = mid - 1;
    }
    const int s = tasks[lo].sn;
    const int chunk = t - tasks[lo].tile_base;
    const int w = sd.w[s], d = sd.d[s], f = w + d;
    const int c0 = chunk * kAsmCols, c1 = min(f, c0 + kAsmCols);
    T *pan = factor + sd.pan_off[s];
    T *Us = (d > 0 && sd.upd_off[s] >= 0) ? upd + sd.upd_off[s] : nullptr;
    const int tid = threadIdx.x, nt = blockDim.x;
    // zero the U_s columns of this chunk
    if (Us) {
        const int u0 = max(c0, w) - w, u1 = c1 - w;
        for (int64_t k = int64_t(u0) * d + tid; k < int64_t(max(u1, u0)) * d; k += nt) Us[k] = T(0);
    }
    __syncthreads();
    const int vb = sd.vb;
    for (int ci = sd.child_ptr[s]; ci < sd.child_ptr[s + 1]; ++ci) {
        const int c = sd.child_list[ci];
        const int dc = sd.d[c];
        const T *U = upd + sd.upd_off[c];
        const int32_t *rel = sd.rel + sd.struct_ptr[c];
        const int nblk = dc / vb;
        // first block entry whose last scalar column reaches c0
        int a = 0, b = nblk;
        while (a < b) { int mid = (a + b) >> 1; if (rel[mid] + vb - 1 < c0) a = mid + 1; else b = mid; }
        int e = a;
        while (e < nblk && rel[e] < c1) ++e;
        const int jc0 = a * vb, jc1 = e * vb;
        const int ncols = jc1 - jc0;
        if (ncols > 0) {
            // pairs (jc, ic) with ic >= jc; iterate jc-major
            for (int jj = 0; jj < ncols; ++jj) {
                const int jc = jc0 + jj;
                const int rj = child_rel(rel, jc, vb);
                if (rj < c0 || rj >= c1) continue;
                const T *Ucol = U + int64_t(jc) * dc;
                for (int ic = jc + tid; ic < dc; ic += nt) {
                    const int ri = child_rel(rel, ic, vb);
                    const T v = Ucol[ic];
                    if (rj < w) pan[int64_t(rj) * f + ri] += v;
                    else Us[int64_t(rj - w) * d + (ri - w)] += v;
                }
            }
        }
        __syncthreads();
    }
}

// K3: Cholesky of one nb x nb diagonal block per CTA.
template <typename T>
__global__ void __launch_bounds__(256) potrf_kernel(const PotrfTask *__restrict__ tasks, T *__restrict__ factor,
                                                    int *__restrict__ fail_col) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *S = reinterpret_cast<T *>(smem_raw);
    const PotrfTask tk = tasks[blockIdx.x];
    const int nb = tk.nb, ld = tk.ld;
    T *blk = factor + tk.off;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int k = tid; k < nb * nb; k += nt) {
        const int j = k / nb, i = k - j * nb;
        S[k] = i >= j ? blk[int64_t(j) * ld + i] : T(0);
    }
    __syncthreads();
    for (int k = 0; k < nb; ++k) {
        T *colk = S + k * nb;
        if (tid == 0) {
            T a = colk[k];
            if (!(a > T(0))) { atomicMin(fail_col, tk.col + k); a = T(1); }
            colk[k] = dev_sqrt(a);
        }
        __syncthreads();
        const T piv = colk[k];
        for (int i = k + 1 + tid; i < nb; i += nt) colk[i] = colk[i] / piv;
        __syncthreads();
        const int m = nb - k - 1;
        for (int t = tid; t < m * m; t += nt) {
            const int jj = t / m, ii = t - jj * m;
            if (ii < jj) continue;
            S[(k + 1 + jj) * nb + (k + 1 + ii)] -= colk[k + 1 + ii] * colk[k + 1 + jj];
        }
        __syncthreads();
    }
    for (int k = tid; k < nb * nb; k += nt) {
        const int j = k / nb, i = k - j * nb;
        if (i >= j) blk[int64_t(j) * ld + i] = S[k];
    }
}

// K4: rows below a factored diagonal block, X L^T = B, one thread per row.
template <typename T>
__global__ void __launch_bounds__(kTrsmRows) trsm_kernel(const TrsmTask *__restrict__ tasks, int ntasks,
                                                          T *__restrict__ factor) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int t = blockIdx.x;
    int lo = 0, hi = ntasks - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (tasks[mid].tile_base <= t) lo = mid; else hi = mid - 1;
    }
    const TrsmTask tk = tasks[lo];
    const int tile = t - tk.tile_base;
    const int nb = tk.nb, ld = tk.ld;
    T *L = reinterpret_cast<T *>(smem_raw);             // nb x nb
    T *B = L + nb * nb;                                 // kTrsmRows x (nb+1), row-major
    const int bld = nb + 1;
    const int tid = threadIdx.x;
    for (int k = tid; k < nb * nb; k += blockDim.x) {
        const int j = k / nb, i = k - j * nb;
        L[k] = i >= j ? factor[tk.l_off + int64_t(j) * ld + i] : T(0);
    }
    const int r0 = tile * kTrsmRows;
    const int rows = min(kTrsmRows, tk.m - r0);
    for (int k = tid; k < kTrsmRows * nb; k += blockDim.x) {
        const int j = k / kTrsmRows, i = k - j * kTrsmRows;
        if (i < rows) B[i * bld + j] = factor[tk.b_off + int64_t(j) * ld + r0 + i];
    }
    __syncthreads();
    if (tid < rows) {
        T *x = B + tid * bld;
        for (int j = 0; j < nb; ++j) {
            T acc = x[j];
            for (int k = 0; k < j; ++k) acc -= x[k] * L[k * nb + j];
            x[j] = acc / L[j * nb + j];
        }
    }
    __syncthreads();
    for (int k = tid; k < kTrsmRows * nb; k += blockDim.x) {
        const int j = k / kTrsmRows, i = k - j * kTrsmRows;
        if (i < rows) factor[tk.b_off + int64_t(j) * ld + r0 + i] = B[i * bld + j];
    }
}

// K5: C(i,j) -= sum_k A(i,k) A(j,k), 64x64 tile per CTA, FMA path.
template <typename T>
__global__ void __launch_bounds__(256) gemm_update_kernel(const GemmTask *__restrict__ tasks, int ntasks,
                                                          const T *__restrict__ A, T *__restrict__ C) {
    const int t = blockIdx.x;
    int lo = 0, hi = ntasks - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (tasks[mid].tile_base <= t) lo = mid; else hi = mid - 1;
    }
    const GemmTask tk = tasks[lo];
    const int local = t - tk.tile_base;
    const int ti = local % tk.tiles_m, tj = local / tk.tiles_m;
    const int i0 = ti * kGemmTile, j0 = tj * kGemmTile;
    if (tk.lower && i0 + kGemmTile - 1 < j0) return;
    constexpr int KC = 16;
    __shared__ T As[KC][kGemmTile + 1];
    __shared__ T Bs[KC][kGemmTile + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    T acc[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) acc[r][c] = T(0);
    const T *Aa = A + tk.a_off;
    const T *Ab = A + tk.b_off;
    for (int k0 = 0; k0 < tk.k; k0 += KC) {
        for (int l = threadIdx.x; l < KC * kGemmTile; l += 256) {
            const int kk = l / kGemmTile, ii = l - kk * kGemmTile;
            const int gk = k0 + kk;
            const int gi = i0 + ii, gj = j0 + ii;
            As[kk][ii] = (gi < tk.m && gk < tk.k) ? Aa[int64_t(gk) * tk.lda + gi] : T(0);
            Bs[kk][ii] = (gj < tk.n && gk < tk.k) ? Ab[int64_t(gk) * tk.lda + gj] : T(0);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < KC; ++kk) {
            T a[4], b[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) a[r] = As[kk][tx + 16 * r];
#pragma unroll
            for (int c = 0; c < 4; ++c) b[c] = Bs[kk][ty + 16 * c];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] += a[r] * b[c];
        }
        __syncthreads();
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int j = j0 + ty + 16 * c;
        if (j >= tk.n) continue;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int i = i0 + tx + 16 * r;
            if (i >= tk.m || (tk.lower && i < j)) continue;
            C[tk.c_off + int64_t(j) * tk.ldc + i] -= acc[r][c];
        }
    }
}

inline int grid_for(int64_t n, int threads) {
    int64_t g = (n + threads - 1) / threads;
    if (g > 148 * 32) g = 148 * 32;
    if (g < 1) g = 1;
    return int(g);
}

}  // namespace

template <typename T>
void launch_zero(T *p, int64_t n, cudaStream_t st) {
    if (n <= 0) return;
    ++g_kernel_launches;
    zero_kernel<T><<<grid_for(n, 256), 256, 0, st>>>(p, n);
}

template <typename T>
void launch_inject(const PlanEntryDev *plan, int64_t nplan, int vb, int src_ld, const double *Ax, const double *Bx,
                   double sigma_b, T *factor, cudaStream_t st) {
    if (nplan <= 0) return;
    ++g_kernel_launches;
    inject_kernel<T><<<grid_for(nplan * vb * vb, 256), 256, 0, st>>>(plan, nplan, vb, src_ld, Ax, Bx, sigma_b,
                                                                      factor);
}

template <typename T>
void launch_diag_shift(const int64_t *diag_off, int64_t n, double sigma, T *factor, cudaStream_t st) {
    if (n <= 0) return;
    ++g_kernel_launches;
    diag_shift_kernel<T><<<grid_for(n, 256), 256, 0, st>>>(diag_off, n, sigma, factor);
}

template <typename T>
void launch_small_factor(const int32_t *list, int count, int max_front, SnDev sd, T *factor, T *upd, int *fail_col,
                         cudaStream_t st) {
    if (count <= 0) return;
    const size_t smem = size_t(max_front) * max_front * sizeof(T);
    cudaFuncSetAttribute(small_factor_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    ++g_kernel_launches;
    small_factor_kernel<T><<<count, 256, smem, st>>>(list, sd, factor, upd, fail_col);
}

template <typename T>
void launch_assemble_large(const AssembleTask *tasks, int ntasks, int ntiles, SnDev sd, T *factor, T *upd,
                           cudaStream_t st) {
    if (ntiles <= 0) return;
    ++g_kernel_launches;
    assemble_large_kernel<T><<<ntiles, 256, 0, st>>>(tasks, ntasks, sd, factor, upd);
}

template <typename T>
void launch_potrf(const PotrfTask *tasks, int ntasks, int max_nb, T *factor, int *fail_col, cudaStream_t st) {
    if (ntasks <= 0) return;
    const size_t smem = size_t(max_nb) * max_nb * sizeof(T);
    cudaFuncSetAttribute(potrf_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    ++g_kernel_launches;
    potrf_kernel<T><<<ntasks, 256, smem, st>>>(tasks, factor, fail_col);
}

template <typename T>
void launch_trsm(const TrsmTask *tasks, int ntasks, int ntiles, int max_nb, T *factor, cudaStream_t st) {
    if (ntiles <= 0) return;
    const size_t smem = (size_t(max_nb) * max_nb + size_t(kTrsmRows) * (max_nb + 1)) * sizeof(T);
    cudaFuncSetAttribute(trsm_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    ++g_kernel_launches;
    trsm_kernel<T><<<ntiles, kTrsmRows, smem, st>>>(tasks, ntasks, factor);
}

template <typename T>
void launch_gemm_update(const GemmTask *tasks, int ntasks, int ntiles, const T *a, T *c, int use_tc,
                        cudaStream_t st) {
    (void)use_tc;
    if (ntiles <= 0) return;
    ++g_kernel_launches;
    gemm_update_kernel<T><<<ntiles, 256, 0, st>>>(tasks, ntasks, a, c);
}

#define MFS_INSTANTIATE(T)                                                                                        \
    template void launch_zero<T>(T *, int64_t, cudaStream_t);                                                      \
    template void launch_inject<T>(const PlanEntryDev *, int64_t, int, int, const double *, const double *, double, \
                                   T *, cudaStream_t);                                                            \
    template void launch_diag_shift<T>(const int64_t *, int64_t, double, T *, cudaStream_t);                       \
    template void launch_small_factor<T>(const int32_t *, int, int, SnDev, T *, T *, int *, cudaStream_t);         \
    template void launch_assemble_large<T>(const AssembleTask *, int, int, SnDev, T *, T *, cudaStream_t);         \
    template void launch_potrf<T>(const PotrfTask *, int, int, T *, int *, cudaStream_t);                          \
    template void launch_trsm<T>(const TrsmTask *, int, int, int, T *, cudaStream_t);                              \
    template void launch_gemm_update<T>(const GemmTask *, int, int, const T *, T *, int, cudaStream_t);

MFS_INSTANTIATE(double)
MFS_INSTANTIATE(float)

}  // namespace mfs
