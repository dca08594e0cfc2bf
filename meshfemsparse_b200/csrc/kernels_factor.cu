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

// A non-positive (or NaN) pivot. Without perturbation (plain solves, the
// reference's semantics) the smallest failing column is recorded and 1 is used
// so the launch completes; the host then reports the failure. With
// perturbation (the FP32 factor used as a preconditioner under FP64
// refinement) the pivot becomes max(|a|, kPivotFloor * A(col,col)) of the
// injected matrix, which keeps the factor SPD, and the event is counted.
constexpr double kPivotFloor = 1e-3;
template <typename T>
__device__ __forceinline__ T bad_pivot(T a, int col, const PivotCtl &pv, bool record) {
    if (pv.dorig) {
        const T floor_v = T(kPivotFloor * fabs(pv.dorig[col]));
        const T m = fabs(a);
        if (record) atomicAdd(pv.perturbed, 1);
        return (m > floor_v) ? m : (floor_v > T(0) ? floor_v : T(1));
    }
    if (record) atomicMin(pv.fail_col, col);
    return T(1);
}

template <typename T>
__global__ void extract_diag_kernel(const int64_t *__restrict__ diag_off, int64_t n, const T *__restrict__ factor,
                                    double *__restrict__ out) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        out[i] = double(factor[diag_off[i]]);
}

// Small fronts: the whole (w+d)^2 front lives in shared memory.
template <typename T>
__global__ void __launch_bounds__(256) small_factor_kernel(const int32_t *__restrict__ list, SnDev sd,
                                                           T *__restrict__ factor, T *__restrict__ upd,
                                                           PivotCtl pv) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *F = reinterpret_cast<T *>(smem_raw);
    const int s = list[blockIdx.x];
    const int w = sd.w[s], d = sd.d[s], f = w + d;
    const int tid = threadIdx.x, nt = blockDim.x;
    T *pan = factor + sd.pan_off[s];
    const int ld = sd.ld[s];
    const int fw = f * w;
    for (int k = tid; k < f * f; k += nt) F[k] = k < fw ? pan[(k / f) * ld + k % f] : T(0);
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
            if (!(a > T(0))) a = bad_pivot(a, sd.col0[s] + k, pv, true);
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
    for (int k = tid; k < fw; k += nt) pan[(k / f) * ld + k % f] = F[k];
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
// child_rel with the analysis block size known at compile time (1 or 3), else vb.
template <int VB>
__device__ __forceinline__ int child_rel_vb(const int32_t *rel, int i, int vb) {
    if constexpr (VB > 0) return rel[i / VB] + i % VB;
    return rel[i / vb] + i % vb;
}

template <typename T, int VB>
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
    const int ld = sd.ld[s];
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
            // One warp per child column (columns jc0 + warp, + 8, ...), lanes over the
            // rows ic >= jc with 8 read-modify-writes in flight per lane. Targets are
            // distinct (child_rel_indices is injective).
            const int lane = tid & 31, warp = tid >> 5, nwarps = nt >> 5;
            for (int jj = warp; jj < ncols; jj += nwarps) {
                const int jc = jc0 + jj;
                const int rj = child_rel_vb<VB>(rel, jc, vb);
                if (rj < c0 || rj >= c1) continue;
                const T *Ucol = U + int64_t(jc) * dc;
                T *dcol = (rj < w) ? pan + int64_t(rj) * ld : Us + int64_t(rj - w) * d - w;
                for (int ib = jc + lane; ib < dc; ib += 8 * 32) {
                    T v[8], old[8];
                    int ri[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const int ic = ib + 32 * u;
                        ri[u] = -1;
                        if (ic < dc) {
                            ri[u] = child_rel_vb<VB>(rel, ic, vb);
                            v[u] = Ucol[ic];
                        }
                    }
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if (ri[u] >= 0) old[u] = dcol[ri[u]];
#pragma unroll
                    for (int u = 0; u < 8; ++u)
                        if (ri[u] >= 0) dcol[ri[u]] = old[u] + v[u];
                }
            }
        }
        __syncthreads();
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
void launch_small_factor(const int32_t *list, int count, int max_front, SnDev sd, T *factor, T *upd, PivotCtl pv,
                         cudaStream_t st) {
    if (count <= 0) return;
    const size_t smem = size_t(max_front) * max_front * sizeof(T);
    static PerDeviceOnce once;
    once([] { cudaFuncSetAttribute(small_factor_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmemOptin); });
    ++g_kernel_launches;
    small_factor_kernel<T><<<count, 256, smem, st>>>(list, sd, factor, upd, pv);
}

template <typename T>
void launch_assemble_large(const AssembleTask *tasks, int ntasks, int ntiles, SnDev sd, T *factor, T *upd,
                           cudaStream_t st) {
    if (ntiles <= 0) return;
    ++g_kernel_launches;
    if (sd.vb == 3) assemble_large_kernel<T, 3><<<ntiles, 256, 0, st>>>(tasks, ntasks, sd, factor, upd);
    else if (sd.vb == 1) assemble_large_kernel<T, 1><<<ntiles, 256, 0, st>>>(tasks, ntasks, sd, factor, upd);
    else assemble_large_kernel<T, 0><<<ntiles, 256, 0, st>>>(tasks, ntasks, sd, factor, upd);
}

template <typename T>
void launch_extract_diag(const int64_t *diag_off, int64_t n, const T *factor, double *out, cudaStream_t st) {
    if (n <= 0) return;
    ++g_kernel_launches;
    extract_diag_kernel<T><<<grid_for(n, 256), 256, 0, st>>>(diag_off, n, factor, out);
}

#define MFS_INSTANTIATE(T)                                                                                        \
    template void launch_zero<T>(T *, int64_t, cudaStream_t);                                                      \
    template void launch_inject<T>(const PlanEntryDev *, int64_t, int, int, const double *, const double *, double, \
                                   T *, cudaStream_t);                                                            \
    template void launch_diag_shift<T>(const int64_t *, int64_t, double, T *, cudaStream_t);                       \
    template void launch_small_factor<T>(const int32_t *, int, int, SnDev, T *, T *, PivotCtl, cudaStream_t);      \
    template void launch_assemble_large<T>(const AssembleTask *, int, int, SnDev, T *, T *, cudaStream_t);         \
    template void launch_extract_diag<T>(const int64_t *, int64_t, const T *, double *, cudaStream_t);

MFS_INSTANTIATE(double)
MFS_INSTANTIATE(float)


namespace {
// One CTA per front: the largest injected diagonal over the front's rows (its own
// columns and its structure rows), then the exponent that keeps its square root
// below 2^12.
__global__ void __launch_bounds__(256) front_scale_kernel(const int32_t *__restrict__ fronts, SnDev sd,
                                                          const double *__restrict__ diag, int32_t *__restrict__ sexp) {
    const int s = fronts[blockIdx.x];
    const int w = sd.w[s], d = sd.d[s], c0 = sd.col0[s], vb = sd.vb;
    const int32_t *rows = sd.struct_rows + sd.struct_ptr[s];
    double m = 0.0;
    for (int i = threadIdx.x; i < w + d; i += blockDim.x) {
        const int r = i < w ? c0 + i : rows[(i - w) / vb] * vb + (i - w) % vb;
        m = fmax(m, fabs(diag[r]));
    }
    __shared__ double red[256];
    red[threadIdx.x] = m;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double mx = red[0];
        sexp[s] = (mx > 0.0 && isfinite(mx)) ? ilogb(sqrt(mx)) + 1 - 12 : 0;
    }
}
}  // namespace

void launch_front_scale(const int32_t *fronts, int nfronts, SnDev sd, const double *diag, int32_t *sexp,
                        cudaStream_t st) {
    if (nfronts <= 0) return;
    ++g_kernel_launches;
    front_scale_kernel<<<nfronts, 256, 0, st>>>(fronts, sd, diag, sexp);
}

}  // namespace mfs
