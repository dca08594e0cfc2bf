// Multi-RHS forward / backward solves (K6) over the lower part of the assembly
// tree, one independent subtree per CTA.
//
// Below the cut level the tree has many small fronts and few rows per front:
// level-by-level kernels there spend their time on launches, barriers and
// load latency rather than on reading L. Here a CTA walks a whole subtree
// (a contiguous postorder range of supernodes) with the front's right-hand
// side block (front rows x up to 4 RHS) held in shared memory:
//   forward  (postorder)  v = [x(cols); 0] + children's u (child order, through
//            child_rel_indices); y = L11^{-1} v[0:w] (64-row blocks through the
//            stored diagonal inverses, or column substitution for fronts factored
//            in shared memory, which then also yields u); u = v[w:f] - L21 y;
//            y -> x, u -> solve arena (read by the parent, later in this CTA or
//            by the level kernels above the cut);
//   backward (reverse postorder) v = [x(cols); x(struct rows)] (ancestors are
//            final); v[0:w] -= L21^T x_struct; x = L11^{-T} v[0:w].
// The next front's panel (ld x w, contiguous) is copied into shared memory with
// cp.async while the current one is solved (panels up to kPanelStageBytes;
// bigger ones are read from global memory). Fronts factored in shared memory
// (no stored inverse) are substituted by one warp per right-hand side. Nothing
// is shared between CTAs, so no flags are needed. Subtrees are assigned
// round-robin in order of decreasing work.
#include "device.h"

#include <algorithm>

namespace mfs {

namespace {

constexpr int kSubThreads = 256;
constexpr int kSubRhs = 4;                 // right-hand sides per pass (more are looped)
constexpr int kSubRed = 4 * kSubRhs * 64;  // split-k partials of a 64-row block
constexpr int kPanelStageBytes = 8192;     // per staging buffer (two buffers); larger ones cost occupancy

__device__ __forceinline__ void sub_cp16(void *dst_smem, const void *src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst_smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void sub_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void sub_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Panel of s staged into buf when it fits (ld x w elements are contiguous and
// 16-byte aligned); returns whether it was staged.
template <typename T>
__device__ __forceinline__ bool stage_panel(int s, const SnDev &sd, const T *factor, T *buf) {
    const int64_t n = int64_t(sd.ld[s]) * sd.w[s];
    if (n * int64_t(sizeof(T)) > kPanelStageBytes) return false;
    const T *src = factor + sd.pan_off[s];
    constexpr int E = 16 / int(sizeof(T));
    for (int q = threadIdx.x; q * E < n; q += blockDim.x) sub_cp16(buf + q * E, src + q * E);
    return true;
}

template <int VB>
__device__ __forceinline__ int crel(const int32_t *rel, int i, int vb) {
    if constexpr (VB > 0) return rel[i / VB] + i % VB;
    return rel[i / vb] + i % vb;
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    return x;
}

// ------------------------------------------------------------------ forward
template <typename T, int VB>
__device__ __forceinline__ void fwd_front(int s, const SnDev &sd, const T *__restrict__ factor, const T *pan,
                                          double *__restrict__ X, int64_t ldx, int nrhs, int rg, int nr,
                                          double *__restrict__ sol, double *v, double *red) {
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    const int w = sd.w[s], d = sd.d[s], f = w + d, c0 = sd.col0[s], ld = sd.ld[s];
    for (int q = tid; q < nr * f; q += nt) {
        const int r = q / f, i = q - r * f;
        v[q] = i < w ? X[c0 + i + int64_t(rg + r) * ldx] : 0.0;
    }
    __syncthreads();
    for (int ci = sd.child_ptr[s]; ci < sd.child_ptr[s + 1]; ++ci) {
        const int c = sd.child_list[ci];
        const int dc = sd.d[c];
        if (dc == 0) continue;
        const int32_t *rel = sd.rel + sd.struct_ptr[c];
        const double *uc = sol + sd.sol_off[c] * nrhs;
        for (int q = tid; q < nr * dc; q += nt) {
            const int r = q / dc, i = q - r * dc;
            v[r * f + crel<VB>(rel, i, sd.vb)] += uc[i + int64_t(rg + r) * dc];
        }
        __syncthreads();
    }
    const int64_t inv = sd.inv_off[s];
    if (inv >= 0) {
        const int nbw = (w + 63) / 64;
        const int i = tid & 63, g = tid >> 6;             // row of the block, k-split group (4)
        for (int rb = 0; rb < nbw; ++rb) {
            const int r0 = rb * 64, nrr = min(64, w - r0);
            if (rb > 0) {
                // v[r0 + i] -= sum_{j < r0} L(r0 + i, j) y_j, j split over the 4 groups
                double acc[kSubRhs] = {0.0, 0.0, 0.0, 0.0};
                if (i < nrr)
                    for (int j = g; j < r0; j += 4) {
                        const double l = double(pan[int64_t(j) * ld + r0 + i]);
#pragma unroll
                        for (int r = 0; r < kSubRhs; ++r)
                            if (r < nr) acc[r] += l * v[r * f + j];
                    }
#pragma unroll
                for (int r = 0; r < kSubRhs; ++r) red[(g * kSubRhs + r) * 64 + i] = acc[r];
                __syncthreads();
                if (g == 0 && i < nrr)
#pragma unroll
                    for (int r = 0; r < kSubRhs; ++r)
                        if (r < nr)
                            v[r * f + r0 + i] -= red[r * 64 + i] + red[(kSubRhs + r) * 64 + i] +
                                                 red[(2 * kSubRhs + r) * 64 + i] + red[(3 * kSubRhs + r) * 64 + i];
                __syncthreads();
            }
            // y = inv(L(rb, rb)) v_block, j split over the 4 groups
            {
                const T *ib = factor + inv + int64_t(rb) * 4096;   // column-major 64 x 64
                double acc[kSubRhs] = {0.0, 0.0, 0.0, 0.0};
                if (i < nrr)
                    for (int j = g; j <= i; j += 4) {
                        const double l = double(ib[j * 64 + i]);
#pragma unroll
                        for (int r = 0; r < kSubRhs; ++r)
                            if (r < nr) acc[r] += l * v[r * f + r0 + j];
                    }
#pragma unroll
                for (int r = 0; r < kSubRhs; ++r) red[(g * kSubRhs + r) * 64 + i] = acc[r];
                __syncthreads();
                if (g == 0 && i < nrr)
#pragma unroll
                    for (int r = 0; r < kSubRhs; ++r)
                        if (r < nr)
                            v[r * f + r0 + i] = red[r * 64 + i] + red[(kSubRhs + r) * 64 + i] +
                                                red[(2 * kSubRhs + r) * 64 + i] + red[(3 * kSubRhs + r) * 64 + i];
                __syncthreads();
            }
        }
        // u = v[w:f] - L21 y
        for (int k = tid; k < d; k += nt) {
            double acc[kSubRhs] = {0.0, 0.0, 0.0, 0.0};
            for (int j = 0; j < w; ++j) {
                const double l = double(pan[int64_t(j) * ld + w + k]);
#pragma unroll
                for (int r = 0; r < kSubRhs; ++r)
                    if (r < nr) acc[r] += l * v[r * f + j];
            }
#pragma unroll
            for (int r = 0; r < kSubRhs; ++r)
                if (r < nr) v[r * f + w + k] -= acc[r];
        }
    } else if (warp < nr) {
        // column substitution over the whole front (y and u together), warp r for rhs r
        double *vr = v + warp * f;
        for (int j = 0; j < w; ++j) {
            const double y = vr[j] / double(pan[int64_t(j) * ld + j]);
            __syncwarp();
            if (lane == 0) vr[j] = y;
            for (int i = j + 1 + lane; i < f; i += 32) vr[i] -= double(pan[int64_t(j) * ld + i]) * y;
            __syncwarp();
        }
    }
    __syncthreads();
    const bool has_u = d > 0 && sd.sol_off[s] >= 0;
    for (int q = tid; q < nr * f; q += nt) {
        const int r = q / f, i = q - r * f;
        if (i < w) X[c0 + i + int64_t(rg + r) * ldx] = v[q];
        else if (has_u) sol[sd.sol_off[s] * nrhs + (i - w) + int64_t(rg + r) * d] = v[q];
    }
    __syncthreads();
}

// ------------------------------------------------------------------ backward
template <typename T, int VB>
__device__ __forceinline__ void bwd_front(int s, const SnDev &sd, const T *__restrict__ factor, const T *pan,
                                          double *__restrict__ X, int64_t ldx, int rg, int nr, double *v) {
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    const int w = sd.w[s], d = sd.d[s], f = w + d, c0 = sd.col0[s], ld = sd.ld[s];
    const int32_t *rows = sd.struct_rows + sd.struct_ptr[s];
    const int vb = sd.vb;
    for (int q = tid; q < nr * f; q += nt) {
        const int r = q / f, i = q - r * f;
        int64_t gi;
        if (i < w) gi = c0 + i;
        else {
            const int li = i - w;
            gi = int64_t(rows[li / (VB > 0 ? VB : vb)]) * (VB > 0 ? VB : vb) + li % (VB > 0 ? VB : vb);
        }
        v[q] = X[gi + int64_t(rg + r) * ldx];
    }
    __syncthreads();
    const int64_t inv = sd.inv_off[s];
    // v[0:w] -= L21^T x_struct: one warp per column, lanes over rows (fronts with
    // inverses; the substitution below covers the struct rows otherwise)
    if (d > 0 && inv >= 0) {
        for (int j = warp; j < w; j += nw) {
            double acc[kSubRhs] = {0.0, 0.0, 0.0, 0.0};
            for (int k = lane; k < d; k += 32) {
                const double l = double(pan[int64_t(j) * ld + w + k]);
#pragma unroll
                for (int r = 0; r < kSubRhs; ++r)
                    if (r < nr) acc[r] += l * v[r * f + w + k];
            }
#pragma unroll
            for (int r = 0; r < kSubRhs; ++r) {
                const double sum = warp_sum(acc[r]);
                if (lane == 0 && r < nr) v[r * f + j] -= sum;
            }
        }
        __syncthreads();
    }
    if (inv >= 0) {
        const int nbw = (w + 63) / 64;
        for (int rb = nbw - 1; rb >= 0; --rb) {
            const int r0 = rb * 64, nrr = min(64, w - r0);
            if (r0 + 64 < w) {
                // v[r0 + j] -= sum_{i >= r0 + 64} L(i, r0 + j) x_i
                for (int j = warp; j < nrr; j += nw) {
                    double acc[kSubRhs] = {0.0, 0.0, 0.0, 0.0};
                    for (int i = r0 + 64 + lane; i < w; i += 32) {
                        const double l = double(pan[int64_t(r0 + j) * ld + i]);
#pragma unroll
                        for (int r = 0; r < kSubRhs; ++r)
                            if (r < nr) acc[r] += l * v[r * f + i];
                    }
#pragma unroll
                    for (int r = 0; r < kSubRhs; ++r) {
                        const double sum = warp_sum(acc[r]);
                        if (lane == 0 && r < nr) v[r * f + r0 + j] -= sum;
                    }
                }
                __syncthreads();
            }
            // x_block = inv(L(rb, rb))^T v_block, one warp per column of the inverse
            const T *ib = factor + inv + int64_t(rb) * 4096;
            for (int j0 = 0; j0 < nrr; j0 += 2 * nw) {          // 2 columns per warp and round
                double out[2][kSubRhs];
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    const int j = j0 + warp + t * nw;
                    double acc[kSubRhs] = {0.0, 0.0, 0.0, 0.0};
                    if (j < nrr)
                        for (int i = j + lane; i < nrr; i += 32) {
                            const double l = double(ib[j * 64 + i]);
#pragma unroll
                            for (int r = 0; r < kSubRhs; ++r)
                                if (r < nr) acc[r] += l * v[r * f + r0 + i];
                        }
#pragma unroll
                    for (int r = 0; r < kSubRhs; ++r) out[t][r] = warp_sum(acc[r]);
                }
                __syncthreads();                              // all reads of this round done
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    const int j = j0 + warp + t * nw;
                    if (lane == 0 && j < nrr)
#pragma unroll
                        for (int r = 0; r < kSubRhs; ++r)
                            if (r < nr) v[r * f + r0 + j] = out[t][r];
                }
                __syncthreads();
            }
        }
    } else if (warp < nr) {
        // left-looking backward substitution, warp r for rhs r:
        // x_j = (v_j - sum_{i > j} L(i, j) x_i) / L_jj over front rows i (struct rows included)
        double *vr = v + warp * f;
        for (int j = w - 1; j >= 0; --j) {
            double acc = 0.0;
            for (int i = j + 1 + lane; i < f; i += 32) acc += double(pan[int64_t(j) * ld + i]) * vr[i];
            acc = warp_sum(acc);
            if (lane == 0) vr[j] = (vr[j] - acc) / double(pan[int64_t(j) * ld + j]);
            __syncwarp();
        }
    }
    __syncthreads();
    for (int q = tid; q < nr * w; q += nt) {
        const int r = q / w, j = q - r * w;
        X[c0 + j + int64_t(rg + r) * ldx] = v[r * f + j];
    }
    __syncthreads();
}

template <typename T, int VB>
__global__ void __launch_bounds__(kSubThreads) subtree_fwd_kernel(const int2 *__restrict__ subs, int nsub, SnDev sd,
                                                                  const T *__restrict__ factor, double *X, int64_t ldx,
                                                                  int nrhs, double *sol) {
    extern __shared__ __align__(16) double sub_smem[];
    T *pbuf = reinterpret_cast<T *>(sub_smem);                       // 2 staging buffers
    double *red = sub_smem + 2 * kPanelStageBytes / 8;
    double *v = red + kSubRed;
    for (int k = blockIdx.x; k < nsub; k += gridDim.x) {
        const int2 sr = subs[k];
        for (int rg = 0; rg < nrhs; rg += kSubRhs) {
            const int nr = min(kSubRhs, nrhs - rg);
            constexpr int PB = kPanelStageBytes / int(sizeof(T));
            bool staged = stage_panel(sr.x, sd, factor, pbuf);
            sub_commit();
            for (int s = sr.x; s <= sr.y; ++s) {
                const int b = (s - sr.x) & 1;
                const bool next = s < sr.y && stage_panel(s + 1, sd, factor, pbuf + (b ^ 1) * PB);
                sub_commit();
                sub_wait1();
                __syncthreads();
                const T *pan = staged ? pbuf + b * PB : factor + sd.pan_off[s];
                fwd_front<T, VB>(s, sd, factor, pan, X, ldx, nrhs, rg, nr, sol, v, red);
                staged = next;
            }
            asm volatile("cp.async.wait_all;" ::: "memory");
            __syncthreads();
        }
    }
}

template <typename T, int VB>
__global__ void __launch_bounds__(kSubThreads) subtree_bwd_kernel(const int2 *__restrict__ subs, int nsub, SnDev sd,
                                                                  const T *__restrict__ factor, double *X, int64_t ldx,
                                                                  int nrhs) {
    extern __shared__ __align__(16) double sub_smem[];
    T *pbuf = reinterpret_cast<T *>(sub_smem);
    double *v = sub_smem + 2 * kPanelStageBytes / 8 + kSubRed;
    for (int k = blockIdx.x; k < nsub; k += gridDim.x) {
        const int2 sr = subs[k];
        for (int rg = 0; rg < nrhs; rg += kSubRhs) {
            const int nr = min(kSubRhs, nrhs - rg);
            constexpr int PB = kPanelStageBytes / int(sizeof(T));
            bool staged = stage_panel(sr.y, sd, factor, pbuf);
            sub_commit();
            for (int s = sr.y; s >= sr.x; --s) {
                const int b = (sr.y - s) & 1;
                const bool next = s > sr.x && stage_panel(s - 1, sd, factor, pbuf + (b ^ 1) * PB);
                sub_commit();
                sub_wait1();
                __syncthreads();
                const T *pan = staged ? pbuf + b * PB : factor + sd.pan_off[s];
                bwd_front<T, VB>(s, sd, factor, pan, X, ldx, rg, nr, v);
                staged = next;
            }
            asm volatile("cp.async.wait_all;" ::: "memory");
            __syncthreads();
        }
    }
}

int sub_sm_count() { return device_sm_count(); }

}  // namespace

size_t subtree_smem_bytes(int fmax) {
    return size_t(2) * kPanelStageBytes + (size_t(kSubRed) + size_t(kSubRhs) * fmax) * sizeof(double);
}

template <typename T>
void launch_subtree_solve(bool forward, const int2 *subs, int nsub, int fmax, SnDev sd, const T *factor, double *X,
                          int64_t ldx, int nrhs, double *sol, cudaStream_t st) {
    if (nsub <= 0) return;
    const size_t smem = subtree_smem_bytes(fmax);
    static PerDeviceOnce once;
    once([] {
        cudaFuncSetAttribute(subtree_fwd_kernel<T, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmemOptin);
        cudaFuncSetAttribute(subtree_fwd_kernel<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmemOptin);
        cudaFuncSetAttribute(subtree_fwd_kernel<T, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmemOptin);
        cudaFuncSetAttribute(subtree_bwd_kernel<T, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmemOptin);
        cudaFuncSetAttribute(subtree_bwd_kernel<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmemOptin);
        cudaFuncSetAttribute(subtree_bwd_kernel<T, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmemOptin);
    });
    const int grid = std::min(nsub, 8 * sub_sm_count());
    ++g_kernel_launches;
    const int vb = sd.vb;
    if (forward) {
        if (vb == 3) subtree_fwd_kernel<T, 3><<<grid, kSubThreads, smem, st>>>(subs, nsub, sd, factor, X, ldx, nrhs, sol);
        else if (vb == 1) subtree_fwd_kernel<T, 1><<<grid, kSubThreads, smem, st>>>(subs, nsub, sd, factor, X, ldx, nrhs, sol);
        else subtree_fwd_kernel<T, 0><<<grid, kSubThreads, smem, st>>>(subs, nsub, sd, factor, X, ldx, nrhs, sol);
    } else {
        if (vb == 3) subtree_bwd_kernel<T, 3><<<grid, kSubThreads, smem, st>>>(subs, nsub, sd, factor, X, ldx, nrhs);
        else if (vb == 1) subtree_bwd_kernel<T, 1><<<grid, kSubThreads, smem, st>>>(subs, nsub, sd, factor, X, ldx, nrhs);
        else subtree_bwd_kernel<T, 0><<<grid, kSubThreads, smem, st>>>(subs, nsub, sd, factor, X, ldx, nrhs);
    }
}

template void launch_subtree_solve<float>(bool, const int2 *, int, int, SnDev, const float *, double *, int64_t, int,
                                          double *, cudaStream_t);
template void launch_subtree_solve<double>(bool, const int2 *, int, int, SnDev, const double *, double *, int64_t,
                                           int, double *, cudaStream_t);

}  // namespace mfs
