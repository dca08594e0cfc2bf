// Level-scheduled multi-RHS triangular solves (K6), one pass over L per
// direction.
//
// Reference: SparseLDL::Solve (forward L y = b, backward L^T x = y; called at
// Solvers/CatamariFactorizer.cc:54,70) with its per-supernode kernels
// (trs_kernels::SolveLowerTri / MultiplyLowerBlock, solve_kernels::fused_forward /
// fused_backward, tests/test_catamari_solve_kernels.cc).
//
// Per elimination-tree level:
//   forward   1. fwd_asm: zero u_s and pull every child's update vector u_c into
//                the front (x rows of the supernode, or u_s) through child_rel_indices,
//                children in order (deterministic, no atomics);
//             2. fwd_tri: one task per 64-row block of every front. A diagonal row
//                block r subtracts L(r, k) y_k for k < r, solves its triangle and
//                publishes y_r through an epoch flag; a structure row block
//                subtracts all L(r, k) y_k into u_s.
//   backward  bwd_tri: one task per diagonal block, descending: subtract
//                L(struct, r)^T x_struct (ancestors are final) and L(k, r)^T x_k for
//                k > r (waiting on their flags), then solve the transposed triangle.
// The tri kernels are cooperative launches (all CTAs co-resident); every CTA
// walks its tasks in ascending order and a task only waits on lower-numbered
// tasks of the same front, so the lowest unfinished task can always proceed.
// Every wait is bounded in time: after kWaitNs the kernel records an error and
// stops waiting (later waits return at once) so the launch always completes;
// the host then reports MFS_TIMEOUT.
#include "device.h"

#include <algorithm>

namespace mfs {

namespace {

constexpr int kRB = 64;                     // rows per task
constexpr int kTriThreads = 128;
constexpr unsigned long long kWaitNs = 2000000000ull;   // 2 s per wait at most

__device__ __forceinline__ int child_rel(const int32_t *rel, int i, int vb) { return rel[i / vb] + i % vb; }

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// thread 0 waits for flag == epoch (bounded), then the whole block proceeds
__device__ __forceinline__ void wait_flag(const int *flag, int epoch, int *err) {
    if (threadIdx.x == 0) {
        if (ld_acquire(flag) != epoch) {
            const unsigned long long t0 = gtimer();
            while (ld_acquire(flag) != epoch) {
                if (*(volatile int *)err) break;
                if (gtimer() - t0 > kWaitNs) {
                    atomicExch(err, 1);
                    break;
                }
                __nanosleep(64);
            }
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(256) fwd_asm_kernel(const SolveAsmTask *__restrict__ tasks, int ntasks, SnDev sd,
                                                      double *__restrict__ X, int64_t ldx, int nrhs,
                                                      double *__restrict__ sol) {
    const int t = blockIdx.x;
    int lo = 0, hi = ntasks - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (tasks[mid].tile_base <= t) lo = mid; else hi = mid - 1;
    }
    const int s = tasks[lo].sn;
    const int chunk = t - tasks[lo].tile_base;
    const int w = sd.w[s], d = sd.d[s], f = w + d;
    const int c0 = sd.col0[s];
    const int r0 = chunk * kSolveAsmRows, r1 = min(f, r0 + kSolveAsmRows);
    double *us = (d > 0 && sd.sol_off[s] >= 0) ? sol + sd.sol_off[s] * nrhs : nullptr;
    const int tid = threadIdx.x, nt = blockDim.x;
    if (us) {
        const int u0 = max(r0, w) - w, u1 = r1 - w;
        if (u1 > u0)
            for (int q = tid; q < (u1 - u0) * nrhs; q += nt) {
                const int r = q / (u1 - u0), i = u0 + q % (u1 - u0);
                us[i + r * d] = 0.0;
            }
    }
    __syncthreads();
    const int vb = sd.vb;
    for (int ci = sd.child_ptr[s]; ci < sd.child_ptr[s + 1]; ++ci) {
        const int c = sd.child_list[ci];
        const int dc = sd.d[c];
        const double *uc = sol + sd.sol_off[c] * nrhs;
        const int32_t *rel = sd.rel + sd.struct_ptr[c];
        const int nblk = dc / vb;
        int a = 0, b = nblk;
        while (a < b) { int mid = (a + b) >> 1; if (rel[mid] + vb - 1 < r0) a = mid + 1; else b = mid; }
        int e = a;
        while (e < nblk && rel[e] < r1) ++e;
        const int i0 = a * vb, n = (e - a) * vb;
        for (int q = tid; q < n * nrhs; q += nt) {
            const int r = q / n, i = i0 + q % n;
            const int ri = child_rel(rel, i, vb);
            if (ri < r0 || ri >= r1) continue;
            const double v = uc[i + r * dc];
            if (ri < w) X[c0 + ri + r * ldx] += v;
            else us[(ri - w) + r * d] += v;
        }
        __syncthreads();
    }
}

// shared memory: acc[kRB * nrhs] | vec[kRB * nrhs] | tile[kRB][kRB + 1]
__host__ __device__ inline size_t tri_smem(int nrhs) {
    return (size_t(2) * kRB * nrhs + size_t(kRB) * (kRB + 1)) * sizeof(double);
}

template <typename T>
__global__ void __launch_bounds__(kTriThreads) fwd_tri_kernel(const SolveTask *__restrict__ tasks, int ntasks, SnDev sd,
                                                              const T *__restrict__ factor, double *__restrict__ X,
                                                              int64_t ldx, int nrhs, double *__restrict__ sol,
                                                              int *__restrict__ flags, int epoch,
                                                              int *__restrict__ err) {
    extern __shared__ __align__(16) double smem_d[];
    double *acc = smem_d;
    double *yk = acc + kRB * nrhs;
    double *tile = yk + kRB * nrhs;            // tile[i * (kRB+1) + j] = L(r0+i, k0+j)
    const int tid = threadIdx.x;
    for (int t = blockIdx.x; t < ntasks; t += gridDim.x) {
        const SolveTask tk = tasks[t];
        const int s = tk.sn;
        const int w = sd.w[s], d = sd.d[s], f = w + d;
        const int c0 = sd.col0[s];
        const int nbw = (w + kRB - 1) / kRB;
        const bool diag = tk.blk < nbw;
        const int r0 = diag ? tk.blk * kRB : w + (tk.blk - nbw) * kRB;
        const int r1 = diag ? min(w, r0 + kRB) : min(f, r0 + kRB);
        const int nr = r1 - r0;
        const T *pan = factor + sd.pan_off[s];
        double *us = (d > 0 && sd.sol_off[s] >= 0) ? sol + sd.sol_off[s] * nrhs : nullptr;
        for (int q = tid; q < nr * nrhs; q += kTriThreads) {
            const int i = q / nrhs, r = q % nrhs;
            acc[q] = diag ? X[c0 + r0 + i + r * ldx] : us[(r0 - w + i) + r * d];
        }
        const int kend = diag ? tk.blk : nbw;
        for (int k = 0; k < kend; ++k) {
            const int k0 = k * kRB, nk = min(kRB, w - k0);
            // the L tile does not depend on the flag: load it first
            for (int q = tid; q < nr * nk; q += kTriThreads) {
                const int j = q / nr, i = q % nr;
                tile[i * (kRB + 1) + j] = double(pan[int64_t(k0 + j) * f + r0 + i]);
            }
            wait_flag(flags + tk.flag_base + k, epoch, err);
            for (int q = tid; q < nk * nrhs; q += kTriThreads) {
                const int j = q / nrhs, r = q % nrhs;
                yk[q] = __ldcg(&X[c0 + k0 + j + r * ldx]);
            }
            __syncthreads();
            for (int q = tid; q < nr * nrhs; q += kTriThreads) {
                const int i = q / nrhs, r = q % nrhs;
                const double *trow = tile + i * (kRB + 1);
                double a = 0.0;
                for (int j = 0; j < nk; ++j) a += trow[j] * yk[j * nrhs + r];
                acc[q] -= a;
            }
            __syncthreads();
        }
        if (diag) {
            for (int q = tid; q < nr * nr; q += kTriThreads) {
                const int j = q / nr, i = q % nr;
                tile[i * (kRB + 1) + j] = i >= j ? double(pan[int64_t(r0 + j) * f + r0 + i]) : 0.0;
            }
            __syncthreads();
            if (tid < 32) {
                for (int j = 0; j < nr; ++j) {
                    const double ljj = tile[j * (kRB + 1) + j];
                    for (int r = tid; r < nrhs; r += 32) acc[j * nrhs + r] /= ljj;
                    __syncwarp();
                    for (int i = j + 1 + tid; i < nr; i += 32) {
                        const double lij = tile[i * (kRB + 1) + j];
                        for (int r = 0; r < nrhs; ++r) acc[i * nrhs + r] -= lij * acc[j * nrhs + r];
                    }
                    __syncwarp();
                }
            }
            __syncthreads();
            for (int q = tid; q < nr * nrhs; q += kTriThreads) {
                const int i = q / nrhs, r = q % nrhs;
                X[c0 + r0 + i + r * ldx] = acc[q];
            }
            __threadfence();
            __syncthreads();
            if (tid == 0) st_release(flags + tk.flag_base + tk.blk, epoch);
        } else {
            __syncthreads();
            for (int q = tid; q < nr * nrhs; q += kTriThreads) {
                const int i = q / nrhs, r = q % nrhs;
                us[(r0 - w + i) + r * d] = acc[q];
            }
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void __launch_bounds__(kTriThreads) bwd_tri_kernel(const SolveTask *__restrict__ tasks, int ntasks, SnDev sd,
                                                              const T *__restrict__ factor, double *__restrict__ X,
                                                              int64_t ldx, int nrhs, int *__restrict__ flags, int epoch,
                                                              int *__restrict__ err) {
    extern __shared__ __align__(16) double smem_d[];
    double *acc = smem_d;
    double *xk = acc + kRB * nrhs;
    double *tile = xk + kRB * nrhs;            // tile[i * (kRB+1) + j] = L(i0+i, r0+j)
    const int tid = threadIdx.x;
    const int vb = sd.vb;
    for (int t = blockIdx.x; t < ntasks; t += gridDim.x) {
        const SolveTask tk = tasks[t];
        const int s = tk.sn;
        const int w = sd.w[s], d = sd.d[s], f = w + d;
        const int c0 = sd.col0[s];
        const int nbw = (w + kRB - 1) / kRB;
        const int r0 = tk.blk * kRB, nr = min(kRB, w - r0);
        const T *pan = factor + sd.pan_off[s];
        const int32_t *rows = sd.struct_rows + sd.struct_ptr[s];
        for (int q = tid; q < nr * nrhs; q += kTriThreads) {
            const int j = q / nrhs, r = q % nrhs;
            acc[q] = X[c0 + r0 + j + r * ldx];
        }
        // chunks: structure rows first (no dependency), then diagonal blocks k > blk, descending
        const int nsc = (d + kRB - 1) / kRB;
        const int nchunks = nsc + (nbw - 1 - tk.blk);
        for (int ch = 0; ch < nchunks; ++ch) {
            const bool st = ch < nsc;
            const int k = st ? -1 : nbw - 1 - (ch - nsc);
            const int i0 = st ? w + ch * kRB : k * kRB;
            const int ni = st ? min(kRB, f - i0) : min(kRB, w - i0);
            for (int q = tid; q < ni * nr; q += kTriThreads) {
                const int j = q / ni, i = q % ni;
                tile[i * (kRB + 1) + j] = double(pan[int64_t(r0 + j) * f + i0 + i]);
            }
            if (!st) wait_flag(flags + tk.flag_base + k, epoch, err);
            for (int q = tid; q < ni * nrhs; q += kTriThreads) {
                const int i = q / nrhs, r = q % nrhs;
                if (st) {
                    const int li = i0 - w + i;
                    const int64_t gi = int64_t(rows[li / vb]) * vb + li % vb;
                    xk[q] = X[gi + r * ldx];
                } else {
                    xk[q] = __ldcg(&X[c0 + i0 + i + r * ldx]);
                }
            }
            __syncthreads();
            for (int q = tid; q < nr * nrhs; q += kTriThreads) {
                const int j = q / nrhs, r = q % nrhs;
                double a = 0.0;
                for (int i = 0; i < ni; ++i) a += tile[i * (kRB + 1) + j] * xk[i * nrhs + r];
                acc[q] -= a;
            }
            __syncthreads();
        }
        // transposed triangle: x_j = (acc_j - sum_{i>j} L(i,j) x_i) / L(j,j), descending
        for (int q = tid; q < nr * nr; q += kTriThreads) {
            const int j = q / nr, i = q % nr;
            tile[i * (kRB + 1) + j] = i >= j ? double(pan[int64_t(r0 + j) * f + r0 + i]) : 0.0;
        }
        __syncthreads();
        if (tid < 32) {
            for (int j = nr - 1; j >= 0; --j) {
                for (int r = tid; r < nrhs; r += 32) acc[j * nrhs + r] /= tile[j * (kRB + 1) + j];
                __syncwarp();
                for (int i = tid; i < j; i += 32) {
                    const double lji = tile[j * (kRB + 1) + i];
                    for (int r = 0; r < nrhs; ++r) acc[i * nrhs + r] -= lji * acc[j * nrhs + r];
                }
                __syncwarp();
            }
        }
        __syncthreads();
        for (int q = tid; q < nr * nrhs; q += kTriThreads) {
            const int j = q / nrhs, r = q % nrhs;
            X[c0 + r0 + j + r * ldx] = acc[q];
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) st_release(flags + tk.flag_base + tk.blk, epoch);
        __syncthreads();
    }
}

int sm_count() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    return sms;
}

template <typename K>
int coop_grid(K kernel, size_t smem, int ntasks) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTriThreads, smem);
    const int g = std::max(1, per_sm) * sm_count();
    return std::min(g, std::max(1, ntasks));
}

}  // namespace

void launch_fwd_asm(const SolveAsmTask *tasks, int ntasks, int ntiles, SnDev sd, double *X, int64_t ldx, int nrhs,
                    double *sol, cudaStream_t st) {
    if (ntiles <= 0) return;
    ++g_kernel_launches;
    fwd_asm_kernel<<<ntiles, 256, 0, st>>>(tasks, ntasks, sd, X, ldx, nrhs, sol);
}

template <typename T>
cudaError_t launch_fwd_tri(const SolveTask *tasks, int ntasks, SnDev sd, const T *factor, double *X, int64_t ldx,
                           int nrhs, double *sol, int *flags, int epoch, int *err, cudaStream_t st) {
    if (ntasks <= 0) return cudaSuccess;
    auto kern = fwd_tri_kernel<T>;
    const size_t smem = tri_smem(nrhs);
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tri_smem(kMaxSolveRhs)));
    const int grid = coop_grid(kern, smem, ntasks);
    void *args[] = {(void *)&tasks, (void *)&ntasks, (void *)&sd, (void *)&factor, (void *)&X, (void *)&ldx,
                    (void *)&nrhs, (void *)&sol, (void *)&flags, (void *)&epoch, (void *)&err};
    ++g_kernel_launches;
    return cudaLaunchCooperativeKernel((void *)kern, dim3(grid), dim3(kTriThreads), args, smem, st);
}

template <typename T>
cudaError_t launch_bwd_tri(const SolveTask *tasks, int ntasks, SnDev sd, const T *factor, double *X, int64_t ldx,
                           int nrhs, int *flags, int epoch, int *err, cudaStream_t st) {
    if (ntasks <= 0) return cudaSuccess;
    auto kern = bwd_tri_kernel<T>;
    const size_t smem = tri_smem(nrhs);
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(tri_smem(kMaxSolveRhs)));
    const int grid = coop_grid(kern, smem, ntasks);
    void *args[] = {(void *)&tasks, (void *)&ntasks, (void *)&sd, (void *)&factor, (void *)&X, (void *)&ldx,
                    (void *)&nrhs, (void *)&flags, (void *)&epoch, (void *)&err};
    ++g_kernel_launches;
    return cudaLaunchCooperativeKernel((void *)kern, dim3(grid), dim3(kTriThreads), args, smem, st);
}

template cudaError_t launch_fwd_tri<double>(const SolveTask *, int, SnDev, const double *, double *, int64_t, int,
                                            double *, int *, int, int *, cudaStream_t);
template cudaError_t launch_fwd_tri<float>(const SolveTask *, int, SnDev, const float *, double *, int64_t, int,
                                           double *, int *, int, int *, cudaStream_t);
template cudaError_t launch_bwd_tri<double>(const SolveTask *, int, SnDev, const double *, double *, int64_t, int,
                                            int *, int, int *, cudaStream_t);
template cudaError_t launch_bwd_tri<float>(const SolveTask *, int, SnDev, const float *, double *, int64_t, int,
                                           int *, int, int *, cudaStream_t);

int solve_rows_per_task() { return kRB; }

}  // namespace mfs
