// Level-scheduled multi-RHS triangular solves (K6), one pass over L per
// direction.
//
// Reference: SparseLDL::Solve (forward L y = b, backward L^T x = y; called at
// Solvers/CatamariFactorizer.cc:54,70) with its per-supernode kernels
// (trs_kernels::SolveLowerTri / MultiplyLowerBlock, solve_kernels::fused_forward /
// fused_backward, tests/test_catamari_solve_kernels.cc).
//
// A front of supernode s is [L11; L21] (w + d rows, w columns). Per level:
//   forward   fwd_asm      zero u_s and pull every child's update vector u_c into the
//                          front through child_rel_indices (children in order);
//             fwd_diag     L11 y = v, one task per pair of 64-row diagonal blocks; a
//                          pair subtracts L11(rows, k) y_k for every earlier block k
//                          (waiting on block k's epoch flag) and solves its two
//                          triangles inside the CTA, publishing each block's flag;
//             str_fwd      P = L21(rows, chunk) y(chunk) for 1024-row slabs of L21 and
//                          256-column chunks (independent tasks);
//             fwd_reduce   u_s(rows) -= sum over chunks of P, in chunk order.
//   backward  str_bwd      P = L21(chunk, cols)^T x_struct for 64-column blocks and
//                          2048-row (FP64: 1024-row) chunks of L21 (ancestors are final);
//             bwd_reduce   x(cols) -= sum over chunks of P, in chunk order;
//             bwd_diag     L11^T x = y, pairs and blocks descending, waiting on flags.
// Everything is summed in a fixed order: results are run-to-run identical.
// The diag kernels are cooperative launches (all CTAs co-resident); every CTA
// walks its tasks in ascending order and a task only waits on lower-numbered
// tasks of the same front, so the lowest unfinished task can always proceed.
// Every wait is bounded in time (kWaitNs): on expiry the kernel records an
// error and stops waiting so the launch completes; the host reports MFS_TIMEOUT.
// Flags are cleared before each solve; the forward pass publishes epoch 1 and
// the backward pass epoch 2, so the launch sequence is fixed (graph-capturable).
#include "device.h"

#include <algorithm>
#include <type_traits>

namespace mfs {

namespace {

constexpr int kRB = 64;                     // rows / columns per task
constexpr int kDG = 2;                      // 64-row blocks per diagonal-chain task (one flag per task)
constexpr int kDiagThreads = 256;
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
        // 4 independent read-modify-writes in flight per thread (targets are distinct)
        for (int q0 = tid; q0 < n * nrhs; q0 += 4 * nt) {
            double v[4], old[4];
            double *dst[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                dst[u] = nullptr;
                const int q = q0 + u * nt;
                if (q < n * nrhs) {
                    const int r = q / n, i = i0 + q % n;
                    const int ri = child_rel(rel, i, vb);
                    if (ri >= r0 && ri < r1) {
                        v[u] = uc[i + r * dc];
                        dst[u] = (ri < w) ? X + c0 + ri + r * ldx : us + (ri - w) + r * d;
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (dst[u]) old[u] = *dst[u];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (dst[u]) *dst[u] = old[u] + v[u];
        }
        __syncthreads();
    }
}

// Tiles of L in shared memory are column-major with leading dimension TL
// (64 rows + room for the 16-byte alignment shift of the first row).
template <typename T>
struct TileLd;
template <>
struct TileLd<float> {
    static constexpr int v = 68;
};
template <>
struct TileLd<double> {
    static constexpr int v = 66;
};

__device__ __forceinline__ void cpa16(void *dst_smem, const void *src, int bytes) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst_smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cpa8(void *dst_smem, const void *src) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst_smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Stage panel rows [row0, row0 + nrows) x columns [col0, col0 + ncols) (at most
// 64 x 64) into dst: element (i, j) lands at dst[j * TL + sh + i], sh = row0 % E
// (E elements per 16 bytes; panel columns start 16-byte aligned). The rows of the
// first 16-byte chunk before row0 belong to the same column and are copied too;
// the last chunk is zero-filled past the range.
template <typename T, int TL>
__device__ __forceinline__ int stage_tile(T *dst, const T *pan, int64_t ld, int row0, int nrows, int col0,
                                          int ncols, int tid, int nth) {
    constexpr int E = 16 / int(sizeof(T));
    const int sh = row0 % E;
    const int start = row0 - sh;
    const int nch = (nrows + sh + E - 1) / E;
    const int tot = ncols * nch;
#pragma unroll 4
    for (int q = tid; q < tot; q += nth) {
        const int j = q / nch, c = q - j * nch;
        const int r = start + c * E;
        const int nv = min(E, row0 + nrows - r);
        cpa16(dst + j * TL + c * E, pan + int64_t(col0 + j) * ld + r, nv * int(sizeof(T)));
    }
    return sh;
}

// shared memory of the diag kernels: acc[kDG][kRB * nrhs] | vec[kRB * nrhs] (double) |
// tile[3][kRB][TL] (ring of two, in-task tile) | dblk[kDG][kRB][kRB + 1] (factor type)
template <typename T>
__host__ __device__ inline size_t diag_smem(int nrhs) {
    return size_t(kDG + 1) * kRB * nrhs * sizeof(double) + size_t(3) * kRB * TileLd<T>::v * sizeof(T) +
           size_t(kDG) * kRB * (kRB + 1) * sizeof(T);
}

// Diagonal block `blk` of the front into dblk (row-major, ld kRB + 1): the stored
// inverse of L(r, r) when the front has one, else the lower triangle of L(r, r).
template <typename T>
__device__ __forceinline__ bool load_diag_block(T *dblk, const T *factor, const T *pan, int64_t inv, int ld, int r0,
                                                int nr, int blk) {
    const int tid = threadIdx.x, nt = blockDim.x;
    if (inv >= 0) {
        const T *src = factor + inv + int64_t(blk) * kRB * kRB;   // column-major 64 x 64
#pragma unroll 8
        for (int q = tid; q < kRB * kRB; q += nt) {
            const int j = q >> 6, i = q & 63;
            dblk[i * (kRB + 1) + j] = src[q];
        }
        return true;
    }
    for (int q = tid; q < nr * nr; q += nt) {
        const int j = q / nr, i = q % nr;
        dblk[i * (kRB + 1) + j] = i >= j ? pan[int64_t(r0 + j) * ld + r0 + i] : T(0);
    }
    return false;
}

// acc -= tile * v (forward: acc(i) -= sum_j L(r0 + i, k0 + j) v(j)); tile (i, j) at [j * TL + i]
template <typename T, int TL>
__device__ __forceinline__ void tile_sub_fwd(double *acc, const T *tl, const double *v, int nrows, int nrhs) {
    const int nq = kRB * nrhs;
    for (int q = threadIdx.x; q < nq; q += blockDim.x) {
        const int i = q & (kRB - 1), r = q >> 6;
        if (i >= nrows) continue;
        const double *vr = v + r * kRB;
        double a0 = 0.0, a1 = 0.0;
#pragma unroll 8
        for (int j = 0; j < kRB; j += 2) {
            a0 += double(tl[j * TL + i]) * vr[j];
            a1 += double(tl[(j + 1) * TL + i]) * vr[j + 1];
        }
        acc[q] -= a0 + a1;
    }
}

// acc -= tile^T * v (backward: acc(j) -= sum_i L(i0 + i, c0 + j) v(i), i < ni); rows in
// skewed order so the lanes of a warp read 32 different rows (distinct banks)
template <typename T, int TL>
__device__ __forceinline__ void tile_sub_bwd(double *acc, const T *tl, const double *v, int ni, int ncols, int nrhs) {
    const int nq = kRB * nrhs;
    for (int q = threadIdx.x; q < nq; q += blockDim.x) {
        const int j = q & (kRB - 1), r = q >> 6;
        if (j >= ncols) continue;
        const double *xr = v + r * kRB;
        double a0 = 0.0, a1 = 0.0;
#pragma unroll 8
        for (int u = 0; u < kRB; u += 2) {
            const int i = (u + j) & (kRB - 1), i1 = (u + 1 + j) & (kRB - 1);
            a0 += (i < ni ? double(tl[j * TL + i]) : 0.0) * xr[i];
            a1 += (i1 < ni ? double(tl[j * TL + i1]) : 0.0) * xr[i1];
        }
        acc[q] -= a0 + a1;
    }
}

// acc := L(b, b)^{-1} acc for one 64-row block, in place (rows >= nr zeroed): through
// the stored inverse, or by substitution on the lower triangle (warp 0). The result
// also goes to X.
template <typename T>
__device__ __forceinline__ void diag_apply_fwd(bool has_inv, const T *dblk, double *acc, int nr, int nrhs, double *X,
                                               int64_t row0, int64_t ldx) {
    const int tid = threadIdx.x, nt = blockDim.x, nq = kRB * nrhs;
    if (has_inv) {
        double out[kMaxSolveRhs * kRB / kDiagThreads];
        int c = 0;
        for (int q = tid; q < nq; q += nt, ++c) {
            const int i = q & (kRB - 1), r = q >> 6;
            double v = 0.0;
            if (i < nr) {
                const T *irow = dblk + i * (kRB + 1);
                const double *ar = acc + r * kRB;
                double a0 = 0.0, a1 = 0.0;
                int j = 0;
                for (; j + 1 <= i; j += 2) {
                    a0 += double(irow[j]) * ar[j];
                    a1 += double(irow[j + 1]) * ar[j + 1];
                }
                if (j == i) a0 += double(irow[j]) * ar[j];
                v = a0 + a1;
            }
            out[c] = v;
        }
        __syncthreads();                                 // every read of acc is done
        c = 0;
        for (int q = tid; q < nq; q += nt, ++c) {
            const int i = q & (kRB - 1), r = q >> 6;
            acc[q] = out[c];
            if (i < nr) X[row0 + i + r * ldx] = out[c];
        }
    } else {
        if (tid < 32) {
            for (int j = 0; j < nr; ++j) {
                const double ljj = double(dblk[j * (kRB + 1) + j]);
                for (int r = tid; r < nrhs; r += 32) acc[r * kRB + j] /= ljj;
                __syncwarp();
                for (int i = j + 1 + tid; i < nr; i += 32) {
                    const double lij = double(dblk[i * (kRB + 1) + j]);
                    for (int r = 0; r < nrhs; ++r) acc[r * kRB + i] -= lij * acc[r * kRB + j];
                }
                __syncwarp();
            }
        }
        __syncthreads();
        for (int q = tid; q < nq; q += nt) {
            const int i = q & (kRB - 1), r = q >> 6;
            if (i < nr) X[row0 + i + r * ldx] = acc[q];
            else acc[q] = 0.0;
        }
    }
}

// acc := L(b, b)^{-T} acc for one 64-column block, in place (stored inverse or
// substitution); also to X.
template <typename T>
__device__ __forceinline__ void diag_apply_bwd(bool has_inv, const T *dblk, double *acc, int nr, int nrhs, double *X,
                                               int64_t row0, int64_t ldx) {
    const int tid = threadIdx.x, nt = blockDim.x, nq = kRB * nrhs;
    if (has_inv) {
        double out[kMaxSolveRhs * kRB / kDiagThreads];
        int c = 0;
        for (int q = tid; q < nq; q += nt, ++c) {
            const int j = q & (kRB - 1), r = q >> 6;
            double v = 0.0;
            if (j < nr) {
                const double *ar = acc + r * kRB;
                double a0 = 0.0, a1 = 0.0;
                int i = j;
                for (; i + 1 < nr; i += 2) {
                    a0 += double(dblk[i * (kRB + 1) + j]) * ar[i];
                    a1 += double(dblk[(i + 1) * (kRB + 1) + j]) * ar[i + 1];
                }
                if (i < nr) a0 += double(dblk[i * (kRB + 1) + j]) * ar[i];
                v = a0 + a1;
            }
            out[c] = v;
        }
        __syncthreads();
        c = 0;
        for (int q = tid; q < nq; q += nt, ++c) {
            const int j = q & (kRB - 1), r = q >> 6;
            acc[q] = out[c];
            if (j < nr) X[row0 + j + r * ldx] = out[c];
        }
    } else {
        if (tid < 32) {
            for (int j = nr - 1; j >= 0; --j) {
                for (int r = tid; r < nrhs; r += 32) acc[r * kRB + j] /= double(dblk[j * (kRB + 1) + j]);
                __syncwarp();
                for (int i = tid; i < j; i += 32) {
                    const double lji = double(dblk[j * (kRB + 1) + i]);
                    for (int r = 0; r < nrhs; ++r) acc[r * kRB + i] -= lji * acc[r * kRB + j];
                }
                __syncwarp();
            }
        }
        __syncthreads();
        for (int q = tid; q < nq; q += nt) {
            const int j = q & (kRB - 1), r = q >> 6;
            if (j < nr) X[row0 + j + r * ldx] = acc[q];
            else acc[q] = 0.0;
        }
    }
}

// Forward diagonal chain. A task is a pair of consecutive 64-row blocks b0, b0 + 1
// of L11 (the last task of a front may hold one); every block has its own flag. The
// task subtracts L11(block b0 + h, block k) y_k for every earlier block k as k's flag
// arrives, finishes block b0 and publishes it before its last tile for block b0 + 1,
// then applies the in-task tile L(b0 + 1, b0) (prefetched into its own buffer) and
// finishes block b0 + 1. Tiles stream through a double-buffered cp.async ring;
// vectors are column-major per RHS: v[r * kRB + i].
template <typename T>
__global__ void __launch_bounds__(kDiagThreads) fwd_diag_kernel(const SolveTask *__restrict__ tasks, int ntasks,
                                                                SnDev sd, const T *__restrict__ factor,
                                                                double *__restrict__ X, int64_t ldx, int nrhs,
                                                                int *__restrict__ flags, int *__restrict__ err) {
    constexpr int TL = TileLd<T>::v;
    extern __shared__ __align__(16) double smem_d[];
    const int nq = kRB * nrhs;
    double *acc = smem_d;                               // [kDG][nq]: accumulators, then y in place
    double *vec = acc + kDG * nq;                       // [nq]: y_k of the block being applied
    T *tiles = reinterpret_cast<T *>(vec + nq);         // [3][kRB * TL]: ring of 2, in-task tile
    T *tin = tiles + 2 * kRB * TL;
    T *dblk = tiles + 3 * kRB * TL;                     // [kDG][kRB * (kRB + 1)]
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int t = blockIdx.x; t < ntasks; t += gridDim.x) {
        const SolveTask tk = tasks[t];
        const int s = tk.sn;
        const int w = sd.w[s], ld = sd.ld[s];
        const int c0 = sd.col0[s];
        const int nbw = (w + kRB - 1) / kRB;
        const int b0 = tk.blk * kDG, nb = min(kDG, nbw - b0);
        const int nr0 = min(kRB, w - b0 * kRB), nr1 = nb == 2 ? min(kRB, w - (b0 + 1) * kRB) : 0;
        const T *pan = factor + sd.pan_off[s];
        const int64_t inv = sd.inv_off[s];
        const int nseq = b0 * nb;                       // tiles (k, h), k < b0 ascending, h < nb
        auto stage = [&](int q, int buf) {
            const int k = q / nb, h = q - k * nb;
            const int r0 = (b0 + h) * kRB;
            stage_tile<T, TL>(tiles + buf * kRB * TL, pan, ld, r0, min(kRB, w - r0), k * kRB, kRB, tid, nt);
        };
        auto publish = [&](int blk) {
            __syncthreads();
            if (tid == 0) {
                __threadfence();
                st_release(flags + tk.flag_base + blk, 1);
            }
        };
        __syncthreads();                                  // previous task done with shared memory
        if (nb == 2) stage_tile<T, TL>(tin, pan, ld, (b0 + 1) * kRB, nr1, b0 * kRB, kRB, tid, nt);
        if (nseq > 0) stage(0, 0);
        cpa_commit();
        bool has_inv[kDG];
#pragma unroll
        for (int h = 0; h < kDG; ++h) {
            has_inv[h] = false;
            if (h < nb)
                has_inv[h] = load_diag_block(dblk + h * kRB * (kRB + 1), factor, pan, inv, ld, (b0 + h) * kRB,
                                             h == 0 ? nr0 : nr1, b0 + h);
        }
        for (int q = tid; q < kDG * nq; q += nt) {
            const int h = q / nq, i = q & (kRB - 1), r = (q - h * nq) >> 6;
            const int row = (b0 + h) * kRB + i;
            acc[q] = (h < nb && row < w) ? X[c0 + row + r * ldx] : 0.0;
        }
        bool done0 = false;
        for (int q = 0; q < nseq; ++q) {
            const int k = q / nb, h = q - k * nb;
            if (q + 1 < nseq) stage(q + 1, (q + 1) & 1);
            cpa_commit();
            if (h == 0) {
                wait_flag(flags + tk.flag_base + k, 1, err);
                for (int e = tid; e < nq; e += nt) {
                    const int j = e & (kRB - 1), r = e >> 6;
                    vec[e] = __ldcg(&X[c0 + k * kRB + j + r * ldx]);
                }
            }
            cpa_wait<1>();
            __syncthreads();
            if (h == 1 && k == b0 - 1) {
                // every dependency of block b0 is in: finish and publish it first
                diag_apply_fwd<T>(has_inv[0], dblk, acc, nr0, nrhs, X, c0 + b0 * kRB, ldx);
                publish(b0);
                done0 = true;
            }
            tile_sub_fwd<T, TL>(acc + h * nq, tiles + (q & 1) * kRB * TL, vec, h == 0 ? nr0 : nr1, nrhs);
            __syncthreads();                              // the ring buffer is refilled two tiles later
        }
        cpa_wait<0>();
        __syncthreads();
        if (!done0) {
            diag_apply_fwd<T>(has_inv[0], dblk, acc, nr0, nrhs, X, c0 + b0 * kRB, ldx);
            publish(b0);
        }
        if (nb == 2) {
            __syncthreads();
            tile_sub_fwd<T, TL>(acc + nq, tin, acc, nr1, nrhs);
            __syncthreads();
            diag_apply_fwd<T>(has_inv[1], dblk + kRB * (kRB + 1), acc + nq, nr1, nrhs, X, c0 + (b0 + 1) * kRB, ldx);
            publish(b0 + 1);
        }
    }
}

// Backward diagonal chain (L11^T x = y), blocks descending. A task (pair b0, b0 + 1)
// subtracts L11(block k, block b0 + h)^T x_k for every later block k as k's flag
// arrives, finishes block b0 + 1 and publishes it before its last tile for block b0,
// then applies the in-task tile L(b0 + 1, b0)^T x_{b0+1} and finishes block b0.
template <typename T>
__global__ void __launch_bounds__(kDiagThreads) bwd_diag_kernel(const SolveTask *__restrict__ tasks, int ntasks,
                                                                SnDev sd, const T *__restrict__ factor,
                                                                double *__restrict__ X, int64_t ldx, int nrhs,
                                                                int *__restrict__ flags, int *__restrict__ err) {
    constexpr int TL = TileLd<T>::v;
    extern __shared__ __align__(16) double smem_d[];
    const int nq = kRB * nrhs;
    double *acc = smem_d;                               // [kDG][nq]: accumulators, then x in place
    double *vec = acc + kDG * nq;                       // [nq]: x_k of the block being applied
    T *tiles = reinterpret_cast<T *>(vec + nq);
    T *tin = tiles + 2 * kRB * TL;
    T *dblk = tiles + 3 * kRB * TL;
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int t = blockIdx.x; t < ntasks; t += gridDim.x) {
        const SolveTask tk = tasks[t];
        const int s = tk.sn;
        const int w = sd.w[s], ld = sd.ld[s];
        const int c0 = sd.col0[s];
        const int nbw = (w + kRB - 1) / kRB;
        const int b0 = tk.blk * kDG, nb = min(kDG, nbw - b0);
        const int nr0 = min(kRB, w - b0 * kRB), nr1 = nb == 2 ? min(kRB, w - (b0 + 1) * kRB) : 0;
        const T *pan = factor + sd.pan_off[s];
        const int64_t inv = sd.inv_off[s];
        const int nlater = nbw - (b0 + nb);
        const int nseq = nlater * nb;                   // tiles (k, h): k descending, h descending
        auto tile_of = [&](int q, int &k, int &h) {
            k = nbw - 1 - q / nb;
            h = nb - 1 - (q - (q / nb) * nb);
        };
        auto stage = [&](int q, int buf) {
            int k, h;
            tile_of(q, k, h);
            const int i0 = k * kRB, cc = (b0 + h) * kRB;
            stage_tile<T, TL>(tiles + buf * kRB * TL, pan, ld, i0, min(kRB, w - i0), cc, min(kRB, w - cc), tid, nt);
        };
        auto publish = [&](int blk) {
            __syncthreads();
            if (tid == 0) {
                __threadfence();
                st_release(flags + tk.flag_base + blk, 2);
            }
        };
        __syncthreads();
        if (nb == 2) stage_tile<T, TL>(tin, pan, ld, (b0 + 1) * kRB, nr1, b0 * kRB, kRB, tid, nt);
        if (nseq > 0) stage(0, 0);
        cpa_commit();
        bool has_inv[kDG];
#pragma unroll
        for (int h = 0; h < kDG; ++h) {
            has_inv[h] = false;
            if (h < nb)
                has_inv[h] = load_diag_block(dblk + h * kRB * (kRB + 1), factor, pan, inv, ld, (b0 + h) * kRB,
                                             h == 0 ? nr0 : nr1, b0 + h);
        }
        for (int q = tid; q < kDG * nq; q += nt) {
            const int h = q / nq, j = q & (kRB - 1), r = (q - h * nq) >> 6;
            const int row = (b0 + h) * kRB + j;
            acc[q] = (h < nb && row < w) ? X[c0 + row + r * ldx] : 0.0;
        }
        bool done1 = false;
        for (int q = 0; q < nseq; ++q) {
            int k, h;
            tile_of(q, k, h);
            if (q + 1 < nseq) stage(q + 1, (q + 1) & 1);
            cpa_commit();
            const int ni = min(kRB, w - k * kRB);
            if (h == nb - 1) {
                wait_flag(flags + tk.flag_base + k, 2, err);
                for (int e = tid; e < nq; e += nt) {
                    const int i = e & (kRB - 1), r = e >> 6;
                    vec[e] = i < ni ? __ldcg(&X[c0 + k * kRB + i + r * ldx]) : 0.0;
                }
            }
            cpa_wait<1>();
            __syncthreads();
            if (nb == 2 && h == 0 && k == b0 + 2) {
                // every dependency of block b0 + 1 is in: finish and publish it first
                diag_apply_bwd<T>(has_inv[1], dblk + kRB * (kRB + 1), acc + nq, nr1, nrhs, X, c0 + (b0 + 1) * kRB,
                                  ldx);
                publish(b0 + 1);
                done1 = true;
            }
            tile_sub_bwd<T, TL>(acc + h * nq, tiles + (q & 1) * kRB * TL, vec, ni, h == 0 ? nr0 : nr1, nrhs);
            __syncthreads();
        }
        cpa_wait<0>();
        __syncthreads();
        if (nb == 2) {
            if (!done1) {
                diag_apply_bwd<T>(has_inv[1], dblk + kRB * (kRB + 1), acc + nq, nr1, nrhs, X, c0 + (b0 + 1) * kRB,
                                  ldx);
                publish(b0 + 1);
            }
            __syncthreads();
            tile_sub_bwd<T, TL>(acc, tin, acc + nq, nr1, kRB, nrhs);
            __syncthreads();
        }
        diag_apply_bwd<T>(has_inv[0], dblk, acc, nr0, nrhs, X, c0 + b0 * kRB, ldx);
        publish(b0);
    }
}

// Structure part, forward: P(task) = L21(rows, cols) y(cols); backward:
// P(task) = L21(rows, cols)^T x(struct rows). Both stream L21 straight from global
// memory with 16-byte loads (panel columns are 16-byte aligned; a task's rows start
// at w rounded down to a multiple of 4), four right-hand sides per pass:
//   forward   task = kStrRows aligned rows x kStrCols columns; warp = 128 of the
//             rows (lane = 4 of them: one FP32 / two FP64 loads per column) over all
//             the task's columns, the vector slice y(cols) in shared memory
//             (broadcast); no sums across warps;
//   backward  task = kStrBCols columns x kStrBRows aligned rows, the x slice in
//             shared memory; warp = 8 columns, lane = 4 rows of every 128: per
//             128-row block the lane's x values go to registers once and serve the
//             warp's 8 columns (8 independent loads in flight); one shuffle
//             reduction per column at the end.
// Rows of a task outside the front's L21 (rows < w, or >= f) are read but never
// used: the forward reduction skips them, the backward x values there are zero
// (the values read there are finite: panel entries, zeroed padding, or the zeroed
// tail of the factor array). With an FP32 factor the products are FP32 (partials
// combined in FP64); an FP64 factor keeps FP64. P slab layout: P[task][r][rows or
// columns].
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
    using type = float4;
};
template <>
struct Vec16<double> {
    using type = double2;
};

template <typename T, int NG>
__global__ void __launch_bounds__(256) str_fwd_kernel(const StrTask *__restrict__ tasks, SnDev sd,
                                                      const T *__restrict__ factor, const double *__restrict__ X,
                                                      int64_t ldx, int nrhs, double *__restrict__ P) {
    using Q = std::conditional_t<sizeof(T) == 4, float, double>;
    using V = typename Vec16<T>::type;
    constexpr int E = 16 / int(sizeof(T));
    constexpr int NVL = 4 / E;                             // loads per lane and column (4 rows)
    __shared__ __align__(16) Q ys[NG][kStrCols];
    const StrTask tk = tasks[blockIdx.x];
    const int s = tk.sn;
    const int w = sd.w[s], f = sd.f[s], ld = sd.ld[s], c0 = sd.col0[s];
    const T *pan = factor + sd.pan_off[s];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int rbase = (w & ~3) + tk.idx * kStrRows + warp * 128;
    const int jb = tk.chunk * kStrCols, nj = min(w - jb, kStrCols);
    int row0[NVL];
    bool vok[NVL];
#pragma unroll
    for (int v = 0; v < NVL; ++v) {
        row0[v] = rbase + v * 32 * E + E * lane;
        vok[v] = row0[v] < f;
    }
    const bool active = rbase < f;
    double *Pt = P + int64_t(blockIdx.x) * kStrRows * nrhs + warp * 128;
    for (int g = 0; g < nrhs; g += NG) {
        const int ng = min(NG, nrhs - g);
        __syncthreads();                                   // the previous pass is done with ys
        for (int q = tid; q < NG * kStrCols; q += 256) {
            const int r = q / kStrCols, j = q - r * kStrCols;
            ys[r][j] = (r < ng && j < nj) ? Q(X[c0 + jb + j + (g + r) * ldx]) : Q(0);
        }
        __syncthreads();
        if (!active) continue;
        Q acc[4][NG];
#pragma unroll
        for (int e = 0; e < 4; ++e)
#pragma unroll
            for (int r = 0; r < NG; ++r) acc[e][r] = Q(0);
        const T *col = pan + int64_t(jb) * ld;
#pragma unroll 8
        for (int j = 0; j < nj; ++j, col += ld) {
            V lv[NVL];
#pragma unroll
            for (int v = 0; v < NVL; ++v) {
                if (vok[v]) lv[v] = *reinterpret_cast<const V *>(col + row0[v]);
                else lv[v] = V{};
            }
            Q yv[NG];
#pragma unroll
            for (int r = 0; r < NG; ++r) yv[r] = ys[r][j];
#pragma unroll
            for (int v = 0; v < NVL; ++v) {
                const T *lp = reinterpret_cast<const T *>(&lv[v]);
#pragma unroll
                for (int e = 0; e < E; ++e)
#pragma unroll
                    for (int r = 0; r < NG; ++r) acc[v * E + e][r] += Q(lp[e]) * yv[r];
            }
        }
#pragma unroll
        for (int v = 0; v < NVL; ++v)
#pragma unroll
            for (int e = 0; e < E; ++e)
#pragma unroll
                for (int r = 0; r < NG; ++r)
                    if (r < ng) Pt[(g + r) * kStrRows + v * 32 * E + E * lane + e] = double(acc[v * E + e][r]);
    }
}

template <typename T, int NG>
__global__ void __launch_bounds__(256) str_bwd_kernel(const StrTask *__restrict__ tasks, SnDev sd,
                                                      const T *__restrict__ factor, const double *__restrict__ X,
                                                      int64_t ldx, int nrhs, double *__restrict__ P) {
    using Q = std::conditional_t<sizeof(T) == 4, float, double>;
    using V = typename Vec16<T>::type;
    constexpr int E = 16 / int(sizeof(T));
    constexpr int NVL = 4 / E;                             // loads per lane, column and 128-row block
    constexpr int BR = str_bwd_rows(sizeof(T) == 8);
    extern __shared__ __align__(16) unsigned char str_raw[];
    Q *xs = reinterpret_cast<Q *>(str_raw);                // [NG][BR]
    const StrTask tk = tasks[blockIdx.x];
    const int s = tk.sn;
    const int w = sd.w[s], f = sd.f[s], ld = sd.ld[s], c0 = sd.col0[s];
    const int vb = sd.vb;
    const T *pan = factor + sd.pan_off[s];
    const int32_t *rows = sd.struct_rows + sd.struct_ptr[s];
    const int rbase = (w & ~3) + tk.chunk * BR;
    const int nrb = min(BR, f - rbase + 127) / 128;        // 128-row blocks reaching row f - 1
    const int j0 = tk.idx * kStrBCols + (threadIdx.x >> 5) * 8;
    const int nj = max(0, min(8, w - j0));
    const int tid = threadIdx.x, lane = tid & 31;
    double *Pt = P + int64_t(blockIdx.x) * kStrBCols * nrhs + (threadIdx.x >> 5) * 8;
    for (int g = 0; g < nrhs; g += NG) {
        const int ng = min(NG, nrhs - g);
        __syncthreads();
        for (int q = tid; q < NG * BR; q += 256) {
            const int r = q / BR, i = q - r * BR;
            const int row = rbase + i, li = row - w;
            Q v = Q(0);
            if (r < ng && row >= w && row < f) v = Q(X[int64_t(rows[li / vb]) * vb + li % vb + (g + r) * ldx]);
            xs[q] = v;
        }
        __syncthreads();
        Q acc[8][NG];
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int r = 0; r < NG; ++r) acc[u][r] = Q(0);
        for (int b = 0; b < nrb; ++b) {
            int row0[NVL];
            bool vok[NVL];
            Q xv[4][NG];
#pragma unroll
            for (int v = 0; v < NVL; ++v) {
                const int i0 = b * 128 + v * 32 * E + E * lane;
                row0[v] = rbase + i0;
                vok[v] = row0[v] < f;
#pragma unroll
                for (int r = 0; r < NG; ++r) {
                    const V xv4 = *reinterpret_cast<const V *>(xs + r * BR + i0);
                    const Q *xp = reinterpret_cast<const Q *>(&xv4);
#pragma unroll
                    for (int e = 0; e < E; ++e) xv[v * E + e][r] = xp[e];
                }
            }
            V lv[8][NVL];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const T *col = pan + int64_t(j0 + min(u, nj - 1)) * ld;
#pragma unroll
                for (int v = 0; v < NVL; ++v) {
                    if (vok[v] && u < nj) lv[u][v] = *reinterpret_cast<const V *>(col + row0[v]);
                    else lv[u][v] = V{};
                }
            }
#pragma unroll
            for (int u = 0; u < 8; ++u)
#pragma unroll
                for (int v = 0; v < NVL; ++v) {
                    const T *lp = reinterpret_cast<const T *>(&lv[u][v]);
#pragma unroll
                    for (int e = 0; e < E; ++e)
#pragma unroll
                        for (int r = 0; r < NG; ++r) acc[u][r] += Q(lp[e]) * xv[v * E + e][r];
                }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int r = 0; r < NG; ++r) {
                Q sum = acc[u][r];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
                if (lane == 0 && r < ng && u < nj) Pt[(g + r) * kStrBCols + u] = double(sum);
            }
    }
}

// Subtract the chunk partials of one forward row slab (from u_s) or backward column
// slab (from x), in chunk order.
template <bool FWD>
__global__ void __launch_bounds__(256) str_reduce_kernel(const StrReduce *__restrict__ red, SnDev sd,
                                                         double *__restrict__ X, int64_t ldx, int nrhs,
                                                         double *__restrict__ sol, const double *__restrict__ P) {
    const StrReduce rd = red[blockIdx.x];
    const int s = rd.sn;
    const int w = sd.w[s], d = sd.d[s];
    constexpr int NS = FWD ? kStrRows : kStrBCols;
    const int64_t stride = int64_t(NS) * nrhs;
    for (int q = threadIdx.x; q < NS * nrhs; q += blockDim.x) {
        const int a = q % NS, r = q / NS;
        double acc = 0.0;
        for (int c = 0; c < rd.nchunks; ++c) acc += P[int64_t(rd.first + c) * stride + r * NS + a];
        if (FWD) {
            const int drow = (w & ~3) + rd.idx * kStrRows + a - w;
            if (drow >= 0 && drow < d) sol[sd.sol_off[s] * nrhs + drow + int64_t(r) * d] -= acc;
        } else {
            const int col = rd.idx * kStrBCols + a;
            if (col < w) X[sd.col0[s] + col + r * ldx] -= acc;
        }
    }
}

int sm_count() { return device_sm_count(); }

template <typename K>
int coop_grid(K kernel, size_t smem, int ntasks) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kDiagThreads, smem);
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
cudaError_t launch_diag(bool forward, const SolveTask *tasks, int ntasks, SnDev sd, const T *factor, double *X,
                        int64_t ldx, int nrhs, int *flags, int *err, cudaStream_t st) {
    if (ntasks <= 0) return cudaSuccess;
    void *kern = forward ? (void *)fwd_diag_kernel<T> : (void *)bwd_diag_kernel<T>;
    const size_t smem = diag_smem<T>(nrhs);
    // one-time per kernel and device: shared-memory opt-in and co-resident grid per RHS count
    static PerDeviceOnce once;
    once([] {
        cudaFuncSetAttribute(fwd_diag_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(diag_smem<T>(kMaxSolveRhs)));
        cudaFuncSetAttribute(bwd_diag_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             int(diag_smem<T>(kMaxSolveRhs)));
    });
    static int grid_cache[kMaxDevices][2][kMaxSolveRhs + 1] = {};
    const int dev = current_device();
    int gtmp = 0;
    int &gmax = (dev >= 0 && dev < kMaxDevices) ? grid_cache[dev][forward ? 0 : 1][nrhs] : gtmp;
    if (!gmax) gmax = forward ? coop_grid(fwd_diag_kernel<T>, smem, 1 << 30) : coop_grid(bwd_diag_kernel<T>, smem, 1 << 30);
    const int grid = std::min(gmax, ntasks);
    void *args[] = {(void *)&tasks, (void *)&ntasks, (void *)&sd, (void *)&factor, (void *)&X, (void *)&ldx,
                    (void *)&nrhs, (void *)&flags, (void *)&err};
    ++g_kernel_launches;
    return cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kDiagThreads), args, smem, st);
}

template <typename T, int NG>
void launch_str_ng(bool forward, const StrTask *tasks, int ntasks, const StrReduce *red, int nred, SnDev sd,
                   const T *factor, double *X, int64_t ldx, int nrhs, double *sol, double *P, cudaStream_t st) {
    using Q = std::conditional_t<sizeof(T) == 4, float, double>;
    const size_t smem = size_t(NG) * str_bwd_rows(sizeof(T) == 8) * sizeof(Q);
    static PerDeviceOnce once;
    once([smem] { cudaFuncSetAttribute(str_bwd_kernel<T, NG>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)); });
    if (forward) {
        str_fwd_kernel<T, NG><<<ntasks, 256, 0, st>>>(tasks, sd, factor, X, ldx, nrhs, P);
        str_reduce_kernel<true><<<nred, 256, 0, st>>>(red, sd, X, ldx, nrhs, sol, P);
    } else {
        str_bwd_kernel<T, NG><<<ntasks, 256, smem, st>>>(tasks, sd, factor, X, ldx, nrhs, P);
        str_reduce_kernel<false><<<nred, 256, 0, st>>>(red, sd, X, ldx, nrhs, sol, P);
    }
}

// Right-hand sides per sweep over L21: 4, or 8 for an FP32 factor with more than
// four (each sweep streams the task's L21 once; FP64 keeps 4 for its registers).
template <typename T>
void launch_str(bool forward, const StrTask *tasks, int ntasks, const StrReduce *red, int nred, SnDev sd,
                const T *factor, double *X, int64_t ldx, int nrhs, double *sol, double *P, cudaStream_t st) {
    if (ntasks <= 0) return;
    g_kernel_launches += 2;
    if constexpr (sizeof(T) == 4) {
        if (nrhs > 4) {
            launch_str_ng<T, 8>(forward, tasks, ntasks, red, nred, sd, factor, X, ldx, nrhs, sol, P, st);
            return;
        }
    }
    launch_str_ng<T, 4>(forward, tasks, ntasks, red, nred, sd, factor, X, ldx, nrhs, sol, P, st);
}

#define MFS_TRI_INSTANTIATE(T)                                                                                    \
    template cudaError_t launch_diag<T>(bool, const SolveTask *, int, SnDev, const T *, double *, int64_t, int,   \
                                        int *, int *, cudaStream_t);                                              \
    template void launch_str<T>(bool, const StrTask *, int, const StrReduce *, int, SnDev, const T *, double *,   \
                                int64_t, int, double *, double *, cudaStream_t);
MFS_TRI_INSTANTIATE(double)
MFS_TRI_INSTANTIATE(float)

int solve_rows_per_task() { return kRB; }
int diag_blocks_per_task() { return kDG; }

}  // namespace mfs
