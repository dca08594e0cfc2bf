// Diagonal-block solves of the level-scheduled triangular solves (K6) through
// explicit inverses of 256-row superblocks of L11.
//
// Reference: SparseLDL::Solve (forward L y = b, backward L^T x = y; called at
// Solvers/CatamariFactorizer.cc:54,70) and its per-supernode kernels
// (trs_kernels::SolveLowerTri, tests/test_catamari_solve_kernels.cc). The
// dependency chain of a front's L11 solve is what bounds the solve: a block of y
// cannot start before every earlier block is known. Here the chain runs over
// superblocks of SB = 256 rows: after the numeric factorization,
// sb_inverse_kernel writes inv(L_KK) of every superblock K of every front above
// the solve cut (dense, column-major, nrp x nrp with nrp = 64 * ceil(rows / 64),
// zeros above the diagonal), built from the 64 x 64 diagonal inverses by block
// forward substitution. A solve task is one superblock of one front, run by one
// CTA:
//   forward   acc = b_K - sum_{J < K} L_KJ y_J   (waiting on superblock J's flag),
//             y_K = inv(L_KK) acc, publish (one thread per row);
//   backward  acc = y_K - sum_{J > K} L_JK^T x_J (J descending),
//             x_K = inv(L_KK)^T acc, publish (one warp per column, shuffle sums).
// L and the inverse stream through shared memory in 32 KB chunks of whole columns
// (256 rows x 32 FP32 / 16 FP64 columns; the inverse's rows above a chunk's first
// column are zero and skipped): one thread issues a bulk copy per column, the
// chunk completes on its ring slot's mbarrier, and up to six chunks are in flight,
// so the chunks of the next dependency are already on chip when its flag comes.
// Bulk copies of a superblock's rows are rounded up to 64 rows; the extra rows lie
// inside the factor array (the next rows or column of the panel, or the inverses
// stored after the panels) and are never used.
// The chain thus takes one flag hop, one superblock-wide product and one
// inverse product per 256 rows. Launches are cooperative (all CTAs co-resident);
// every CTA walks its tasks in ascending order and a task waits only on
// lower-numbered tasks of its front, so the lowest unfinished task can always
// proceed. Waits are bounded in time: on expiry the kernel records an error and
// stops waiting; the host reports MFS_TIMEOUT. Sums run in a fixed order, so
// results are run-to-run identical. With an FP32 factor (the preconditioner of
// FP64 refinement) the products with off-diagonal superblocks are FP32 (chunk
// results accumulated in FP64) and the inverse of the diagonal superblock is
// applied in FP64; an FP64 factor keeps FP64 throughout.
#include "device.h"

#include <algorithm>
#include <type_traits>

namespace mfs {

namespace {

constexpr int SB = kSuperBlock;
constexpr int kSbThreads = 256;
constexpr int kRG = 8;                                    // right-hand sides per register group
constexpr unsigned long long kWaitNs = 2000000000ull;    // 2 s per wait at most
static_assert(SB == kSbThreads, "one thread per superblock row");

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
__device__ __forceinline__ void cpa16(void *dst_smem, const void *src, int bytes) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst_smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cpa_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cpa_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Stage `ncols` columns of a column-major source (leading dimension lds), rows
// [row0, row0 + ncopy) of each (ncopy a multiple of 16 bytes), into dst with
// element (i, j) at dst[j * ldd + i]; rows at or past row0 + nvalid are zero-filled.
template <typename T>
__device__ __forceinline__ void stage_cols(T *dst, int ldd, const T *src, int64_t lds, int row0, int nvalid,
                                           int ncopy, int ncols) {
    constexpr int E = 16 / int(sizeof(T));
    const int nch = ncopy / E;
    const int tot = nch * ncols;
    for (int q = threadIdx.x; q < tot; q += blockDim.x) {
        const int j = q / nch, c = q - j * nch;
        const int i = c * E;
        const int nv = max(0, min(E, nvalid - i));
        const T *s = src + int64_t(j) * lds + row0 + i;
        cpa16(dst + j * ldd + i, nv ? s : src, nv * int(sizeof(T)));
    }
}

// Product type of the off-diagonal chunk sums: FP32 for an FP32 factor, FP64 otherwise.
template <typename T>
using PT = std::conditional_t<sizeof(T) == 4, float, double>;

// Chunks of 32 KB: CW whole columns (SB rows) of L or of the inverse, column-major in
// shared memory with leading dimension SB, streamed through an NST-deep ring of bulk
// copies (one per column) that complete on the slot's mbarrier.
template <typename T>
struct SbChunk {
    static constexpr int CW = 32768 / (SB * int(sizeof(T)));   // 32 columns (FP32), 16 (FP64)
    static constexpr int BYTES = CW * SB * int(sizeof(T));
};
template <typename T, int NST>
struct SbLayout {
    // doubles: acc[nrhs][SB] | out[nrhs][SB] | vec[nrhs][SB]; PT copy of vec [nrhs][SB]; ring
    static __host__ __device__ constexpr size_t ring_off(int nrhs) {
        return (size_t(3) * nrhs * SB * sizeof(double) + size_t(nrhs) * SB * sizeof(PT<T>) + 127) & ~size_t(127);
    }
    static __host__ __device__ constexpr size_t bytes(int nrhs) {
        return ring_off(nrhs) + size_t(NST) * SbChunk<T>::BYTES;
    }
};

// Rows of superblock K of a front with w columns, and its 64-rounded extent.
__device__ __forceinline__ int sb_rows(int w, int K) { return min(SB, w - K * SB); }
__device__ __forceinline__ int sb_pad(int nr) { return (nr + 63) & ~63; }

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Every thread waits for the chunk's copies (bounded; on expiry the error is
// recorded and the chunk's contents are not trusted).
__device__ __forceinline__ void mbar_wait_all(uint32_t bar, uint32_t parity, int *err) {
    if (mbar_try(bar, parity)) return;
    const unsigned long long t0 = gtimer();
    for (int it = 1;; ++it) {
        if (mbar_try(bar, parity)) return;
        if ((it & 63) == 0) {
            if (*(volatile int *)err) return;
            if (gtimer() - t0 > kWaitNs) {
                atomicExch(err, 1);
                return;
            }
        }
    }
}
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
// One thread: ncols columns of a column-major source (leading dimension lds), rows
// [row0, row0 + nrows) of each (16-byte aligned, a multiple of 16 bytes), to
// dst + j * SB elements, completing on `bar`.
template <typename T>
__device__ __forceinline__ void stage_bulk(T *dst, const T *src, int64_t lds, int row0, int nrows, int ncols,
                                           uint32_t bar) {
    const uint32_t bytes = uint32_t(nrows) * sizeof(T);
    mbar_expect_tx(bar, bytes * uint32_t(ncols));
    const uint32_t d0 = smem_u32(dst);
    for (int j = 0; j < ncols; ++j)
        bulk_copy(d0 + uint32_t(j) * SB * sizeof(T), src + int64_t(j) * lds + row0, bytes, bar);
}

// After an error (a wait that gave up), the copies a CTA issued may still be in
// flight: thread 0 waits, again bounded, for the last use of every ring slot, so
// no copy lands in shared memory after the CTA has exited.
template <int NST>
__device__ __forceinline__ void ring_drain(uint64_t *bars, long long issued, const int *err) {
    if (threadIdx.x != 0 || !*(volatile const int *)err) return;
    for (int b = 0; b < NST; ++b) {
        if (issued <= b) continue;
        const long long last = b + ((issued - 1 - b) / NST) * NST;
        const uint32_t bar = smem_u32(&bars[b]), par = uint32_t((last / NST) & 1);
        const unsigned long long t0 = gtimer();
        while (!mbar_try(bar, par) && gtimer() - t0 < kWaitNs) {
        }
    }
}

// Row mode (forward): this thread's row (chunk row trow), dst[r * SB] -/+=
// sum_j tl[j * SB + trow] v[r * SB + j], j < ncol, for the NR right-hand sides.
template <typename Q, int NR, typename T>
__device__ __forceinline__ void row_chunk(const T *tl, int trow, const Q *v, int ncol, int nrhs, double *dst,
                                          bool sub) {
    Q p[NR];
#pragma unroll
    for (int u = 0; u < NR; ++u) p[u] = Q(0);
#pragma unroll 8
    for (int j = 0; j < ncol; ++j) {
        const Q a = Q(tl[j * SB + trow]);
#pragma unroll
        for (int u = 0; u < NR; ++u) p[u] += a * v[u * SB + j];
    }
#pragma unroll
    for (int u = 0; u < NR; ++u)
        if (u < nrhs) {
            if (sub) dst[u * SB] -= double(p[u]);
            else dst[u * SB] += double(p[u]);
        }
}
// Column mode (backward): one warp per column j of the chunk (columns warp, warp + 8,
// ...): s_r = sum_{i < nrow} tl[j * SB + i] v[r * SB + i] over the lanes, reduced by
// shuffles; lane 0 applies dst[r * SB + j] -= s_r (mode 0) or = s_r (mode 1).
template <typename Q, int NR, typename T>
__device__ __forceinline__ void col_chunk(const T *tl, const Q *v, int nrow, int ncol, int nrhs, double *dst,
                                          int mode) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int j = warp; j < ncol; j += nw) {
        const T *col = tl + j * SB;
        Q p[NR];
#pragma unroll
        for (int u = 0; u < NR; ++u) p[u] = Q(0);
        for (int i = lane; i < nrow; i += 32) {
            const Q a = Q(col[i]);
#pragma unroll
            for (int u = 0; u < NR; ++u) p[u] += a * v[u * SB + i];
        }
#pragma unroll
        for (int u = 0; u < NR; ++u) {
            Q g = p[u];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) g += __shfl_down_sync(0xffffffffu, g, o);
            if (lane == 0 && u < nrhs) {
                if (mode == 0) dst[u * SB + j] -= double(g);
                else dst[u * SB + j] = double(g);
            }
        }
    }
}

// Vectors hold NR right-hand sides (columns >= nrhs are zero), so the products above
// run without predicates.
template <typename T, int NST, int NR>
__global__ void __launch_bounds__(kSbThreads, 1) sb_fwd_kernel(const SbTask *__restrict__ tasks, int ntasks,
                                                               SnDev sd, const T *__restrict__ factor,
                                                               double *__restrict__ X, int64_t ldx, int nrhs,
                                                               int *__restrict__ flags, int *__restrict__ err) {
    using L = SbLayout<T, NST>;
    using P = PT<T>;
    constexpr int CW = SbChunk<T>::CW;
    constexpr int BUF = CW * SB;
    constexpr int per = SB / CW;                         // chunks per earlier superblock
    extern __shared__ __align__(128) double sb_smem[];
    __shared__ __align__(8) uint64_t bars[NST];
    double *acc = sb_smem;
    double *out = acc + NR * SB;
    double *vec = out + NR * SB;
    P *vp = reinterpret_cast<P *>(vec + NR * SB);
    T *ring = reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(sb_smem) + L::ring_off(NR));
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int b = 0; b < NST; ++b) mbar_init(smem_u32(&bars[b]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    long long gq = 0;                                    // chunks this CTA has consumed (ring phase)
    for (int t = blockIdx.x; t < ntasks; t += gridDim.x) {
        const SbTask tk = tasks[t];
        const int s = tk.sn, K = tk.K;
        const int w = sd.w[s], ld = sd.ld[s], c0 = sd.col0[s];
        const T *pan = factor + sd.pan_off[s];
        const T *inv = factor + tk.inv;
        const int nr = sb_rows(w, K), nrp = sb_pad(nr);
        const int r0 = K * SB;
        const int ninv = (nrp + CW - 1) / CW;            // column chunks of the inverse
        const int nq = K * per + ninv;
        // chunk q: L(rows of K, CW columns of superblock J = q / per), or the inverse's
        // columns [c CW, c CW + CW) with their rows from c CW on (the rest is zero)
        auto stage = [&](int q) {
            const int slot = int((gq + q) % NST);
            T *dst = ring + slot * BUF;
            const uint32_t bar = smem_u32(&bars[slot]);
            if (q < K * per) {
                const int J = q / per, c = q - J * per;
                stage_bulk<T>(dst, pan + int64_t(J * SB + c * CW) * ld, ld, r0, nrp, CW, bar);
            } else {
                const int c = q - K * per;
                stage_bulk<T>(dst, inv + int64_t(c * CW) * nrp, nrp, c * CW, nrp - c * CW, min(CW, nrp - c * CW),
                              bar);
            }
        };
        __syncthreads();                                 // the previous task is done with shared memory
        if (tid == 0)
            for (int q = 0; q < NST - 1 && q < nq; ++q) stage(q);
        for (int r = 0; r < NR; ++r) {
            acc[r * SB + tid] = (r < nrhs && tid < nr) ? X[c0 + r0 + tid + r * ldx] : 0.0;
            out[r * SB + tid] = 0.0;
        }
        for (int q = 0; q < nq; ++q) {
            if (tid == 0 && q + NST - 1 < nq) stage(q + NST - 1);
            const bool lpart = q < K * per;
            const int J = lpart ? q / per : K, c = lpart ? q - J * per : q - K * per;
            if (lpart && c == 0) {
                // y_J: wait for its superblock, then load it (written by another CTA: through L2)
                wait_flag(flags + tk.flag0 + J, 1, err);
                for (int r = 0; r < NR; ++r) {
                    const double v = r < nrhs ? __ldcg(&X[c0 + J * SB + tid + r * ldx]) : 0.0;
                    vec[r * SB + tid] = v;
                    vp[r * SB + tid] = P(v);
                }
            }
            const int slot = int((gq + q) % NST);
            mbar_wait_all(smem_u32(&bars[slot]), uint32_t(((gq + q) / NST) & 1), err);
            __syncthreads();                             // (also: vectors and acc are complete)
            const T *tl = ring + slot * BUF;
            if (lpart) {
                // off-diagonal superblock: products of the factor's precision
                if (tid < nr) row_chunk<P, NR>(tl, tid, vp + c * CW, CW, nrhs, acc + tid, true);
            } else if (tid < nr && tid >= c * CW) {
                // inverse of the diagonal superblock (rows from c CW): FP64 products
                row_chunk<double, NR>(tl, tid - c * CW, acc + c * CW, min(CW, nrp - c * CW), nrhs, out + tid,
                                      false);
            }
            __syncthreads();                             // the ring slot is refilled NST - 1 chunks later
        }
        gq += nq;
        if (tid < nr)
            for (int r = 0; r < nrhs; ++r) X[c0 + r0 + tid + r * ldx] = out[r * SB + tid];
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            st_release(flags + tk.flag0 + K, 1);
        }
    }
    ring_drain<NST>(bars, gq, err);
}

template <typename T, int NST, int NR>
__global__ void __launch_bounds__(kSbThreads, 1) sb_bwd_kernel(const SbTask *__restrict__ tasks, int ntasks,
                                                               SnDev sd, const T *__restrict__ factor,
                                                               double *__restrict__ X, int64_t ldx, int nrhs,
                                                               int *__restrict__ flags, int *__restrict__ err) {
    using L = SbLayout<T, NST>;
    using P = PT<T>;
    constexpr int CW = SbChunk<T>::CW;
    constexpr int BUF = CW * SB;
    constexpr int per = SB / CW;                         // column chunks per later superblock
    extern __shared__ __align__(128) double sb_smem[];
    __shared__ __align__(8) uint64_t bars[NST];
    double *acc = sb_smem;
    double *out = acc + NR * SB;
    double *vec = out + NR * SB;
    P *vp = reinterpret_cast<P *>(vec + NR * SB);
    T *ring = reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(sb_smem) + L::ring_off(NR));
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int b = 0; b < NST; ++b) mbar_init(smem_u32(&bars[b]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    long long gq = 0;
    for (int t = blockIdx.x; t < ntasks; t += gridDim.x) {
        const SbTask tk = tasks[t];
        const int s = tk.sn, K = tk.K;
        const int w = sd.w[s], ld = sd.ld[s], c0 = sd.col0[s];
        const T *pan = factor + sd.pan_off[s];
        const T *inv = factor + tk.inv;
        const int nr = sb_rows(w, K), nrp = sb_pad(nr);
        const int r0 = K * SB;
        const int nsb = (w + SB - 1) / SB;
        // chunk q: for J = nsb - 1 down to K + 1, L(rows of J, columns [r0 + c CW, + CW)
        // of K) (K is not the last superblock then, so its SB columns are whole); then
        // the inverse's columns [c CW, + CW) with their rows from c CW on
        const int nql = (nsb - 1 - K) * per;
        const int ninv = (nrp + CW - 1) / CW;
        const int nq = nql + ninv;
        auto jinfo = [&](int q, int &J, int &c) {
            const int m = q / per;
            J = nsb - 1 - m;
            c = q - m * per;
        };
        auto stage = [&](int q) {
            const int slot = int((gq + q) % NST);
            T *dst = ring + slot * BUF;
            const uint32_t bar = smem_u32(&bars[slot]);
            if (q < nql) {
                int J, c;
                jinfo(q, J, c);
                stage_bulk<T>(dst, pan + int64_t(r0 + c * CW) * ld, ld, J * SB, sb_pad(sb_rows(w, J)), CW, bar);
            } else {
                const int c = q - nql;
                stage_bulk<T>(dst, inv + int64_t(c * CW) * nrp, nrp, c * CW, nrp - c * CW, min(CW, nrp - c * CW),
                              bar);
            }
        };
        __syncthreads();
        if (tid == 0)
            for (int q = 0; q < NST - 1 && q < nq; ++q) stage(q);
        for (int r = 0; r < NR; ++r) {
            acc[r * SB + tid] = (r < nrhs && tid < nr) ? X[c0 + r0 + tid + r * ldx] : 0.0;
            out[r * SB + tid] = 0.0;
        }
        for (int q = 0; q < nq; ++q) {
            if (tid == 0 && q + NST - 1 < nq) stage(q + NST - 1);
            const bool lpart = q < nql;
            int J = K, c = q - nql;
            if (lpart) jinfo(q, J, c);
            const int nrJ = lpart ? sb_rows(w, J) : 0;
            if (lpart && c == 0) {
                wait_flag(flags + tk.flag0 + J, 2, err);
                for (int r = 0; r < NR; ++r) {
                    const double v = (r < nrhs && tid < nrJ) ? __ldcg(&X[c0 + J * SB + tid + r * ldx]) : 0.0;
                    vec[r * SB + tid] = v;
                    vp[r * SB + tid] = P(v);
                }
            }
            const int slot = int((gq + q) % NST);
            mbar_wait_all(smem_u32(&bars[slot]), uint32_t(((gq + q) / NST) & 1), err);
            __syncthreads();                             // (also: vectors and acc are complete)
            const T *tl = ring + slot * BUF;
            if (lpart) {
                // acc(columns of the chunk) -= L(J rows, chunk columns)^T x_J
                col_chunk<P, NR>(tl, vp, nrJ, CW, nrhs, acc + c * CW, 0);
            } else {
                // x(chunk columns) = inv(L_KK)(rows from c CW, chunk columns)^T acc: FP64 products
                col_chunk<double, NR>(tl, acc + c * CW, nrp - c * CW, min(CW, nrp - c * CW), nrhs, out + c * CW, 1);
            }
            __syncthreads();
        }
        gq += nq;
        if (tid < nr)
            for (int r = 0; r < nrhs; ++r) X[c0 + r0 + tid + r * ldx] = out[r * SB + tid];
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            st_release(flags + tk.flag0 + K, 2);
        }
    }
    ring_drain<NST>(bars, gq, err);
}

// inv(L_KK) of superblock K of front s (nr rows), nrp x nrp column-major at
// factor + tk.inv. The 64 x 64 diagonal inverses D_b come from the panel kernel's
// stored inverses when the front has them, else by column-wise substitution on
// L_bb (one thread per column); then X_ab = -D_a sum_{c=b}^{a-1} L_ac X_cb.
template <typename T>
__global__ void __launch_bounds__(256) sb_inverse_kernel(const SbTask *__restrict__ tasks, SnDev sd, T *factor) {
    constexpr int LD = 65;
    constexpr int DPAR = sizeof(T) == 4 ? 4 : 2;          // diagonal blocks inverted at once
    extern __shared__ __align__(16) double inv_smem[];
    T *Ls = reinterpret_cast<T *>(inv_smem);              // [DPAR][64 * LD] diagonal blocks of L
    T *Xs = Ls + DPAR * 64 * LD;                          // [DPAR][64 * LD] their inverses / a product tile
    const SbTask tk = tasks[blockIdx.x];
    const int s = tk.sn, K = tk.K;
    const int w = sd.w[s], ld = sd.ld[s];
    const T *pan = factor + sd.pan_off[s];
    T *out = factor + tk.inv;
    const int nr = sb_rows(w, K), nrp = sb_pad(nr), nbk = nrp / 64;
    const int r0 = K * SB;
    const int tid = threadIdx.x;
    const int64_t dinv = sd.inv_off[s];
    auto Lv = [&](int i, int j) -> T {                     // superblock-local L(i, j), 0 outside
        return (i < nr && j < nr) ? pan[int64_t(r0 + j) * ld + r0 + i] : T(0);
    };
    // zero the strict upper block triangle of the output
    for (int q = tid; q < nrp * nrp; q += blockDim.x) {
        const int j = q / nrp, i = q - j * nrp;
        if ((i >> 6) < (j >> 6)) out[q] = T(0);
    }
    // 1. diagonal inverses
    for (int b0 = 0; b0 < nbk; b0 += DPAR) {
        const int g = tid >> 6, j = tid & 63, b = b0 + g;
        if (dinv >= 0) {
            for (int q = tid; q < min(DPAR, nbk - b0) * 4096; q += blockDim.x) {
                const int bb = b0 + (q >> 12), e = q & 4095, jj = e >> 6, ii = e & 63;
                const T v = factor[dinv + int64_t(K * (SB / 64) + bb) * 4096 + e];
                out[int64_t(bb * 64 + jj) * nrp + bb * 64 + ii] = (bb * 64 + ii < nr && bb * 64 + jj < nr) ? v : T(0);
            }
            continue;
        }
        __syncthreads();
        if (g < DPAR && b < nbk)
            for (int q = j; q < 64 * 64; q += 64) {
                const int jj = q >> 6, ii = q & 63;
                Ls[g * 64 * LD + jj * LD + ii] = Lv(b * 64 + ii, b * 64 + jj);
            }
        __syncthreads();
        if (g < DPAR && b < nbk) {
            const T *Lb = Ls + g * 64 * LD;
            T *Xb = Xs + g * 64 * LD;
            const int nb = min(64, nr - b * 64);
            for (int k = 0; k < 64; ++k) {
                T v = T(0);
                if (k >= j && k < nb && j < nb) {
                    v = k == j ? T(1) : T(0);
                    for (int m = j; m < k; ++m) v -= Lb[m * LD + k] * Xb[j * LD + m];
                    v /= Lb[k * LD + k];
                }
                Xb[j * LD + k] = v;
            }
            for (int k = 0; k < 64; ++k) out[int64_t(b * 64 + j) * nrp + b * 64 + k] = Xb[j * LD + k];
        }
    }
    __syncthreads();
    // 2. off-diagonal blocks, column block by column block
    T *Ts = Xs;                                           // 64 x 64 product tile (ld LD)
    const int i = tid & 63, jg = tid >> 6;                // row, 16-column group
    for (int b = 0; b + 1 < nbk; ++b)
        for (int a = b + 1; a < nbk; ++a) {
            T acc[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) acc[u] = T(0);
            for (int c = b; c < a; ++c)
                for (int m = 0; m < 64; ++m) {
                    const T l = Lv(a * 64 + i, c * 64 + m);
#pragma unroll
                    for (int u = 0; u < 16; ++u)
                        acc[u] += l * __ldcg(&out[int64_t(b * 64 + jg * 16 + u) * nrp + c * 64 + m]);
                }
            __syncthreads();
#pragma unroll
            for (int u = 0; u < 16; ++u) Ts[(jg * 16 + u) * LD + i] = acc[u];
            __syncthreads();
#pragma unroll
            for (int u = 0; u < 16; ++u) acc[u] = T(0);
            for (int m = 0; m < 64; ++m) {
                const T dv = __ldcg(&out[int64_t(a * 64 + m) * nrp + a * 64 + i]);
#pragma unroll
                for (int u = 0; u < 16; ++u) acc[u] -= dv * Ts[(jg * 16 + u) * LD + m];
            }
#pragma unroll
            for (int u = 0; u < 16; ++u) out[int64_t(b * 64 + jg * 16 + u) * nrp + a * 64 + i] = acc[u];
            __syncthreads();
        }
}

template <typename K>
int coop_grid(K kernel, size_t smem, int ntasks) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kSbThreads, smem);
    const int g = std::max(1, per_sm) * device_sm_count();
    return std::min(g, std::max(1, ntasks));
}

// NR: the right-hand sides the vectors hold (nrhs <= NR)
template <typename T, int NST, int NR>
cudaError_t launch_sb_impl(bool forward, const SbTask *tasks, int ntasks, SnDev sd, const T *factor, double *X,
                           int64_t ldx, int nrhs, int *flags, int *err, cudaStream_t st) {
    using L = SbLayout<T, NST>;
    static_assert(L::bytes(NR) + 64 <= size_t(kMaxSmemOptin), "superblock solve shared memory");
    void *kern = forward ? (void *)sb_fwd_kernel<T, NST, NR> : (void *)sb_bwd_kernel<T, NST, NR>;
    const size_t smem = L::bytes(NR);
    static PerDeviceOnce once;
    once([] {
        cudaFuncSetAttribute(sb_fwd_kernel<T, NST, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(L::bytes(NR)));
        cudaFuncSetAttribute(sb_bwd_kernel<T, NST, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(L::bytes(NR)));
    });
    const int grid = forward ? coop_grid(sb_fwd_kernel<T, NST, NR>, smem, ntasks)
                             : coop_grid(sb_bwd_kernel<T, NST, NR>, smem, ntasks);
    void *args[] = {(void *)&tasks, (void *)&ntasks, (void *)&sd, (void *)&factor, (void *)&X, (void *)&ldx,
                    (void *)&nrhs, (void *)&flags, (void *)&err};
    ++g_kernel_launches;
    return cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kSbThreads), args, smem, st);
}

}  // namespace

template <typename T>
cudaError_t launch_sb_solve(bool forward, const SbTask *tasks, int ntasks, SnDev sd, const T *factor, double *X,
                            int64_t ldx, int nrhs, int *flags, int *err, cudaStream_t st) {
    if (ntasks <= 0) return cudaSuccess;
    if (nrhs > kMaxSolveRhs) return cudaErrorInvalidValue;
    // ring depth: the deepest that fits beside the vectors of nrhs right-hand sides
    if (nrhs <= 4) return launch_sb_impl<T, 6, 4>(forward, tasks, ntasks, sd, factor, X, ldx, nrhs, flags, err, st);
    if (nrhs <= 8) return launch_sb_impl<T, 4, 8>(forward, tasks, ntasks, sd, factor, X, ldx, nrhs, flags, err, st);
    return launch_sb_impl<T, 2, kMaxSolveRhs>(forward, tasks, ntasks, sd, factor, X, ldx, nrhs, flags, err, st);
}

template <typename T>
void launch_sb_inverse(const SbTask *tasks, int ntasks, SnDev sd, T *factor, cudaStream_t st) {
    if (ntasks <= 0) return;
    constexpr int DPAR = sizeof(T) == 4 ? 4 : 2;
    const size_t smem = size_t(2) * DPAR * 64 * 65 * sizeof(T);
    static PerDeviceOnce once;
    once([smem] { cudaFuncSetAttribute(sb_inverse_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)); });
    ++g_kernel_launches;
    sb_inverse_kernel<T><<<ntasks, 256, smem, st>>>(tasks, sd, factor);
}

template cudaError_t launch_sb_solve<float>(bool, const SbTask *, int, SnDev, const float *, double *, int64_t, int,
                                            int *, int *, cudaStream_t);
template cudaError_t launch_sb_solve<double>(bool, const SbTask *, int, SnDev, const double *, double *, int64_t,
                                             int, int *, int *, cudaStream_t);
template void launch_sb_inverse<float>(const SbTask *, int, SnDev, float *, cudaStream_t);
template void launch_sb_inverse<double>(const SbTask *, int, SnDev, double *, cudaStream_t);

}  // namespace mfs
