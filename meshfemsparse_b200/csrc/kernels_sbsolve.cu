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
// forward substitution.
//
// A solve task is one 64-row part h of superblock K of one front, run by one CTA;
// the (up to) four parts of a superblock run side by side:
//   forward   a_h = b_h - sum_{J < K} L(rows h, superblock J) y_J (J ascending, as
//             J's count reaches its part count), a_h to a scratch vector, count;
//             once every part of K has counted, y_h = inv(L_KK)(rows h, :) a_K, count;
//   backward  a_h = y_h - sum_{J > K} L(superblock J, columns h)^T x_J (J
//             descending), then x_h = inv(L_KK)(:, columns h)^T a_K the same way.
// A superblock thus costs two hops between CTAs and two 64 x 256 products on the
// chain, and what a task reads after its last dependency arrives (64 x 256 of L
// and at most 64 x 256 of the inverse) is already on chip: L and the inverse
// stream through shared memory in 32 KB chunks (64 rows x 128 FP32 / 64 FP64
// columns forward, 128 / 64 rows x 64 columns backward), one 2D TMA box per chunk
// issued by one thread through per-front / per-inverse tensor maps, completing on
// the ring slot's mbarrier, up to six chunks in flight. A box reaching past the
// front's L11 or past the inverse reads zeros there.
//
// Launches are cooperative (all CTAs co-resident); every CTA walks its tasks in
// ascending order and a task waits only on lower-numbered tasks and on the other
// parts of its own superblock (adjacent task numbers, so on other CTAs), hence
// the lowest unfinished task can always proceed. Counts are zeroed before each
// solve: forward targets are the superblock's part count, backward ones twice
// that. Waits are bounded in time: on expiry the kernel records an error and
// stops waiting; the host reports MFS_TIMEOUT. Sums run in a fixed order, so
// results are run-to-run identical. With an FP32 factor (the preconditioner of
// FP64 refinement) the products with off-diagonal superblocks are FP32
// (accumulated per thread over the task, combined in FP64) and the inverse of the
// diagonal superblock is applied in FP64; an FP64 factor keeps FP64 throughout.
#include "device.h"

#include <algorithm>
#include <type_traits>

namespace mfs {

namespace {

constexpr int SB = kSuperBlock;
constexpr int kSbThreads = 256;
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
// Product type of the off-diagonal chunk sums: FP32 for an FP32 factor, FP64 otherwise.
template <typename T>
using PT = std::conditional_t<sizeof(T) == 4, float, double>;

// Chunks of 32 KB: forward 64 rows x FC columns (column-major, ld 64), backward
// FC rows x 64 columns (column-major, ld FC).
template <typename T>
struct SpChunk {
    static constexpr int FC = 32768 / (64 * int(sizeof(T)));   // 128 (FP32), 64 (FP64)
    static constexpr int ELEMS = 64 * FC;
    static constexpr int BYTES = ELEMS * int(sizeof(T));
};
// Shared memory: ring [NST][32 KB] | vec [NR][SB] doubles | vp [NR][SB] products' type
// | red [4][NR][64] doubles | own [NR][64] doubles.
template <typename T, int NST, int NR>
struct SpLayout {
    static constexpr size_t vec_off = size_t(NST) * SpChunk<T>::BYTES;
    static constexpr size_t vp_off = vec_off + size_t(NR) * SB * sizeof(double);
    static constexpr size_t red_off = vp_off + size_t(NR) * SB * sizeof(PT<T>);
    static constexpr size_t own_off = red_off + size_t(4) * NR * 64 * sizeof(double);
    static constexpr size_t bytes = own_off + size_t(NR) * 64 * sizeof(double);
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
// 2D tiled TMA load of one box of the tensor map at `map` (device memory written
// before the launch), box origin (x = row, y = column), completing on `bar`.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const char *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
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

// Thread 0 waits until the count at p reaches target (bounded), then the block proceeds.
__device__ __forceinline__ void wait_count(const int *p, int target, int *err) {
    if (threadIdx.x == 0) {
        if (ld_acquire(p) < target) {
            const unsigned long long t0 = gtimer();
            while (ld_acquire(p) < target) {
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
// After a __syncthreads that follows this block's writes: publish them and count.
__device__ __forceinline__ void count_up(int *p) {
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(p, 1);
    }
}

// Forward task (s, K, h = tk.pad): rows R0 = K SB + 64 h, nrh of them. Chunks: for
// J < K, L(rows R0.., columns J SB + c FC ..) (c < SB / FC), then the inverse's
// rows 64 h.. of columns [c FC, c FC + FC) up to column 64 h + 63 (the rest of
// the row is zero). Thread (i = tid % 64, part = tid / 64) sums columns
// [part FC / 4, (part + 1) FC / 4) of every chunk for row i.
template <typename T, int NST, int NR>
__global__ void __launch_bounds__(kSbThreads, 1) sp_fwd_kernel(const SbTask *__restrict__ tasks, int ntasks,
                                                               SnDev sd, const T *__restrict__ factor,
                                                               const char *__restrict__ maps, double *__restrict__ X, int64_t ldx, int nrhs,
                                                               double *__restrict__ scratch, int *__restrict__ flags,
                                                               int *__restrict__ err) {
    using Lay = SpLayout<T, NST, NR>;
    using P = PT<T>;
    constexpr int FC = SpChunk<T>::FC, CE = SpChunk<T>::ELEMS;
    constexpr int per = SB / FC;                         // chunks per earlier superblock
    constexpr int QC = FC / 4;
    extern __shared__ __align__(128) unsigned char sp_dyn[];
    __shared__ __align__(8) uint64_t bars[NST];
    // TMA destinations: 128-byte aligned (the launch adds 128 bytes for this)
    unsigned char *sp_raw = sp_dyn + ((128u - (smem_u32(sp_dyn) & 127u)) & 127u);
    T *ring = reinterpret_cast<T *>(sp_raw);
    double *vec = reinterpret_cast<double *>(sp_raw + Lay::vec_off);
    P *vp = reinterpret_cast<P *>(sp_raw + Lay::vp_off);
    double *red = reinterpret_cast<double *>(sp_raw + Lay::red_off);
    double *own = reinterpret_cast<double *>(sp_raw + Lay::own_off);
    const int tid = threadIdx.x, i = tid & 63, part = tid >> 6;
    if (tid == 0) {
        for (int b = 0; b < NST; ++b) mbar_init(smem_u32(&bars[b]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    long long gq = 0;                                    // chunks this CTA has consumed (ring phase)
    for (int t = blockIdx.x; t < ntasks; t += gridDim.x) {
        const SbTask tk = tasks[t];
        const int s = tk.sn, K = tk.K, h = tk.pad;
        const int w = sd.w[s], c0 = sd.col0[s];
        const int nrK = sb_rows(w, K), nrpK = sb_pad(nrK), nhK = nrpK / 64;
        const int R0 = K * SB + h * 64, nrh = min(64, w - R0);
        const int icols = (h + 1) * 64;                  // nonzero columns of the inverse's rows
        const int ndep = K * per;
        const int nq = ndep + (icols + FC - 1) / FC;
        int *ycnt = flags + tk.flag0;                    // [2 J]: parts of J done, [2 J + 1]: a_J parts
        auto stage = [&](int q) {
            const int slot = int((gq + q) % NST);
            T *dst = ring + slot * CE;
            const uint32_t bar = smem_u32(&bars[slot]);
            mbar_expect_tx(bar, SpChunk<T>::BYTES);
            if (q < ndep) {
                const int J = q / per, c = q - J * per;
                tma_load_2d(smem_u32(dst), maps + size_t(tk.pmap) * kTensorMapBytes, R0, J * SB + c * FC, bar);
            } else {
                const int c = q - ndep;
                tma_load_2d(smem_u32(dst), maps + size_t(tk.imap) * kTensorMapBytes, h * 64, c * FC, bar);
            }
        };
        __syncthreads();                                 // the previous task is done with shared memory
        if (tid == 0)
            for (int q = 0; q < NST - 1 && q < nq; ++q) stage(q);
        if (tid < 64)
            for (int r = 0; r < NR; ++r) own[r * 64 + i] = (r < nrhs && i < nrh) ? X[c0 + R0 + i + r * ldx] : 0.0;
        P pacc[NR];
        double dacc[NR];
#pragma unroll
        for (int r = 0; r < NR; ++r) {
            pacc[r] = P(0);
            dacc[r] = 0.0;
        }
        auto chunk = [&](int q) -> const T * {
            const int slot = int((gq + q) % NST);
            mbar_wait_all(smem_u32(&bars[slot]), uint32_t(((gq + q) / NST) & 1), err);
            __syncthreads();                             // (also: vectors are complete)
            return ring + slot * CE;
        };
        for (int q = 0; q < ndep; ++q) {
            if (tid == 0 && q + NST - 1 < nq) stage(q + NST - 1);
            const int J = q / per, c = q - J * per;
            if (c == 0) {
                // y_J: wait for its parts, then load it (written by other CTAs: through L2)
                wait_count(ycnt + 2 * J, SB / 64, err);
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    const double v = r < nrhs ? __ldcg(&X[c0 + J * SB + tid + r * ldx]) : 0.0;
                    vec[r * SB + tid] = v;
                    vp[r * SB + tid] = P(v);
                }
            }
            const T *a = chunk(q) + part * QC * 64 + i;
            const P *v = vp + c * FC + part * QC;
#pragma unroll 8
            for (int j = 0; j < QC; ++j) {
                const P l = P(a[j * 64]);
#pragma unroll
                for (int r = 0; r < NR; ++r) pacc[r] += l * v[r * SB + j];
            }
            __syncthreads();                             // the ring slot is refilled NST - 1 chunks later
        }
        // every dependency is in: a_h = own - sums, to the scratch vector; count, wait
        // for the other parts of K, load a_K
#pragma unroll
        for (int r = 0; r < NR; ++r) red[(part * NR + r) * 64 + i] = double(pacc[r]);
        __syncthreads();
        if (tid < 64)
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const int e = r * 64 + i;
                const double a = own[e] - (((red[e] + red[NR * 64 + e]) + red[2 * NR * 64 + e]) + red[3 * NR * 64 + e]);
                if (r < nrhs && i < nrh) scratch[c0 + R0 + i + r * ldx] = a;
            }
        __syncthreads();
        count_up(ycnt + 2 * K + 1);
        wait_count(ycnt + 2 * K + 1, nhK, err);
#pragma unroll
        for (int r = 0; r < NR; ++r)
            vec[r * SB + tid] = (r < nrhs && tid < nrK) ? __ldcg(&scratch[c0 + K * SB + tid + r * ldx]) : 0.0;
        for (int q = ndep; q < nq; ++q) {
            if (tid == 0 && q + NST - 1 < nq) stage(q + NST - 1);
            const int c = q - ndep;
            const int j0 = part * QC, j1 = min(QC, min(FC, icols - c * FC) - j0);
            const T *a = chunk(q) + j0 * 64 + i;
            const double *v = vec + c * FC + j0;
            for (int j = 0; j < j1; ++j) {
                const double l = double(a[j * 64]);
#pragma unroll
                for (int r = 0; r < NR; ++r) dacc[r] += l * v[r * SB + j];
            }
            __syncthreads();
        }
        gq += nq;
#pragma unroll
        for (int r = 0; r < NR; ++r) red[(part * NR + r) * 64 + i] = dacc[r];
        __syncthreads();
        if (tid < 64)
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const int e = r * 64 + i;
                const double y = ((red[e] + red[NR * 64 + e]) + red[2 * NR * 64 + e]) + red[3 * NR * 64 + e];
                if (r < nrhs && i < nrh) X[c0 + R0 + i + r * ldx] = y;
            }
        __syncthreads();
        count_up(ycnt + 2 * K);
    }
    ring_drain<NST>(bars, gq, err);
}

// Backward task (s, K, h = tk.pad): columns C0 = K SB + 64 h, nch of them. Chunks:
// for J = nsb - 1 down to K + 1, L(rows J SB + c FC .., columns C0..) (the last
// superblock's rows rounded up to 64), then the inverse's columns 64 h.. from row
// 64 h + c FC on. Warp wp sums columns 8 wp .. 8 wp + 7 of every chunk, its lanes
// over the chunk's rows.
template <typename T, int NST, int NR>
__global__ void __launch_bounds__(kSbThreads, 1) sp_bwd_kernel(const SbTask *__restrict__ tasks, int ntasks,
                                                               SnDev sd, const T *__restrict__ factor,
                                                               const char *__restrict__ maps, double *__restrict__ X, int64_t ldx, int nrhs,
                                                               double *__restrict__ scratch, int *__restrict__ flags,
                                                               int *__restrict__ err) {
    using Lay = SpLayout<T, NST, NR>;
    using P = PT<T>;
    constexpr int FC = SpChunk<T>::FC, CE = SpChunk<T>::ELEMS;
    constexpr int per = SB / FC;                         // chunks per full later superblock
    constexpr int RL = FC / 32;                          // chunk rows per lane
    extern __shared__ __align__(128) unsigned char sp_dyn[];
    __shared__ __align__(8) uint64_t bars[NST];
    // TMA destinations: 128-byte aligned (the launch adds 128 bytes for this)
    unsigned char *sp_raw = sp_dyn + ((128u - (smem_u32(sp_dyn) & 127u)) & 127u);
    T *ring = reinterpret_cast<T *>(sp_raw);
    double *vec = reinterpret_cast<double *>(sp_raw + Lay::vec_off);
    P *vp = reinterpret_cast<P *>(sp_raw + Lay::vp_off);
    double *own = reinterpret_cast<double *>(sp_raw + Lay::own_off);
    const int tid = threadIdx.x, lane = tid & 31, wp = tid >> 5;
    if (tid == 0) {
        for (int b = 0; b < NST; ++b) mbar_init(smem_u32(&bars[b]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    long long gq = 0;
    for (int t = blockIdx.x; t < ntasks; t += gridDim.x) {
        const SbTask tk = tasks[t];
        const int s = tk.sn, K = tk.K, h = tk.pad;
        const int w = sd.w[s], c0 = sd.col0[s];
        const int nsb = (w + SB - 1) / SB;
        const int nrK = sb_rows(w, K), nrpK = sb_pad(nrK), nhK = nrpK / 64;
        const int C0 = K * SB + h * 64, nch = min(64, w - C0);
        const int nrl = sb_rows(w, nsb - 1), nql = (sb_pad(nrl) + FC - 1) / FC;   // last superblock
        const int ndep = K < nsb - 1 ? nql + (nsb - 2 - K) * per : 0;
        const int irows = nrpK - h * 64;                 // the inverse's rows from 64 h
        const int nq = ndep + (irows + FC - 1) / FC;
        int *ycnt = flags + tk.flag0;
        // dependency chunk q: superblock J, chunk c
        auto dep = [&](int q, int &J, int &c) {
            if (q < nql) {
                J = nsb - 1;
                c = q;
            } else {
                const int m = q - nql;
                J = nsb - 2 - m / per;
                c = m % per;
            }
        };
        auto stage = [&](int q) {
            const int slot = int((gq + q) % NST);
            T *dst = ring + slot * CE;
            const uint32_t bar = smem_u32(&bars[slot]);
            mbar_expect_tx(bar, SpChunk<T>::BYTES);
            if (q < ndep) {
                int J, c;
                dep(q, J, c);
                tma_load_2d(smem_u32(dst), maps + size_t(tk.pmap + 1) * kTensorMapBytes, J * SB + c * FC, C0, bar);
            } else {
                const int c = q - ndep;
                tma_load_2d(smem_u32(dst), maps + size_t(tk.imap + 1) * kTensorMapBytes, h * 64 + c * FC, h * 64,
                            bar);
            }
        };
        __syncthreads();
        if (tid == 0)
            for (int q = 0; q < NST - 1 && q < nq; ++q) stage(q);
        if (tid < 64)
            for (int r = 0; r < NR; ++r)
                own[r * 64 + tid] = (r < nrhs && tid < nch) ? X[c0 + C0 + tid + r * ldx] : 0.0;
        auto chunk = [&](int q) -> const T * {
            const int slot = int((gq + q) % NST);
            mbar_wait_all(smem_u32(&bars[slot]), uint32_t(((gq + q) / NST) & 1), err);
            __syncthreads();
            return ring + slot * CE;
        };
        {
            P pacc[8][NR];
#pragma unroll
            for (int u = 0; u < 8; ++u)
#pragma unroll
                for (int r = 0; r < NR; ++r) pacc[u][r] = P(0);
            for (int q = 0; q < ndep; ++q) {
                if (tid == 0 && q + NST - 1 < nq) stage(q + NST - 1);
                int J, c;
                dep(q, J, c);
                const int nrJ = sb_rows(w, J);
                if (c == 0) {
                    wait_count(ycnt + 2 * J, 2 * (sb_pad(nrJ) / 64), err);
#pragma unroll
                    for (int r = 0; r < NR; ++r) {
                        const double v = (r < nrhs && tid < nrJ) ? __ldcg(&X[c0 + J * SB + tid + r * ldx]) : 0.0;
                        vec[r * SB + tid] = v;
                        vp[r * SB + tid] = P(v);
                    }
                }
                const T *tl = chunk(q);
                // rows of the chunk at or past the superblock's end are masked out
                const int nv = nrJ - c * FC;
                const P *v = vp + c * FC;
#pragma unroll
                for (int k = 0; k < RL; ++k) {
                    const int row = lane + 32 * k;
                    const bool ok = row < nv;
                    P x[NR];
#pragma unroll
                    for (int r = 0; r < NR; ++r) x[r] = ok ? v[r * SB + row] : P(0);
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const P l = ok ? P(tl[(wp * 8 + u) * FC + row]) : P(0);
#pragma unroll
                        for (int r = 0; r < NR; ++r) pacc[u][r] += l * x[r];
                    }
                }
                __syncthreads();
            }
            __syncthreads();                             // own is complete
#pragma unroll
            for (int u = 0; u < 8; ++u)
#pragma unroll
                for (int r = 0; r < NR; ++r) {
                    P g = pacc[u][r];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) g += __shfl_down_sync(0xffffffffu, g, o);
                    if (lane == 0) own[r * 64 + wp * 8 + u] -= double(g);
                }
        }
        __syncthreads();
        if (tid < 64)
#pragma unroll
            for (int r = 0; r < NR; ++r)
                if (r < nrhs && tid < nch) scratch[c0 + C0 + tid + r * ldx] = own[r * 64 + tid];
        __syncthreads();
        count_up(ycnt + 2 * K + 1);
        wait_count(ycnt + 2 * K + 1, 2 * nhK, err);
#pragma unroll
        for (int r = 0; r < NR; ++r)
            vec[r * SB + tid] = (r < nrhs && tid < nrK) ? __ldcg(&scratch[c0 + K * SB + tid + r * ldx]) : 0.0;
        double dacc[8][NR];
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int r = 0; r < NR; ++r) dacc[u][r] = 0.0;
        for (int q = ndep; q < nq; ++q) {
            if (tid == 0 && q + NST - 1 < nq) stage(q + NST - 1);
            const int c = q - ndep;
            const T *tl = chunk(q);
            const int nv = min(FC, irows - c * FC);
            const double *v = vec + h * 64 + c * FC;
#pragma unroll
            for (int k = 0; k < RL; ++k) {
                const int row = lane + 32 * k;
                if (row < nv) {
                    double x[NR];
#pragma unroll
                    for (int r = 0; r < NR; ++r) x[r] = v[r * SB + row];
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const double l = double(tl[(wp * 8 + u) * FC + row]);
#pragma unroll
                        for (int r = 0; r < NR; ++r) dacc[u][r] += l * x[r];
                    }
                }
            }
            __syncthreads();
        }
        gq += nq;
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                double g = dacc[u][r];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) g += __shfl_down_sync(0xffffffffu, g, o);
                const int col = wp * 8 + u;
                if (lane == 0 && r < nrhs && col < nch) X[c0 + C0 + col + r * ldx] = g;
            }
        __syncthreads();
        count_up(ycnt + 2 * K);
    }
    ring_drain<NST>(bars, gq, err);
}

// inv(L_KK) of superblock K of front s (nr rows), nrp x nrp column-major at
// factor + tk.inv, one CTA per 64-column block b of it (blockIdx.y):
//   X_bb = D_b, X_ab = -D_a sum_{c=b}^{a-1} L_ac X_cb for a > b, X_ab = 0 for a < b,
// with D_a = inv(L_aa) the 64 x 64 diagonal inverses: the panel kernel's stored
// ones when the front has them, else by column-wise substitution on L_aa (one
// thread per column). The column's blocks X_cb stay in shared memory; each L_ac
// and D_a is staged there before its 64 x 64 x 64 product (thread = row i, 16
// columns: the X / T operands are broadcast within a warp).
template <typename T>
__global__ void __launch_bounds__(256) sb_inverse_kernel(const SbTask *__restrict__ tasks, SnDev sd, T *factor) {
    constexpr int LD = 65;
    constexpr int TB = 64 * LD;                           // one staged 64 x 64 block
    extern __shared__ __align__(16) double inv_smem[];
    T *Xc = reinterpret_cast<T *>(inv_smem);              // [4][TB]: X_cb, c = b .. nbk - 1
    T *Ls = Xc + 4 * TB;                                  // L_ac, then T = sum L_ac X_cb
    T *Ds = Ls + TB;                                      // D_a
    const SbTask tk = tasks[blockIdx.x];
    const int s = tk.sn, K = tk.K, b = blockIdx.y;
    const int w = sd.w[s], ld = sd.ld[s];
    const T *pan = factor + sd.pan_off[s];
    T *out = factor + tk.inv;
    const int nr = sb_rows(w, K), nrp = sb_pad(nr), nbk = nrp / 64;
    if (b >= nbk) return;
    const int r0 = K * SB;
    const int tid = threadIdx.x, i = tid & 63, jg = tid >> 6;
    const int64_t dinv = sd.inv_off[s];
    auto Lv = [&](int gi, int gj) -> T {                   // superblock-local L(gi, gj), 0 outside
        return (gi < nr && gj < nr) ? pan[int64_t(r0 + gj) * ld + r0 + gi] : T(0);
    };
    // D_a into dst (ld LD): stored inverse, or substitution on L_aa (staged in scratch)
    auto load_diag = [&](int a, T *dst, T *scratch) {
        if (dinv >= 0) {
            const T *src = factor + dinv + int64_t(K * (SB / 64) + a) * 4096;
            for (int q = tid; q < 4096; q += blockDim.x) {
                const int jj = q >> 6, ii = q & 63;
                dst[jj * LD + ii] = (a * 64 + ii < nr && a * 64 + jj < nr) ? src[q] : T(0);
            }
            __syncthreads();
            return;
        }
        for (int q = tid; q < 4096; q += blockDim.x) {
            const int jj = q >> 6, ii = q & 63;
            scratch[jj * LD + ii] = Lv(a * 64 + ii, a * 64 + jj);
        }
        __syncthreads();
        if (tid < 64) {
            const int j = tid, nb = min(64, nr - a * 64);
            for (int k = 0; k < 64; ++k) {
                T v = T(0);
                if (k >= j && k < nb && j < nb) {
                    v = k == j ? T(1) : T(0);
                    for (int m = j; m < k; ++m) v -= scratch[m * LD + k] * dst[j * LD + m];
                    v /= scratch[k * LD + k];
                }
                dst[j * LD + k] = v;
            }
        }
        __syncthreads();
    };
    // the strict upper blocks of this column are zero
    for (int q = tid; q < b * 64 * 64; q += blockDim.x) {
        const int jj = q / (b * 64), ii = q - jj * (b * 64);
        out[int64_t(b * 64 + jj) * nrp + ii] = T(0);
    }
    // X_bb = D_b
    T *Xb = Xc;
    load_diag(b, Xb, Ls);
    for (int q = tid; q < 4096; q += blockDim.x) {
        const int jj = q >> 6, ii = q & 63;
        out[int64_t(b * 64 + jj) * nrp + b * 64 + ii] = Xb[jj * LD + ii];
    }
    for (int a = b + 1; a < nbk; ++a) {
        T acc[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) acc[u] = T(0);
        for (int c = b; c < a; ++c) {
            __syncthreads();                               // Ls is free
            for (int q = tid; q < 4096; q += blockDim.x) {
                const int m = q >> 6, ii = q & 63;
                Ls[m * LD + ii] = Lv(a * 64 + ii, c * 64 + m);
            }
            __syncthreads();
            const T *X = Xc + (c - b) * TB + (jg * 16) * LD;
#pragma unroll 4
            for (int m = 0; m < 64; ++m) {
                const T l = Ls[m * LD + i];
#pragma unroll
                for (int u = 0; u < 16; ++u) acc[u] += l * X[u * LD + m];
            }
        }
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 16; ++u) Ls[(jg * 16 + u) * LD + i] = acc[u];   // T(i, j)
        load_diag(a, Ds, Xc + (a - b) * TB);               // (synchronizes; X_ab's slot is free)
#pragma unroll
        for (int u = 0; u < 16; ++u) acc[u] = T(0);
        const T *Tt = Ls + (jg * 16) * LD;
#pragma unroll 4
        for (int m = 0; m < 64; ++m) {
            const T dv = Ds[m * LD + i];
#pragma unroll
            for (int u = 0; u < 16; ++u) acc[u] -= dv * Tt[u * LD + m];
        }
        T *Xa = Xc + (a - b) * TB;
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            Xa[(jg * 16 + u) * LD + i] = acc[u];
            out[int64_t(b * 64 + jg * 16 + u) * nrp + a * 64 + i] = acc[u];
        }
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
cudaError_t launch_sp_impl(bool forward, const SbTask *tasks, int ntasks, SnDev sd, const T *factor, const char *maps,
                           double *X, int64_t ldx, int nrhs, double *scratch, int *flags, int *err, cudaStream_t st) {
    using L = SpLayout<T, NST, NR>;
    constexpr size_t smem = L::bytes + 128;
    static_assert(smem + 256 <= size_t(kMaxSmemOptin), "superblock solve shared memory");
    void *kern = forward ? (void *)sp_fwd_kernel<T, NST, NR> : (void *)sp_bwd_kernel<T, NST, NR>;
    static PerDeviceOnce once;
    once([] {
        cudaFuncSetAttribute(sp_fwd_kernel<T, NST, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
        cudaFuncSetAttribute(sp_bwd_kernel<T, NST, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    });
    const int grid = forward ? coop_grid(sp_fwd_kernel<T, NST, NR>, smem, ntasks)
                             : coop_grid(sp_bwd_kernel<T, NST, NR>, smem, ntasks);
    void *args[] = {(void *)&tasks, (void *)&ntasks, (void *)&sd,      (void *)&factor, (void *)&maps, (void *)&X,
                    (void *)&ldx,   (void *)&nrhs,   (void *)&scratch, (void *)&flags,  (void *)&err};
    ++g_kernel_launches;
    return cudaLaunchCooperativeKernel(kern, dim3(grid), dim3(kSbThreads), args, smem, st);
}

}  // namespace

template <typename T>
cudaError_t launch_sb_solve(bool forward, const SbTask *tasks, int ntasks, SnDev sd, const T *factor,
                            const void *maps, double *X, int64_t ldx, int nrhs, double *scratch, int *flags, int *err,
                            cudaStream_t st) {
    const char *mp = static_cast<const char *>(maps);
    if (ntasks <= 0) return cudaSuccess;
    if (nrhs > kSbMaxRhs) return cudaErrorInvalidValue;
    // ring depth: the deepest that fits beside the vectors of nrhs right-hand sides
    constexpr int D4 = sizeof(T) == 4 ? 6 : 5, D8 = sizeof(T) == 4 ? 5 : 4;
    if (nrhs <= 4)
        return launch_sp_impl<T, D4, 4>(forward, tasks, ntasks, sd, factor, mp, X, ldx, nrhs, scratch, flags, err, st);
    return launch_sp_impl<T, D8, kSbMaxRhs>(forward, tasks, ntasks, sd, factor, mp, X, ldx, nrhs, scratch, flags, err,
                                            st);
}

template <typename T>
void launch_sb_inverse(const SbTask *tasks, int ntasks, SnDev sd, T *factor, cudaStream_t st) {
    if (ntasks <= 0) return;
    const size_t smem = size_t(6) * 64 * 65 * sizeof(T);
    static PerDeviceOnce once;
    once([smem] { cudaFuncSetAttribute(sb_inverse_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)); });
    ++g_kernel_launches;
    sb_inverse_kernel<T><<<dim3(ntasks, SB / 64), 256, smem, st>>>(tasks, sd, factor);
}

template cudaError_t launch_sb_solve<float>(bool, const SbTask *, int, SnDev, const float *, const void *, double *,
                                            int64_t, int, double *, int *, int *, cudaStream_t);
template cudaError_t launch_sb_solve<double>(bool, const SbTask *, int, SnDev, const double *, const void *, double *,
                                             int64_t, int, double *, int *, int *, cudaStream_t);
template void launch_sb_inverse<float>(const SbTask *, int, SnDev, float *, cudaStream_t);
template void launch_sb_inverse<double>(const SbTask *, int, SnDev, double *, cudaStream_t);

}  // namespace mfs
