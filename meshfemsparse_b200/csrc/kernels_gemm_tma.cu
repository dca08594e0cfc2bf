// Schur-update GEMM on the 5th-generation tensor cores with TMA-fed operands.
//
//     C(i,j) -= scale * sum_k A(i,k) B(j,k)      (trailing updates and SYRK, mode 0)
//
// Operands are FP32 read as TF32 (kind::tf32) or FP16 (kind::f16, the scaled
// half-precision copy of the factor's panels); C and the accumulation are FP32.
// Same task lists and 128 x 256 task tiles as the cp.async kernel
// (kernels_gemm_tc.cu): one CTA per task tile, 320 threads, two CTAs per SM for
// FP32 and FP16 operands (see Occupancy).
//   warp 0     lane 0 issues the TMA loads of a STAGES-deep ring: per k-block one
//              box of 128 bytes x TBK k rows per 128-byte group of M (N) rows;
//              A and B are 2D tensor maps (rows x k columns, column-major) built
//              on the host, one per factor panel (or per task for the test hook);
//              rows or columns outside a map arrive as zeros.
//   warp 1     allocates 256 TMEM columns (the 128 x 256 FP32 accumulator, or with
//              split FP16 operands two 128 x 128 ones: a 256-column task tile then
//              runs as two CTAs of 128 columns); lane 0 issues tcgen05.mma (M = 128,
//              N = 256 or 128) from shared-memory descriptors and frees ring slots
//              with tcgen05.commit.
//   warps 2-9  epilogue: TMEM -> registers -> C in 16-column chunks (two warps per
//              32-lane quarter of TMEM, one per column half).
// Shared-memory operand layout: MN-major, 128-byte swizzle; FP32 with 32-byte
// atoms (a 512-byte atom holds 4 k rows of 32 elements, the 32-byte chunk index
// XOR-ed with the k row), FP16 with 16-byte atoms (1024-byte atoms of 8 k rows of
// 64 elements, the 16-byte chunk index XOR-ed with the k row); the TMA boxes are
// written in exactly that form by the tensor maps' swizzle modes. Groups of 128
// bytes of M are 128 * TBK bytes apart (descriptor LBO), atoms along k follow
// each other (SBO), and the MMA for k slice g starts 128 * MMA_K * g bytes into
// the group.
//
// Pipeline: full[s] (producer arrive + TMA transaction bytes), empty[s]
// (tcgen05.commit), done (tcgen05.commit after the last MMA). Every wait is
// bounded in time; on expiry the kernel records an error in *err, stops issuing,
// lets the copies and MMAs it issued retire, frees TMEM and returns; the host
// reports MFS_TIMEOUT.
#include "device.h"

#include <cuda.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <mutex>
#include <type_traits>

namespace mfs {

namespace {

constexpr int TBM = 128, TBN = 256;
constexpr int kEpiWarps = 8;
constexpr int kThreads = (2 + kEpiWarps) * 32;
constexpr unsigned long long kWaitNs = 1000000000ull;   // 1 s per wait at most
constexpr int kGroupM = 8;

template <typename E>
struct OpTraits;
template <>
struct OpTraits<float> {
    static constexpr int ATOM = 32;          // elements per 128-byte row of a box
    static constexpr int TBK = 32;           // k rows per stage
    static constexpr int MMA_K = 8;
    static constexpr uint32_t SBO = 512;     // 4 k rows per swizzle atom
    static constexpr uint32_t LAYOUT = 1;    // 128-byte swizzle, 32-byte atoms
    static constexpr uint32_t IDESC_AB = (2u << 7) | (2u << 10);   // TF32 A and B
};
template <>
struct OpTraits<__half> {
    static constexpr int ATOM = 64;
    static constexpr int TBK = 64;
    static constexpr int MMA_K = 16;
    static constexpr uint32_t SBO = 1024;    // 8 k rows per swizzle atom
    static constexpr uint32_t LAYOUT = 2;    // 128-byte swizzle
    static constexpr uint32_t IDESC_AB = 0u; // F16 A and B
};

// Split FP16 operands (hi + 2^-11 lo, each FP16): same atoms as __half, 32 k rows
// per stage so that the four boxes of a stage (A hi / lo, B hi / lo) fit a 4-deep ring.
struct HalfSplit {};
template <>
struct OpTraits<HalfSplit> {
    static constexpr int ATOM = 64;
    static constexpr int TBK = 32;
    static constexpr int MMA_K = 16;
    static constexpr uint32_t SBO = 1024;
    static constexpr uint32_t LAYOUT = 2;
    static constexpr uint32_t IDESC_AB = 0u;
};

// TN: the columns one CTA computes (256, or 128 when a 256-column task tile is split
// between two CTAs)
template <typename E, int TN>
struct StageShape {
    static constexpr int BOX = 128 * OpTraits<E>::TBK;          // bytes of one box (one 128-byte group)
    static constexpr int A = (TBM / OpTraits<E>::ATOM) * BOX;   // 16 KB
    static constexpr int B = (TN / OpTraits<E>::ATOM) * BOX;    // 32 KB for TN = 256
    static constexpr bool SPLIT = std::is_same<E, HalfSplit>::value;
    // ring slot: A hi, B hi (, A lo, B lo)
    static constexpr int BYTES = SPLIT ? 2 * (A + B) : A + B;
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
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
// Bounded wait for the phase with the given parity; false on timeout or when
// another CTA has already reported one.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int *err) {
    if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (int it = 1;; ++it) {
        if (mbar_try(bar, parity)) return true;
        if ((it & 31) == 0) {
            if (*(volatile int *)err) return false;
            if (global_ns() - t0 > kWaitNs) {
                atomicExch(err, 1);
                return false;
            }
        }
    }
}
// Bounded wait that ignores the error flag (lets issued copies / MMAs retire).
__device__ __forceinline__ void mbar_drain(uint32_t bar, uint32_t parity) {
    const unsigned long long t0 = global_ns();
    while (!mbar_try(bar, parity))
        if (global_ns() - t0 > kWaitNs) return;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int x, int y, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void tmap_acquire(const CUtensorMap *map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(map))
                 : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo, uint32_t layout) {
    return uint64_t((addr >> 4) & 0x3FFF) | (uint64_t((lbo >> 4) & 0x3FFF) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFF) << 32) | (uint64_t(1) << 46) | (uint64_t(layout) << 61);
}
// Instruction descriptor: FP32 accumulate, A and B MN-major, M = 128.
template <typename E>
__device__ __forceinline__ uint32_t umma_idesc(int n) {
    return (1u << 4) | OpTraits<E>::IDESC_AB | (1u << 15) | (1u << 16) | (uint32_t(n >> 3) << 17) |
           (uint32_t(TBM >> 4) << 24);
}
template <typename E>
__device__ __forceinline__ void umma(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc);
template <>
__device__ __forceinline__ void umma<float>(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
        "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
        : "memory");
}
template <>
__device__ __forceinline__ void umma<__half>(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
        "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
        : "memory");
}
template <>
__device__ __forceinline__ void umma<HalfSplit>(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc,
                                                uint32_t acc) {
    umma<__half>(tmem, ad, bd, idesc, acc);
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int e = 0; e < 16; ++e) v[e] = __uint_as_float(r[e]);
}

__device__ __forceinline__ int find_task(const GemmTask *tasks, int ntasks, int t) {
    int lo = 0, hi = ntasks - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (tasks[mid].tile_base <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <typename E, int STAGES, int MINB, int CTA_N>
__global__ void __launch_bounds__(kThreads, MINB) gemm_tma_kernel(const GemmTask *__restrict__ tasks, int ntasks,
                                                               const CUtensorMap *__restrict__ maps, float *Cbase,
                                                               const int32_t *__restrict__ sexp, int *err,
                                                               int lo_maps) {
    using Tr = OpTraits<E>;
    using SS = StageShape<E, CTA_N>;
    constexpr bool SPLIT = SS::SPLIT;
    constexpr int HALVES = TBN / CTA_N;                 // CTAs per 256-column task tile
    constexpr int TMEM_COLS = SPLIT ? 2 * CTA_N : CTA_N;   // split: second accumulator at column CTA_N
    extern __shared__ __align__(1024) unsigned char tma_smem_raw[];
    __shared__ __align__(8) uint64_t bars[2 * STAGES + 1];
    __shared__ uint32_t tmem_holder;

    const int t = blockIdx.x / HALVES, hj = blockIdx.x % HALVES;
    const GemmTask tk = tasks[find_task(tasks, ntasks, t)];
    // groups of kGroupM row tiles sweep the columns (co-resident CTAs share panels in L2)
    const int local = t - tk.tile_base;
    const int per_group = kGroupM * tk.tiles_n;
    const int first = (local / per_group) * kGroupM;
    const int gs = min(kGroupM, tk.tiles_m - first);
    const int ti = first + (local % per_group) % gs, tj = (local % per_group) / gs;
    const int i0 = ti * TBM, j0 = tj * TBN + hj * CTA_N;   // CTA tile origin in shifted coordinates
    const int da = tk.shift & 255, db = tk.shift >> 8;  // shifted row x is operand row x - d
    if ((tk.lower && i0 + TBM - 1 - da < j0 - db) || tk.k <= 0 || j0 >= tk.n + db) return;   // CTA-uniform
    const int bn = (tk.n + db - j0 <= 128) ? 128 : CTA_N;
    const int nk = (tk.k + Tr::TBK - 1) / Tr::TBK;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    const uint32_t raw = smem_addr(tma_smem_raw);
    const uint32_t sbase = (raw + 1023u) & ~1023u;
    const uint32_t full0 = smem_addr(&bars[0]);
    const uint32_t empty0 = smem_addr(&bars[STAGES]);
    const uint32_t done = smem_addr(&bars[2 * STAGES]);

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full0 + 8 * s, 1);
            mbar_init(empty0 + 8 * s, 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_addr(&tmem_holder)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_holder;

    if (warp == 0) {
        // ---------------- TMA producer
        if (lane == 0) {
            const CUtensorMap *am = maps + tk.amap;
            const CUtensorMap *bm = maps + tk.bmap;
            tmap_acquire(am);
            if (tk.bmap != tk.amap) tmap_acquire(bm);
            const CUtensorMap *aml = maps + (SPLIT ? tk.amap + lo_maps : tk.amap);
            const CUtensorMap *bml = maps + (SPLIT ? tk.bmap + lo_maps : tk.bmap);
            if (SPLIT) {
                tmap_acquire(aml);
                if (tk.bmap != tk.amap) tmap_acquire(bml);
            }
            const uint32_t bytes = uint32_t(SS::A + (bn / Tr::ATOM) * SS::BOX) * (SPLIT ? 2u : 1u);
            int issued = 0;
            for (int kb = 0; kb < nk; ++kb) {
                const int s = kb % STAGES;
                if (kb >= STAGES && !mbar_wait(empty0 + 8 * s, uint32_t((kb / STAGES) - 1) & 1u, err)) break;
                const uint32_t sa = sbase + uint32_t(s) * SS::BYTES;
                const uint32_t sb = sa + SS::A;
                const uint32_t fb = full0 + 8 * s;
                mbar_expect_tx(fb, bytes);
                const int ky = kb * Tr::TBK;
#pragma unroll
                for (int g = 0; g < TBM / Tr::ATOM; ++g)
                    tma_load_2d(sa + uint32_t(g) * SS::BOX, am, tk.ax + i0 + g * Tr::ATOM, tk.ay + ky, fb);
                for (int g = 0; g < bn / Tr::ATOM; ++g)
                    tma_load_2d(sb + uint32_t(g) * SS::BOX, bm, tk.bx + j0 + g * Tr::ATOM, tk.by + ky, fb);
                if constexpr (SPLIT) {
                    const uint32_t sal = sa + SS::A + SS::B, sbl = sal + SS::A;
#pragma unroll
                    for (int g = 0; g < TBM / Tr::ATOM; ++g)
                        tma_load_2d(sal + uint32_t(g) * SS::BOX, aml, tk.ax + i0 + g * Tr::ATOM, tk.ay + ky, fb);
                    for (int g = 0; g < bn / Tr::ATOM; ++g)
                        tma_load_2d(sbl + uint32_t(g) * SS::BOX, bml, tk.bx + j0 + g * Tr::ATOM, tk.by + ky, fb);
                }
                issued = kb + 1;
            }
            // the copies this thread issued land before the CTA can exit
            for (int kb = max(0, issued - STAGES); kb < issued; ++kb)
                mbar_drain(full0 + 8 * (kb % STAGES), uint32_t(kb / STAGES) & 1u);
        }
    } else if (warp == 1) {
        // ---------------- MMA issuer
        if (lane == 0) {
            const uint32_t idesc = umma_idesc<E>(bn);
            bool broke = false;
            for (int kb = 0; kb < nk; ++kb) {
                const int s = kb % STAGES;
                if (!mbar_wait(full0 + 8 * s, uint32_t(kb / STAGES) & 1u, err)) {
                    broke = true;
                    break;
                }
                tc_fence_after();
                const uint32_t sa = sbase + uint32_t(s) * SS::BYTES;
                const uint32_t sb = sa + SS::A;
#pragma unroll
                for (int g = 0; g < Tr::TBK / Tr::MMA_K; ++g) {
                    const uint32_t off = uint32_t(g) * 128u * Tr::MMA_K;
                    const uint64_t ad = umma_desc(sa + off, SS::BOX, Tr::SBO, Tr::LAYOUT);
                    const uint64_t bd = umma_desc(sb + off, SS::BOX, Tr::SBO, Tr::LAYOUT);
                    const uint32_t first = (kb > 0 || g > 0) ? 1u : 0u;
                    umma<E>(tmem, ad, bd, idesc, first);
                    if constexpr (SPLIT) {
                        // cross terms hi x lo + lo x hi into the second accumulator
                        const uint32_t sal = sa + SS::A + SS::B, sbl = sal + SS::A;
                        const uint64_t adl = umma_desc(sal + off, SS::BOX, Tr::SBO, Tr::LAYOUT);
                        const uint64_t bdl = umma_desc(sbl + off, SS::BOX, Tr::SBO, Tr::LAYOUT);
                        umma<E>(tmem + CTA_N, ad, bdl, idesc, first);
                        umma<E>(tmem + CTA_N, adl, bd, idesc, 1u);
                    }
                }
                umma_commit(empty0 + 8 * s);
            }
            umma_commit(done);
            if (broke) mbar_drain(done, 0u);
        }
    } else {
        // ---------------- epilogue: TMEM -> registers -> C
        bool ok = true;
        if (lane == 0) ok = mbar_wait(done, 0u, err);
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        if (ok) {
            tc_fence_after();
            const int q = warp & 3;                      // TMEM lanes 32q .. 32q+31
            const int half = (warp - 2) >> 2;            // column half of the tile
            const int row = i0 + q * 32 + lane - da;     // operand row
            const int cw = bn / 2;
            const int se = sexp ? 2 * sexp[tk.amap] : tk.scale_exp;
            const float scale = se ? ldexpf(1.0f, se) : 1.0f;
            float *C = Cbase + tk.c_off;
            for (int c0 = half * cw; c0 < (half + 1) * cw; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + (uint32_t(q * 32) << 16) + uint32_t(c0), v);
                if constexpr (SPLIT) {
                    // hi x hi + 2^-11 (hi x lo + lo x hi)
                    float x[16];
                    tmem_ld16(tmem + (uint32_t(q * 32) << 16) + uint32_t(CTA_N + c0), x);
#pragma unroll
                    for (int e = 0; e < 16; ++e) v[e] = fmaf(x[e], 0x1p-11f, v[e]);
                }
                if (row >= 0 && row < tk.m) {
                    const int jb = j0 + c0 - db;
                    const int e_lo = max(0, -jb);
                    const int e_hi = min(16, (tk.lower ? min(tk.n, row + 1) : tk.n) - jb);
                    float *p = C + int64_t(jb) * tk.ldc + row;
                    float cv[16];
#pragma unroll
                    for (int e = 0; e < 16; ++e)
                        if (e >= e_lo && e < e_hi) cv[e] = p[int64_t(e) * tk.ldc];
#pragma unroll
                    for (int e = 0; e < 16; ++e)
                        if (e >= e_lo && e < e_hi) p[int64_t(e) * tk.ldc] = fmaf(-scale, v[e], cv[e]);
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS)
                     : "memory");
    }
}

// Ring depth, CTAs per SM and columns per CTA. The single-operand forms run two CTAs
// per SM (two 48 KB stages each, 256 TMEM columns each), so that one CTA's epilogue
// (the C read-modify-write) overlaps the other's main loop. Split FP16 holds two
// accumulators; it splits every 256-column task tile between two CTAs of 128 columns
// (two 128-column accumulators, 256 TMEM columns; three 32 KB stages) for the same
// two-CTA overlap (one 256-column CTA would hold all 512 TMEM columns alone).
template <typename E>
struct Occupancy {
    static constexpr int STAGES = 2, MINB = 2, CTA_N = TBN;
};
template <>
struct Occupancy<HalfSplit> {
    static constexpr int STAGES = 3, MINB = 2, CTA_N = 128;
};
template <typename E>
constexpr int tma_smem() {
    return Occupancy<E>::STAGES * StageShape<E, Occupancy<E>::CTA_N>::BYTES + 1024;
}
static_assert(2 * (tma_smem<float>() + 1024) <= 228 * 1024, "2 CTAs / SM");
static_assert(2 * (tma_smem<__half>() + 1024) <= 228 * 1024, "2 CTAs / SM");
static_assert(2 * (tma_smem<HalfSplit>() + 1024) <= 228 * 1024, "2 CTAs / SM");

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

template <typename E>
void launch_tma(const GemmTask *tasks, int ntasks, int ntiles, const void *maps, float *C, const int32_t *sexp,
                int *err, cudaStream_t st, int lo_maps) {
    if (ntiles <= 0) return;
    static PerDeviceOnce once;
    once([] {
        cudaFuncSetAttribute(gemm_tma_kernel<E, Occupancy<E>::STAGES, Occupancy<E>::MINB, Occupancy<E>::CTA_N>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, tma_smem<E>());
    });
    ++g_kernel_launches;
    constexpr int halves = TBN / Occupancy<E>::CTA_N;
    gemm_tma_kernel<E, Occupancy<E>::STAGES, Occupancy<E>::MINB, Occupancy<E>::CTA_N>
        <<<ntiles * halves, kThreads, tma_smem<E>(), st>>>(
        tasks, ntasks, static_cast<const CUtensorMap *>(maps), C, sexp, err, lo_maps);
}

}  // namespace

static_assert(sizeof(CUtensorMap) == kTensorMapBytes, "tensor map size");

bool encode_operand_map(void *out, const void *base, int operands, uint64_t rows, uint64_t cols, uint64_t ld) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn || operands < 0 || operands > 2) return false;
    const bool half = operands != 0;
    const uint32_t es = half ? 2 : 4;
    // the box is one 128-byte group of rows by the k rows of one ring stage
    const uint32_t box_k = operands == 2 ? uint32_t(OpTraits<HalfSplit>::TBK)
                           : half        ? uint32_t(OpTraits<__half>::TBK)
                                         : uint32_t(OpTraits<float>::TBK);
    static_assert(StageShape<HalfSplit, 128>::BOX == 128 * OpTraits<HalfSplit>::TBK, "split box");
    cuuint64_t dims[2] = {rows, cols};
    cuuint64_t strides[1] = {ld * es};
    cuuint32_t box[2] = {128u / es, box_k};
    cuuint32_t estr[2] = {1, 1};
    const CUresult r =
        fn(static_cast<CUtensorMap *>(out), half ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
           2, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
           half ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

bool encode_plain_map(void *out, const void *base, int esize, uint64_t rows, uint64_t cols, uint64_t ld,
                      uint32_t box_rows, uint32_t box_cols) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn || (esize != 4 && esize != 8)) return false;
    cuuint64_t dims[2] = {rows, cols};
    cuuint64_t strides[1] = {ld * uint64_t(esize)};
    cuuint32_t box[2] = {box_rows, box_cols};
    cuuint32_t estr[2] = {1, 1};
    const CUresult r = fn(static_cast<CUtensorMap *>(out),
                          esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2,
                          const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

void launch_gemm_tma(int operands, const GemmTask *tasks, int ntasks, int ntiles, const void *maps, float *C,
                     const int32_t *sexp, int *err, cudaStream_t st, int lo_maps) {
    if (operands == 2) launch_tma<HalfSplit>(tasks, ntasks, ntiles, maps, C, sexp, err, st, lo_maps);
    else if (operands == 1) launch_tma<__half>(tasks, ntasks, ntiles, maps, C, sexp, err, st, 0);
    else launch_tma<float>(tasks, ntasks, ntiles, maps, C, sexp, err, st, 0);
}

}  // namespace mfs
