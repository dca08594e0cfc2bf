// TF32 Schur-update GEMM on the 5th-generation tensor cores (tcgen05).
//
//     mode 0:  C(i,j) -= sum_k A(i,k) B(j,k)      (SYRK / trailing update)
//     mode 1:  C(i,j)  = sum_k A(i,k) B(j,k)      (panel rows times inv(L_kk)^T)
//
// With FP16 Schur-update operands the row solve also writes each result, scaled
// by its front's power of two, as FP16 into the half copy of the panels, and
// stores the FP32 factor value as that FP16 value scaled back.
//
// The tensor cores read FP32 operands as TF32 by dropping mantissa bits. The
// factorization therefore keeps every Schur-update operand TF32-exact: the row
// solve (mode 1) rounds its A operand in shared memory and its result to
// nearest (its B operand, inv(L_kk), is stored rounded by the panel kernel), so
// the L21 blocks that mode-0 updates read need no rounding, while the updated
// Schur complements accumulate in FP32.
//
// Same task lists as the mma.sync kernels (GemmTask, 128 x 256 task tiles):
// one CTA per task tile, 288 threads.
//   warps 0-7  stage A (128 x 32) and B (256 x 32, or 128 x 32 when the tile has
//              at most 128 columns left) k-blocks into a STAGES-deep ring with
//              16-byte cp.async (panel columns are 16-byte aligned; a tile starts
//              at the aligned element at or before its operand and the epilogue
//              drops the extra leading rows / columns), writing the canonical
//              MN-major operand layout directly; then they run the epilogue.
//   warp 8     allocates 256 TMEM columns (the 128 x 256 FP32 accumulator);
//              lane 0 issues tcgen05.mma.kind::tf32 (M = 128, N = 256 or 128,
//              K = 8) from shared-memory descriptors and frees ring slots with
//              tcgen05.commit.
// Shared-memory operand layout (per stage): MN-major with the 32-byte-atom
// 128-byte swizzle, the form TF32 operands take when M (or N) is the contiguous
// dimension: a 512-byte atom holds 4 k rows of 32 M elements (128 bytes), the
// 32-byte chunk index inside a row XOR-ed with the row index; the 8 atoms of a
// 32-deep stage follow each other (descriptor SBO = 512) and 32-element M
// groups are 4096 bytes apart (LBO). The MMA for k values 8g .. 8g+7 starts
// 1024g bytes into the stage. A producer warp fills one atom per instruction
// (4 k rows x 8 16-byte chunks): 128 contiguous bytes per k in global memory,
// every lane on its own banks in shared memory.
//
// Pipeline: full[s] (256 producer arrivals after each producer's copies have
// landed and been fenced to the async proxy), empty[s] (tcgen05.commit), done
// (tcgen05.commit after the last MMA). Every wait is bounded in time; on expiry
// the kernel records an error in *err, stops issuing, drains its own copies,
// frees TMEM and returns, and the host reports MFS_TIMEOUT.
#include "device.h"

#include <cuda_fp16.h>

#include <cstdint>

namespace mfs {

namespace {

constexpr int UBM = 128, UBN = 256, UBK = 32;
constexpr int kUStageA = UBM * UBK * 4;              // 16 KB
constexpr int kUStageB = UBN * UBK * 4;              // 32 KB
constexpr int kUStage = kUStageA + kUStageB;         // multiple of 1024
constexpr int kUProducers = 256;
constexpr int kUThreads = kUProducers + 32;
constexpr int kUTmemCols = 256;
constexpr unsigned long long kPipeWaitNs = 1000000000ull;   // 1 s per wait at most
constexpr int kGroupM = 8;
constexpr int kTcStages = 4;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// 16-byte copy of `bytes` (0..16) source bytes, zero-filling the rest.
__device__ __forceinline__ void cp_async16_to(uint32_t dst, const void *src, int bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_commit_group() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
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
            if (global_ns() - t0 > kPipeWaitNs) {
                atomicExch(err, 1);
                return false;
            }
        }
    }
}
// Bounded wait that ignores the error flag: after a timeout the MMA issuer still
// lets the MMAs it has issued retire before the CTA frees TMEM and exits.
__device__ __forceinline__ void mbar_drain(uint32_t bar, uint32_t parity) {
    const unsigned long long t0 = global_ns();
    while (!mbar_try(bar, parity))
        if (global_ns() - t0 > kPipeWaitNs) return;
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor: 128-byte swizzle with 32-byte atoms (layout
// type 1), version 1, base offset 0.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFF) | (uint64_t((lbo >> 4) & 0x3FFF) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFF) << 32) | (uint64_t(1) << 46) | (uint64_t(1) << 61);
}
// Instruction descriptor: FP32 accumulate, TF32 A and B, both MN-major, M = 128.
__device__ __forceinline__ uint32_t umma_idesc(int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | (1u << 15) | (1u << 16) | (uint32_t(n >> 3) << 17) |
           (uint32_t(UBM >> 4) << 24);
}
__device__ __forceinline__ void umma_tf32(uint32_t tmem, uint64_t ad, uint64_t bd, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem), "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int e = 0; e < 32; ++e) v[e] = __uint_as_float(r[e]);
}

__device__ __forceinline__ float tf32_round(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}
__device__ __forceinline__ void round_tf32_16b(uint32_t addr) {
    float a, b, c, d;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(a), "=f"(b), "=f"(c), "=f"(d) : "r"(addr) : "memory");
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(tf32_round(a)), "f"(tf32_round(b)),
                 "f"(tf32_round(c)), "f"(tf32_round(d))
                 : "memory");
}

// hi = rn_tf32(x) in place, lo = x - hi (exact in FP32) at addr + lo_off.
__device__ __forceinline__ void split_tf32_16b(uint32_t addr, uint32_t lo_off) {
    float a, b, c, d;
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(a), "=f"(b), "=f"(c), "=f"(d) : "r"(addr) : "memory");
    const float ha = tf32_round(a), hb = tf32_round(b), hc = tf32_round(c), hd = tf32_round(d);
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(ha), "f"(hb), "f"(hc), "f"(hd)
                 : "memory");
    asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr + lo_off), "f"(a - ha), "f"(b - hb),
                 "f"(c - hc), "f"(d - hd)
                 : "memory");
}

// Byte offset of operand element (row x of the M or N extent, depth k < 32)
// inside one stage buffer.
__device__ __forceinline__ uint32_t swz_off(int x, int k) {
    const int r = k & 3;
    return uint32_t(x >> 5) * 4096u + uint32_t(k >> 2) * 512u + uint32_t(r) * 128u +
           uint32_t((((x >> 3) & 3) ^ r) << 5) + uint32_t(x & 7) * 4u;
}

__device__ __forceinline__ int find_gemm_task(const GemmTask *tasks, int ntasks, int t) {
    int lo = 0, hi = ntasks - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (tasks[mid].tile_base <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// SPLIT (row solves of the split-FP16 mode): A and B are split in shared memory into
// TF32 hi = rn(x) and lo = x - hi (stored one stage-size further on); the MMA adds
// hi x hi + hi x lo + lo x hi, FP32-level products. The result is stored in FP32 as
// is, and into the half copies as hi = rn16(2^-e v) and lo = rn16(2^11 (2^-e v - hi)).
template <int STAGES, bool SPLIT>
__global__ void __launch_bounds__(kUThreads, 1) gemm_tc_kernel(const GemmTask *__restrict__ tasks, int ntasks,
                                                               const float *Abase, const float *__restrict__ Bbase,
                                                               float *Cbase, int *err, __half *h16, __half *h16lo,
                                                               const int32_t *__restrict__ sexp) {
    constexpr uint32_t kSlot = SPLIT ? 2u * kUStage : uint32_t(kUStage);   // ring slot bytes
    extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
    __shared__ __align__(8) uint64_t bars[2 * STAGES + 1];
    __shared__ uint32_t tmem_holder;

    const int t = blockIdx.x;
    const GemmTask tk = tasks[find_gemm_task(tasks, ntasks, t)];
    // Tiles run in groups of kGroupM row tiles sweeping the columns, so that
    // co-resident CTAs share their A and B panels in L2.
    const int local = t - tk.tile_base;
    const int per_group = kGroupM * tk.tiles_n;
    const int first = (local / per_group) * kGroupM;
    const int gs = min(kGroupM, tk.tiles_m - first);
    const int ti = first + (local % per_group) % gs, tj = (local % per_group) / gs;
    const int i0 = ti * UBM, j0 = tj * UBN;             // tile origin in shifted coordinates
    const int da = tk.shift & 255, db = tk.shift >> 8;  // shifted row x is operand row x - d
    if ((tk.lower && i0 + UBM - 1 - da < j0 - db) || tk.k <= 0 || j0 >= tk.n + db) return;   // CTA-uniform
    const int bn = (tk.n + db - j0 <= 128) ? 128 : UBN;  // columns this tile computes
    const int K = tk.k;
    const int nk = (K + UBK - 1) / UBK;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    const uint32_t raw = smem_addr(tc_smem_raw);
    const uint32_t sbase = (raw + 1023u) & ~1023u;       // stages 1024-byte aligned
    const uint32_t full0 = smem_addr(&bars[0]);
    const uint32_t empty0 = smem_addr(&bars[STAGES]);
    const uint32_t done = smem_addr(&bars[2 * STAGES]);

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full0 + 8 * s, kUProducers);
            mbar_init(empty0 + 8 * s, 1);
        }
        mbar_init(done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 8) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_addr(&tmem_holder)),
                     "r"(kUTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_holder;

    if (warp < 8) {
        // ---------------- producers
        // Shifted operands start 16-byte aligned (leading dimensions are multiples of 4).
        const float *A = Abase + (tk.a_off - da);
        const float *B = Bbase + (tk.b_off - db);
        const int am = tk.m + da, bnn = tk.n + db;               // shifted extents
        // lane -> (k row kr of a 4-deep atom, 16-byte chunk c8 of a 128-byte row)
        const int kr = lane >> 3, c8 = lane & 7;
        const int batoms = (bn / 32) * (UBK / 4);                // B atoms staged per k-block
        bool aborted = false;
        for (int kb = 0; kb < nk + STAGES - 1; ++kb) {
            if (kb < nk) {
                const int s = kb % STAGES;
                if (kb >= STAGES && !aborted && !mbar_wait(empty0 + 8 * s, uint32_t((kb / STAGES) - 1) & 1u, err))
                    aborted = true;
                if (!aborted) {
                    const uint32_t sa = sbase + uint32_t(s) * kSlot;
                    const uint32_t sb = sa + kUStageA;
                    const int k0 = kb * UBK;
#pragma unroll
                    for (int p = warp; p < (UBM / 32) * (UBK / 4); p += 8) {
                        const int x = (p & 3) * 32 + c8 * 4, k = (p >> 2) * 4 + kr;
                        const int nv = (k0 + k < K) ? min(4, max(0, am - (i0 + x))) : 0;
                        cp_async16_to(sa + swz_off(x, k), nv ? A + int64_t(k0 + k) * tk.lda + i0 + x : A, 4 * nv);
                    }
#pragma unroll 4
                    for (int p = warp; p < batoms; p += 8) {
                        const int x = (p % (bn / 32)) * 32 + c8 * 4, k = (p / (bn / 32)) * 4 + kr;
                        const int nv = (k0 + k < K) ? min(4, max(0, bnn - (j0 + x))) : 0;
                        cp_async16_to(sb + swz_off(x, k), nv ? B + int64_t(k0 + k) * tk.ldb + j0 + x : B, 4 * nv);
                    }
                }
            }
            cp_commit_group();
            if (kb >= STAGES - 1) {
                const int j = kb - (STAGES - 1);
                cp_wait_group<STAGES - 1>();
                if constexpr (SPLIT) {
                    // split this thread's chunks of k-block j (A and B) into hi / lo
                    if (!aborted) {
                        const uint32_t sa = sbase + uint32_t(j % STAGES) * kSlot;
                        const uint32_t sb = sa + kUStageA;
#pragma unroll
                        for (int p = warp; p < (UBM / 32) * (UBK / 4); p += 8) {
                            const int x = (p & 3) * 32 + c8 * 4, k = (p >> 2) * 4 + kr;
                            split_tf32_16b(sa + swz_off(x, k), uint32_t(kUStage));
                        }
#pragma unroll 4
                        for (int p = warp; p < batoms; p += 8) {
                            const int x = (p % (bn / 32)) * 32 + c8 * 4, k = (p / (bn / 32)) * 4 + kr;
                            split_tf32_16b(sb + swz_off(x, k), uint32_t(kUStage));
                        }
                    }
                } else if (tk.mode == 1 && !aborted) {
                    // Row solve: its A operand (assembled / updated panel rows) is
                    // FP32; round this thread's chunks of k-block j to TF32 (nearest)
                    // in place, as the tensor cores would otherwise truncate them.
                    const uint32_t sa = sbase + uint32_t(j % STAGES) * kUStage;
#pragma unroll
                    for (int p = warp; p < (UBM / 32) * (UBK / 4); p += 8) {
                        const int x = (p & 3) * 32 + c8 * 4, k = (p >> 2) * 4 + kr;
                        round_tf32_16b(sa + swz_off(x, k));
                    }
                }
                fence_async_smem();
                mbar_arrive(full0 + 8 * (j % STAGES));
            }
        }
        cp_wait_group<0>();
        // ---------------- epilogue: TMEM -> registers -> C
        bool ok = true;
        if (lane == 0) ok = mbar_wait(done, 0u, err);
        ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        if (ok) {
            tc_fence_after();
            const int q = warp & 3;                      // TMEM lanes 32q .. 32q+31
            const int half = warp >> 2;                  // column half of the tile
            const int row = i0 + q * 32 + lane - da;     // operand row
            const int cw = bn / 2;
            float *C = Cbase + tk.c_off;
            for (int c0 = half * cw; c0 < (half + 1) * cw; c0 += 32) {
                float v[32];
                tmem_ld32(tmem + (uint32_t(q * 32) << 16) + uint32_t(c0), v);
                if (row >= 0 && row < tk.m) {
                    const int jb = j0 + c0 - db;
                    // columns [e_lo, e_hi) of this chunk are written
                    const int e_lo = max(0, -jb);
                    const int e_hi = min(32, (tk.lower ? min(tk.n, row + 1) : tk.n) - jb);
                    float *p = C + int64_t(jb) * tk.ldc + row;
                    if (tk.mode == 0) {
                        // all loads of the chunk first, then the stores
                        float cv[32];
#pragma unroll
                        for (int e = 0; e < 32; ++e)
                            if (e >= e_lo && e < e_hi) cv[e] = p[int64_t(e) * tk.ldc];
#pragma unroll
                        for (int e = 0; e < 32; ++e)
                            if (e >= e_lo && e < e_hi) p[int64_t(e) * tk.ldc] = cv[e] - v[e];
                    } else if (SPLIT) {
                        // FP32-level result: the factor keeps it as is; the half copies
                        // get its scaled FP16 hi part and the 2^11-scaled remainder
                        const int se = sexp[tk.sn];
                        const float down = ldexpf(1.0f, -se);
                        __half *ph = h16 + tk.c_off + int64_t(jb) * tk.ldc + row;
                        __half *pl = h16lo + tk.c_off + int64_t(jb) * tk.ldc + row;
#pragma unroll
                        for (int e = 0; e < 32; ++e)
                            if (e >= e_lo && e < e_hi) {
                                const float sv = fminf(fmaxf(v[e] * down, -65504.0f), 65504.0f);
                                const __half hv = __float2half_rn(sv);
                                ph[int64_t(e) * tk.ldc] = hv;
                                pl[int64_t(e) * tk.ldc] = __float2half_rn((sv - __half2float(hv)) * 2048.0f);
                                p[int64_t(e) * tk.ldc] = v[e];
                            }
                    } else if (!h16) {
                        // the solved rows become Schur-update operands: store them
                        // TF32-exact (rounded to nearest)
#pragma unroll
                        for (int e = 0; e < 32; ++e)
                            if (e >= e_lo && e < e_hi) p[int64_t(e) * tk.ldc] = tf32_round(v[e]);
                    } else {
                        // FP16 Schur-update operands: the row scaled by the front's power of
                        // two, rounded to FP16 (saturated) into the half copy; the factor
                        // keeps exactly that value scaled back
                        const int se = sexp[tk.sn];
                        const float down = ldexpf(1.0f, -se), up = ldexpf(1.0f, se);
                        __half *ph = h16 + tk.c_off + int64_t(jb) * tk.ldc + row;
#pragma unroll
                        for (int e = 0; e < 32; ++e)
                            if (e >= e_lo && e < e_hi) {
                                const float sv = fminf(fmaxf(v[e] * down, -65504.0f), 65504.0f);
                                const __half hv = __float2half_rn(sv);
                                ph[int64_t(e) * tk.ldc] = hv;
                                p[int64_t(e) * tk.ldc] = __half2float(hv) * up;
                            }
                    }
                }
            }
        }
    } else if (lane == 0) {
        // ---------------- MMA issuer
        const uint32_t idesc = umma_idesc(bn);
        bool broke = false;
        for (int kb = 0; kb < nk; ++kb) {
            const int s = kb % STAGES;
            if (!mbar_wait(full0 + 8 * s, uint32_t(kb / STAGES) & 1u, err)) {
                broke = true;
                break;
            }
            tc_fence_after();
            const uint32_t sa = sbase + uint32_t(s) * kSlot;
            const uint32_t sb = sa + kUStageA;
#pragma unroll
            for (int g = 0; g < UBK / 8; ++g) {
                const uint64_t ad = umma_desc(sa + uint32_t(g) * 1024u, 4096u, 512u);
                const uint64_t bd = umma_desc(sb + uint32_t(g) * 1024u, 4096u, 512u);
                umma_tf32(tmem, ad, bd, idesc, (kb > 0 || g > 0) ? 1u : 0u);
                if constexpr (SPLIT) {
                    const uint64_t adl = umma_desc(sa + kUStage + uint32_t(g) * 1024u, 4096u, 512u);
                    const uint64_t bdl = umma_desc(sb + kUStage + uint32_t(g) * 1024u, 4096u, 512u);
                    umma_tf32(tmem, ad, bdl, idesc, 1u);
                    umma_tf32(tmem, adl, bd, idesc, 1u);
                }
            }
            umma_commit(empty0 + 8 * s);
        }
        umma_commit(done);
        if (broke) mbar_drain(done, 0u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 8) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kUTmemCols)
                     : "memory");
    }
}

constexpr int kTcSmem = kTcStages * kUStage + 1024;
constexpr int kTcSplitStages = 2;
constexpr int kTcSplitSmem = kTcSplitStages * 2 * kUStage + 1024;

}  // namespace

void launch_gemm_tc(const GemmTask *tasks, int ntasks, int ntiles, const float *A, const float *B, float *C, int *err,
                    cudaStream_t st, void *h16, const int32_t *sexp, void *h16lo) {
    if (ntiles <= 0) return;
    static PerDeviceOnce once;
    once([] {
        cudaFuncSetAttribute(gemm_tc_kernel<kTcStages, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem);
        cudaFuncSetAttribute(gemm_tc_kernel<kTcSplitStages, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kTcSplitSmem);
    });
    ++g_kernel_launches;
    if (h16lo)
        gemm_tc_kernel<kTcSplitStages, true><<<ntiles, kUThreads, kTcSplitSmem, st>>>(
            tasks, ntasks, A, B, C, err, static_cast<__half *>(h16), static_cast<__half *>(h16lo), sexp);
    else
        gemm_tc_kernel<kTcStages, false><<<ntiles, kUThreads, kTcSmem, st>>>(
            tasks, ntasks, A, B, C, err, static_cast<__half *>(h16), nullptr, sexp);
}

}  // namespace mfs
