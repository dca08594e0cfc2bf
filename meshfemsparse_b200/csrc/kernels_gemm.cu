// Tensor-core tile GEMMs for the supernodal Schur updates (K5) and the
// inverse-based panel solves (K4):
//     mode 0:  C(i,j) -= sum_k A(i,k) B(j,k)      (SYRK / trailing update, "NT")
//     mode 1:  C(i,j)  = sum_k A(i,k) B(j,k)      (panel rows times inv(L_kk)^T)
// A, B and C are column-major sub-blocks addressed by per-task offsets; a task
// covers an m x n block with tiles_m x tiles_n CTA tiles and an optional lower
// mask (only i >= j is touched, tiles strictly above the diagonal exit early).
// One launch carries the tasks of every large front of a level.
//
// FP32 factors: single-pass TF32 runs on the 5th-generation tensor cores
// (tcgen05, kernels_gemm_tc.cu); the split 3xTF32 form (a = a_hi + a_lo, three
// products, FP32-level accuracy) and a legacy single-pass form run here on
// mma.sync m16n8k8. FP64 factors run on the FP64 tensor-core path (mma.sync
// m8n8k4 DMMA). Tiles are staged through shared memory with 4/8-byte cp.async,
// double buffered. An FP32 task tile is 128 x 256 (the tcgen05 tile); the
// mma.sync kernel covers it as two 128 x 128 halves and ignores the tcgen05
// alignment shift (its extra tiles find no rows or columns).
#include "device.h"

#include <cstdint>

namespace mfs {

namespace {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void cp_async4(void *dst, const void *src, bool valid) {
    const uint32_t d = smem_u32(dst);
    const int sz = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src, bool valid) {
    const uint32_t d = smem_u32(dst);
    const int sz = valid ? 8 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ void mma_f64(double (&c)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ int find_task(const GemmTask *tasks, int ntasks, int t) {
    int lo = 0, hi = ntasks - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (tasks[mid].tile_base <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------- TF32 ----
constexpr int TBM = 128, TBN = 128, TBK = 32, TLD = TBM + 8;   // TLD % 32 == 8: conflict-free fragments
constexpr int kTF32Smem = 2 * 2 * TBK * TLD * 4;
constexpr int kTaskTileN32 = 256;                                // FP32 task tile width

template <int SPLIT>
__device__ __forceinline__ void tf32_tile(const GemmTask &tk, int i0, int j0, const float *Abase,
                                          const float *__restrict__ Bbase, float *Cbase, float *As, float *Bs) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 1, wn = warp >> 1;        // 2 x 4 warps, warp tile 64 x 32
    const int gid = lane >> 2, tig = lane & 3;
    const float *A = Abase + tk.a_off;
    const float *B = Bbase + tk.b_off;
    const int K = tk.k;

    auto load = [&](int stage, int k0) {
        float *as = As + stage * TBK * TLD;
        float *bs = Bs + stage * TBK * TLD;
#pragma unroll
        for (int r = 0; r < (TBK * TBM) / 256; ++r) {
            const int l = tid + 256 * r;
            const int kk = l / TBM, ii = l % TBM;
            const int gk = k0 + kk;
            const bool va = (i0 + ii < tk.m) && gk < K;
            const bool vb = (j0 + ii < tk.n) && gk < K;
            cp_async4(as + kk * TLD + ii, va ? A + int64_t(gk) * tk.lda + i0 + ii : A, va);
            cp_async4(bs + kk * TLD + ii, vb ? B + int64_t(gk) * tk.ldb + j0 + ii : B, vb);
        }
        cp_commit();
    };

    float acc[4][4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.f;

    const int nk = (K + TBK - 1) / TBK;
    load(0, 0);
    for (int kc = 0; kc < nk; ++kc) {
        if (kc + 1 < nk) {
            load((kc + 1) & 1, (kc + 1) * TBK);
            cp_wait<1>();
        } else {
            cp_wait<0>();
        }
        __syncthreads();
        const float *as = As + (kc & 1) * TBK * TLD;
        const float *bs = Bs + (kc & 1) * TBK * TLD;
#pragma unroll
        for (int k8 = 0; k8 < TBK; k8 += 8) {
            uint32_t ah[4][4], bh[4][2];
            uint32_t al[4][4], bl[4][2];
#pragma unroll
            for (int mt = 0; mt < 4; ++mt) {
                const int m = wm * 64 + mt * 16 + gid;
                const float v0 = as[(k8 + tig) * TLD + m], v1 = as[(k8 + tig) * TLD + m + 8];
                const float v2 = as[(k8 + tig + 4) * TLD + m], v3 = as[(k8 + tig + 4) * TLD + m + 8];
                ah[mt][0] = to_tf32(v0); ah[mt][1] = to_tf32(v1); ah[mt][2] = to_tf32(v2); ah[mt][3] = to_tf32(v3);
                if (SPLIT == 3) {
                    al[mt][0] = to_tf32(v0 - __uint_as_float(ah[mt][0]));
                    al[mt][1] = to_tf32(v1 - __uint_as_float(ah[mt][1]));
                    al[mt][2] = to_tf32(v2 - __uint_as_float(ah[mt][2]));
                    al[mt][3] = to_tf32(v3 - __uint_as_float(ah[mt][3]));
                }
            }
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                const int n = wn * 32 + nt * 8 + gid;
                const float v0 = bs[(k8 + tig) * TLD + n], v1 = bs[(k8 + tig + 4) * TLD + n];
                bh[nt][0] = to_tf32(v0); bh[nt][1] = to_tf32(v1);
                if (SPLIT == 3) {
                    bl[nt][0] = to_tf32(v0 - __uint_as_float(bh[nt][0]));
                    bl[nt][1] = to_tf32(v1 - __uint_as_float(bh[nt][1]));
                }
            }
#pragma unroll
            for (int mt = 0; mt < 4; ++mt)
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) {
                    if (SPLIT == 3) {
                        mma_tf32(acc[mt][nt], al[mt], bh[nt]);
                        mma_tf32(acc[mt][nt], ah[mt], bl[nt]);
                    }
                    mma_tf32(acc[mt][nt], ah[mt], bh[nt]);
                }
        }
        __syncthreads();
    }
    float *C = Cbase + tk.c_off;
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int i = i0 + wm * 64 + mt * 16 + gid + (e >> 1) * 8;
                const int j = j0 + wn * 32 + nt * 8 + tig * 2 + (e & 1);
                if (i >= tk.m || j >= tk.n || (tk.lower && i < j)) continue;
                float *p = C + int64_t(j) * tk.ldc + i;
                if (tk.mode == 0) *p -= acc[mt][nt][e];
                else *p = acc[mt][nt][e];
            }
}

template <int SPLIT>
__global__ void __launch_bounds__(256) gemm_tf32_kernel(const GemmTask *__restrict__ tasks, int ntasks,
                                                        const float *Abase, const float *__restrict__ Bbase,
                                                        float *Cbase) {
    extern __shared__ __align__(16) float sm[];
    float *As = sm;                           // [2][TBK][TLD]
    float *Bs = sm + 2 * TBK * TLD;           // [2][TBK][TLD]
    const int t = blockIdx.x;
    const GemmTask tk = tasks[find_task(tasks, ntasks, t)];
    const int local = t - tk.tile_base;
    const int ti = local % tk.tiles_m, tj = local / tk.tiles_m;
    const int i0 = ti * TBM;
    // The halves run in order; an in-place task (C == A, n <= 128) is finished
    // by the first half before the second one (which has no columns) starts.
    for (int h = 0; h < kTaskTileN32 / TBN; ++h) {
        const int j0 = tj * kTaskTileN32 + h * TBN;
        if (j0 >= tk.n || (tk.lower && i0 + TBM - 1 < j0)) break;
        if (h) __syncthreads();
        tf32_tile<SPLIT>(tk, i0, j0, Abase, Bbase, Cbase, As, Bs);
    }
}

// ---------------------------------------------------------------- FP64 ----
constexpr int DBM = 128, DBN = 64, DBK = 16, DLDA = DBM + 4, DLDB = DBN + 4;
constexpr int kF64Smem = 2 * DBK * (DLDA + DLDB) * 8;

__global__ void __launch_bounds__(256) gemm_f64_kernel(const GemmTask *__restrict__ tasks, int ntasks,
                                                       const double *Abase, const double *__restrict__ Bbase,
                                                       double *Cbase) {
    extern __shared__ __align__(16) double smd[];
    double *As = smd;                          // [2][DBK][DLDA]
    double *Bs = smd + 2 * DBK * DLDA;         // [2][DBK][DLDB]
    const int t = blockIdx.x;
    const GemmTask tk = tasks[find_task(tasks, ntasks, t)];
    const int local = t - tk.tile_base;
    const int ti = local % tk.tiles_m, tj = local / tk.tiles_m;
    const int i0 = ti * DBM, j0 = tj * DBN;
    if (tk.lower && i0 + DBM - 1 < j0) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;        // 4 x 2 warps, warp tile 32 x 32
    const int gid = lane >> 2, tig = lane & 3;
    const double *A = Abase + tk.a_off;
    const double *B = Bbase + tk.b_off;
    const int K = tk.k;

    auto load = [&](int stage, int k0) {
        double *as = As + stage * DBK * DLDA;
        double *bs = Bs + stage * DBK * DLDB;
#pragma unroll
        for (int r = 0; r < (DBK * DBM) / 256; ++r) {
            const int l = tid + 256 * r;
            const int kk = l / DBM, ii = l % DBM;
            const int gk = k0 + kk;
            const bool va = (i0 + ii < tk.m) && gk < K;
            cp_async8(as + kk * DLDA + ii, va ? A + int64_t(gk) * tk.lda + i0 + ii : A, va);
        }
#pragma unroll
        for (int r = 0; r < (DBK * DBN) / 256; ++r) {
            const int l = tid + 256 * r;
            const int kk = l / DBN, jj = l % DBN;
            const int gk = k0 + kk;
            const bool vb = (j0 + jj < tk.n) && gk < K;
            cp_async8(bs + kk * DLDB + jj, vb ? B + int64_t(gk) * tk.ldb + j0 + jj : B, vb);
        }
        cp_commit();
    };

    double acc[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;

    const int nk = (K + DBK - 1) / DBK;
    load(0, 0);
    for (int kc = 0; kc < nk; ++kc) {
        if (kc + 1 < nk) {
            load((kc + 1) & 1, (kc + 1) * DBK);
            cp_wait<1>();
        } else {
            cp_wait<0>();
        }
        __syncthreads();
        const double *as = As + (kc & 1) * DBK * DLDA;
        const double *bs = Bs + (kc & 1) * DBK * DLDB;
#pragma unroll
        for (int k4 = 0; k4 < DBK; k4 += 4) {
            double a[4], b[4];
#pragma unroll
            for (int mt = 0; mt < 4; ++mt) a[mt] = as[(k4 + tig) * DLDA + wm * 32 + mt * 8 + gid];
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) b[nt] = bs[(k4 + tig) * DLDB + wn * 32 + nt * 8 + gid];
#pragma unroll
            for (int mt = 0; mt < 4; ++mt)
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) mma_f64(acc[mt][nt], a[mt], b[nt]);
        }
        __syncthreads();
    }
    double *C = Cbase + tk.c_off;
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int i = i0 + wm * 32 + mt * 8 + gid;
                const int j = j0 + wn * 32 + nt * 8 + tig * 2 + e;
                if (i >= tk.m || j >= tk.n || (tk.lower && i < j)) continue;
                double *p = C + int64_t(j) * tk.ldc + i;
                if (tk.mode == 0) *p -= acc[mt][nt][e];
                else *p = acc[mt][nt][e];
            }
}

}  // namespace

int gemm_tile_m(bool fp64) { return fp64 ? DBM : TBM; }
int gemm_tile_n(bool fp64) { return fp64 ? DBN : kTaskTileN32; }

template <>
void launch_gemm<float>(const GemmTask *tasks, int ntasks, int ntiles, const float *A, const float *B, float *C,
                        int split, int *err, cudaStream_t st) {
    if (ntiles <= 0) return;
    if (split == 1) {
        launch_gemm_tc(tasks, ntasks, ntiles, A, B, C, err, st);
        return;
    }
    ++g_kernel_launches;
    if (split == 3) {
        static PerDeviceOnce once3;
        once3([] { cudaFuncSetAttribute(gemm_tf32_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTF32Smem); });
        gemm_tf32_kernel<3><<<ntiles, 256, kTF32Smem, st>>>(tasks, ntasks, A, B, C);
    } else {
        static PerDeviceOnce once1;
        once1([] { cudaFuncSetAttribute(gemm_tf32_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTF32Smem); });
        gemm_tf32_kernel<1><<<ntiles, 256, kTF32Smem, st>>>(tasks, ntasks, A, B, C);
    }
}

template <>
void launch_gemm<double>(const GemmTask *tasks, int ntasks, int ntiles, const double *A, const double *B, double *C,
                         int split, int *err, cudaStream_t st) {
    (void)split;
    (void)err;
    if (ntiles <= 0) return;
    ++g_kernel_launches;
    static PerDeviceOnce once;
    once([] { cudaFuncSetAttribute(gemm_f64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kF64Smem); });
    gemm_f64_kernel<<<ntiles, 256, kF64Smem, st>>>(tasks, ntasks, A, B, C);
}

}  // namespace mfs
