// Large-front column block, first half of K3 + K4: factor the nb x nb
// diagonal block of one column block and invert it.
//
// One launch per column block of all large fronts of a level, one CTA per
// front. The CTA factors the block in shared memory, writes L back in place,
// stores the full inverse inv(L) (nb x nb, column-major, ld ldi) to scratch and
// the 64 x 64 diagonal blocks of inv(L) after the panels for the triangular
// solves. The rows below the block are then solved on the tensor cores as the
// GEMM  X := X inv(L)^T  (launched by the host right after this kernel), so
// the O(m nb^2) part of the TRSM runs at GEMM speed.
//
// The diagonal block is processed in 32-column sub-panels:
//   warp 0 factors the 32 x 32 sub-block with each lane holding its row in
//   registers (column broadcast by warp shuffles), the rows below are solved one
//   thread per row with the row in registers, and the trailing part of the block
//   gets the rank-32 update. The inverse is built blockwise: 32 x 32 diagonal
//   inverses (one warp each, lane = column), then off-diagonal blocks
//   inv(L)_IJ = -inv(L_II) sum_{K=J}^{I-1} L_IK inv(L)_KJ by block distance.
#include "device.h"

namespace mfs {

namespace {

template <typename T>
__device__ __forceinline__ T psqrt(T x);
template <>
__device__ __forceinline__ double psqrt<double>(double x) { return sqrt(x); }
template <>
__device__ __forceinline__ float psqrt<float>(float x) { return sqrtf(x); }

// inv(L) feeding a single-pass TF32 tensor-core row solve is stored rounded to
// TF32 (nearest); the tensor cores would truncate it.
template <typename T>
__device__ __forceinline__ T round_operand(T x) { return x; }
template <>
__device__ __forceinline__ float round_operand<float>(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// Same rule as the small-front kernel: report (plain) or perturb (refined FP32).
template <typename T>
__device__ __forceinline__ T panel_bad_pivot(T a, int col, const PivotCtl &pv, bool record) {
    if (pv.dorig) {
        const T floor_v = T(1e-3 * fabs(pv.dorig[col]));
        const T m = fabs(a);
        if (record) atomicAdd(pv.perturbed, 1);
        return (m > floor_v) ? m : (floor_v > T(0) ? floor_v : T(1));
    }
    if (record) atomicMin(pv.fail_col, col);
    return T(1);
}

// Cholesky of the cw x cw sub-block at (c0, c0) of D (ld LDD) by one warp.
template <typename T>
__device__ __forceinline__ void warp_potrf32(T *D, int LDD, int c0, int cw, int lane, int col_base,
                                             const PivotCtl &pv, bool record) {
    T r[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) r[j] = (j < cw && lane < cw && j <= lane) ? D[(c0 + j) * LDD + c0 + lane] : T(0);
#pragma unroll
    for (int k = 0; k < 32; ++k) {
        if (k < cw) {
            T piv = __shfl_sync(0xffffffffu, r[k], k);
            if (!(piv > T(0))) piv = panel_bad_pivot(piv, col_base + k, pv, record && lane == 0);
            const T lkk = psqrt(piv);
            const T lik = (lane == k) ? lkk : r[k] / lkk;
            if (lane >= k) r[k] = lik;
#pragma unroll
            for (int j = k + 1; j < 32; ++j) {
                const T ljk = __shfl_sync(0xffffffffu, lik, j);
                if (lane >= j && j < cw) r[j] -= lik * ljk;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < 32; ++j)
        if (j < cw && lane < cw && j <= lane) D[(c0 + j) * LDD + c0 + lane] = r[j];
}

template <typename T>
__global__ void __launch_bounds__(256, 1) panel_kernel(const PanelTask *__restrict__ tasks,
                                                       T *__restrict__ factor, T *__restrict__ inv_scratch,
                                                       PivotCtl pv, bool round_inv) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const PanelTask tk = tasks[blockIdx.x];
    const int nb = tk.nb, ld = tk.ld;
    const int LDD = nb + 1;
    const int nblk = (nb + 31) / 32;
    T *D = reinterpret_cast<T *>(smem_raw);          // L, column-major, ld LDD
    T *Iv = D + nb * LDD;                            // inv(L), column-major, ld LDD
    T *Tm = Iv + nb * LDD;                           // 3 x [32][33] temporaries of the blocked inverse
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    T *blk = factor + tk.off;
    for (int q = tid; q < nb * nb; q += nt) {
        const int j = q / nb, i = q - j * nb;
        D[j * LDD + i] = i >= j ? blk[int64_t(j) * ld + i] : T(0);
        Iv[j * LDD + i] = T(0);
    }
    __syncthreads();
    // ---- factor D
    for (int c0 = 0; c0 < nb; c0 += 32) {
        const int cw = min(32, nb - c0);
        if (warp == 0) warp_potrf32(D, LDD, c0, cw, lane, tk.col + c0, pv, true);
        __syncthreads();
        for (int row = c0 + cw + tid; row < nb; row += nt) {
            T x[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) x[j] = j < cw ? D[(c0 + j) * LDD + row] : T(0);
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                if (j < cw) {
                    T a = x[j];
#pragma unroll
                    for (int k = 0; k < j; ++k) a -= x[k] * D[(c0 + k) * LDD + c0 + j];
                    x[j] = a / D[(c0 + j) * LDD + c0 + j];
                }
            }
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (j < cw) D[(c0 + j) * LDD + row] = x[j];
        }
        __syncthreads();
        const int mm = nb - c0 - cw;
        for (int q = tid; q < mm * mm; q += nt) {
            const int jj = q / mm, ii = q - jj * mm;
            if (ii < jj) continue;
            const int i = c0 + cw + ii, j = c0 + cw + jj;
            T a = T(0);
#pragma unroll 8
            for (int k = 0; k < cw; ++k) a += D[(c0 + k) * LDD + i] * D[(c0 + k) * LDD + j];
            D[j * LDD + i] -= a;
        }
        __syncthreads();
    }
    // ---- inv(L): diagonal 32 x 32 blocks, one warp each, lane = column
    if (warp < nblk) {
        const int b0 = warp * 32, bw = min(32, nb - b0);
        T y[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            if (i < bw) {
                T a = (i == lane) ? T(1) : T(0);
#pragma unroll
                for (int k = 0; k < i; ++k) a -= D[(b0 + k) * LDD + b0 + i] * y[k];
                y[i] = (i >= lane) ? a / D[(b0 + i) * LDD + b0 + i] : T(0);
            } else {
                y[i] = T(0);
            }
        }
        if (lane < bw)
#pragma unroll
            for (int i = 0; i < 32; ++i)
                if (i < bw && i >= lane) Iv[(b0 + lane) * LDD + b0 + i] = y[i];
    }
    __syncthreads();
    // ---- off-diagonal blocks by distance
    for (int dist = 1; dist < nblk; ++dist) {
        const int nbl = nblk - dist;                 // blocks (I, J = I - dist), I = dist .. nblk-1
        // Tm[J] = sum_{K=J}^{I-1} L_IK inv(L)_KJ
        for (int q = tid; q < nbl * 1024; q += nt) {
            const int bq = q >> 10, e = q & 1023;
            const int j = e >> 5, i = e & 31;
            const int J = bq, I = bq + dist;
            const int gi = I * 32 + i, gj = J * 32 + j;
            T a = T(0);
            if (gi < nb && gj < nb)
                for (int k = J * 32; k < I * 32; ++k) a += D[k * LDD + gi] * Iv[gj * LDD + k];
            Tm[bq * 32 * 33 + j * 33 + i] = a;
        }
        __syncthreads();
        // inv(L)_IJ = -inv(L_II) Tm
        for (int q = tid; q < nbl * 1024; q += nt) {
            const int bq = q >> 10, e = q & 1023;
            const int j = e >> 5, i = e & 31;
            const int J = bq, I = bq + dist;
            const int gi = I * 32 + i, gj = J * 32 + j;
            if (gi < nb && gj < nb) {
                T a = T(0);
                for (int k = 0; k <= i; ++k) a += Iv[(I * 32 + k) * LDD + gi] * Tm[bq * 32 * 33 + j * 33 + k];
                Iv[gj * LDD + gi] = -a;
            }
        }
        __syncthreads();
    }
    for (int q = tid; q < nb * nb; q += nt) {
        const int j = q / nb, i = q - j * nb;
        if (i >= j) blk[int64_t(j) * ld + i] = D[j * LDD + i];
        T v = i >= j ? Iv[j * LDD + i] : T(0);
        if (round_inv) v = round_operand(v);
        inv_scratch[tk.inv_full + int64_t(j) * tk.ldi + i] = v;
    }
    if (tk.inv_out >= 0) {
        // 64 x 64 diagonal blocks of inv(L) (the inverses of L's 64 x 64 diagonal blocks)
        const int nb64 = (nb + 63) / 64;
        T *inv = factor + tk.inv_out;
        for (int q = tid; q < nb64 * 4096; q += nt) {
            const int b = q >> 12, e = q & 4095;
            const int j = e >> 6, i = e & 63;
            const int gi = b * 64 + i, gj = b * 64 + j;
            inv[q] = (gi < nb && gj < nb && gi >= gj) ? Iv[gj * LDD + gi] : T(0);
        }
    }
}

}  // namespace

size_t panel_smem_bytes(int nb, bool fp64) {
    const size_t el = fp64 ? 8 : 4;
    return (size_t(2) * nb * (nb + 1) + 3 * 32 * 33) * el;
}

template <typename T>
void launch_panel(const PanelTask *tasks, int ntasks, int max_nb, T *factor, T *inv_scratch, PivotCtl pv,
                  bool round_inv, cudaStream_t st) {
    if (ntasks <= 0) return;
    const size_t smem = panel_smem_bytes(max_nb, sizeof(T) == 8);
    static const bool smem_ok =
        (cudaFuncSetAttribute(panel_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmemOptin), true);
    (void)smem_ok;
    ++g_kernel_launches;
    panel_kernel<T><<<ntasks, 256, smem, st>>>(tasks, factor, inv_scratch, pv, round_inv);
}

template void launch_panel<float>(const PanelTask *, int, int, float *, float *, PivotCtl, bool, cudaStream_t);
template void launch_panel<double>(const PanelTask *, int, int, double *, double *, PivotCtl, bool, cudaStream_t);

}  // namespace mfs
