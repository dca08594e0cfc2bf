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
// The block (padded to a multiple of 32 with an identity tail) is processed in
// 32 x 32 tiles I = 0 .. nblk-1, right-looking, two barriers per tile column:
//   phase A  one warp per tile: the tiles below, L_RI = A_RI inv(L_II)^T, and the
//            inverse tiles inv(L)_IJ = -inv(L_II) sum_K P_IJK (J < I).
//   phase B  warp 0 updates tile (I+1, I+1) and at once factors it left-looking
//            (lane = row, reciprocal square root per pivot) and inverts it
//            (lane = column); warps 1-7 meanwhile run the other trailing updates
//            A_RC -= L_RI L_CI^T (R >= C > I) and the products
//            P_{I+1,J,K} = L_{I+1,K} inv(L)_KJ (J <= K <= I) that the next
//            off-diagonal inverse tiles need (they only read final tiles).
// Every tile product runs as a warp-level register-tiled 32 x 32 x 32 GEMM
// (each lane owns a 4 x 8 patch), so the chain of dependent work per tile is
// the 32 pivots of its diagonal factorization and three 32-deep products.
// The code is kept compact (rolled loops, one product routine): the work per
// CTA is small, and fully unrolled variants spent most of their time refetching
// instructions.
#include "device.h"

#include <type_traits>

namespace mfs {

namespace {

constexpr int kPanelThreads = 256;
constexpr int kPanelLoadVecs = 16;                 // 16-byte loads per thread and batch

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

template <typename T>
__device__ __forceinline__ T recip_sqrt(T x);
template <>
__device__ __forceinline__ double recip_sqrt<double>(double x) { return 1.0 / sqrt(x); }
template <>
__device__ __forceinline__ float recip_sqrt<float>(float x) { return rsqrtf(x); }

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
// Kept out of line: it is rare, and inlined into the unrolled pivot loop it
// stops that loop from being unrolled.
// With an FP64 re-factor pending (sflag), a bad pivot only marks the block: the
// FP32 pass still finishes on a floor value and the block is factored again in FP64.
template <typename T>
__device__ __noinline__ T panel_bad_pivot(T a, int col, PivotCtl pv, int *sflag) {
    if (col < 0) return T(1);
    if (sflag) {
        *sflag = 1;
        const T floor_v = T(1e-3 * fabs(pv.dorig[col]));
        const T m = fabs(a);
        return (m > floor_v) ? m : (floor_v > T(0) ? floor_v : T(1));
    }
    if (pv.dorig) {
        const T floor_v = T(1e-3 * fabs(pv.dorig[col]));
        const T m = fabs(a);
        atomicAdd(pv.perturbed, 1);
        return (m > floor_v) ? m : (floor_v > T(0) ? floor_v : T(1));
    }
    atomicMin(pv.fail_col, col);
    return T(1);
}

// Warp-level tile product: c[r][q] += sum_{k < 32} A(4 rq + r, k) * B(8 cq + q, k)
// with rq = lane % 8, cq = lane / 8; A(i, k) = A0[k * lda + i], B(j, k) = B0[j * sj + k * sk].
template <typename T>
__device__ __forceinline__ void tile_mma(T (&c)[4][8], const T *A0, int lda, const T *B0, int sj, int sk,
                                         int lane) {
    const int rq = lane & 7, cq = lane >> 3;
    const T *a = A0 + 4 * rq;
    const T *b = B0 + 8 * cq * sj;
#pragma unroll 2
    for (int k = 0; k < 32; ++k) {
        T av[4], bv[8];
#pragma unroll
        for (int r = 0; r < 4; ++r) av[r] = a[k * lda + r];
#pragma unroll
        for (int q = 0; q < 8; ++q) bv[q] = b[q * sj + k * sk];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int q = 0; q < 8; ++q) c[r][q] += av[r] * bv[q];
    }
}

template <typename T>
__device__ __forceinline__ void tile_zero(T (&c)[4][8]) {
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int q = 0; q < 8; ++q) c[r][q] = T(0);
}

// Store a lane's 4 x 8 patch into a column-major tile (element (i, j) at M[j * ldm + i]),
// scaled by s (and added to the old value when add is set).
template <typename T>
__device__ __forceinline__ void tile_store(T *M, int ldm, const T (&c)[4][8], T s, bool add, int lane) {
    const int rq = lane & 7, cq = lane >> 3;
#pragma unroll
    for (int q = 0; q < 8; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            T *p = M + (8 * cq + q) * ldm + 4 * rq + r;
            *p = add ? *p + s * c[r][q] : s * c[r][q];
        }
}

// Cholesky of the 32 x 32 tile at (c0, c0) of D by one warp, then its inverse.
// Both keep a 32-entry vector per lane in registers, processed four steps at a
// time and then shifted by four, so the current column (row) of step k0 + t is
// entry t: the outer step loop stays rolled (compact code) while every register
// index is static.
//   factor : lane = row i, r[j] = A(i, k0 + j); pivot from lane k by shuffle,
//            reciprocal square root; column k of L goes to Lrot[k][.] rotated by k
//            (Lrot[k][j] = L(k + j, k), zero past the tile) and comes back to every
//            lane as 16-byte broadcast loads for the rank-1 update;
//   inverse: lane = column c, y[i] = Y(k0 + i, c); y_k = y[t] / L(k, k), then
//            y[t + i] -= Lrot[k][i] y_k.
template <typename T>
__device__ __noinline__ void warp_diag_tile(T *D, T *Iv, T *rdiag, T *Lrot, int LDD, int c0, int nb, int lane,
                                            int col_base, int *fail_col, int *perturbed, const double *dorig,
                                            int *sflag) {
    using V = typename Vec16<T>::type;
    constexpr int E = 16 / int(sizeof(T)), NV = 32 / E;
    const PivotCtl pv{fail_col, perturbed, dorig, nullptr};
    T *Dt = D + c0 * LDD + c0;                       // tile element (i, j) at Dt[j * LDD + i]
    T r[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) r[j] = (j <= lane) ? Dt[j * LDD + lane] : T(0);
    // the re-factor test's threshold of this lane's column, loaded once (a global load
    // per pivot would sit on the pivot chain)
    const double tiny_lane = (sflag && c0 + lane < nb) ? kRefactorTiny * fabs(dorig[col_base + c0 + lane]) : 0.0;
#pragma unroll 1
    for (int k0 = 0; k0 < 32; k0 += 4) {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int k = k0 + t;
            T piv = __shfl_sync(0xffffffffu, r[t], k);
            const double tiny = __shfl_sync(0xffffffffu, tiny_lane, k);
            const int gcol = c0 + k < nb ? col_base + c0 + k : -1;
            const bool bad = sflag ? (gcol >= 0 && !(double(piv) > tiny)) : !(piv > T(0));
            if (bad) piv = panel_bad_pivot(piv, gcol, pv, sflag);
            const T rs = recip_sqrt(piv);
            const T lik = (lane == k) ? piv * rs : r[t] * rs;
            if (lane >= k) Dt[k * LDD + lane] = lik;
            if (lane == k) rdiag[c0 + k] = rs;
            T *lr = Lrot + k * 32;
            lr[(lane - k) & 31] = lane >= k ? lik : T(0);
            __syncwarp();
            T c[32];
#pragma unroll
            for (int v = 0; v < NV; ++v) *reinterpret_cast<V *>(&c[v * E]) = reinterpret_cast<const V *>(lr)[v];
#pragma unroll
            for (int j = 1; j + t < 32; ++j) r[t + j] -= lik * c[j];
        }
#pragma unroll
        for (int j = 0; j < 28; ++j) r[j] = r[j + 4];
    }
    __syncwarp();
    T *It = Iv + c0 * LDD + c0;
    T y[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) y[i] = (i == lane) ? T(1) : T(0);
#pragma unroll 1
    for (int k0 = 0; k0 < 32; k0 += 4) {
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int k = k0 + t;
            const T yk = y[t] * rdiag[c0 + k];
            if (k >= lane) It[lane * LDD + k] = yk;
            const T *lr = Lrot + k * 32;
            T c[32];
#pragma unroll
            for (int v = 0; v < NV; ++v) *reinterpret_cast<V *>(&c[v * E]) = reinterpret_cast<const V *>(lr)[v];
#pragma unroll
            for (int i = 1; i + t < 32; ++i) y[t + i] -= c[i] * yk;
        }
#pragma unroll
        for (int i = 0; i < 28; ++i) y[i] = y[i + 4];
    }
    __syncwarp();
}

// FP64 re-factor of one FP32 diagonal block whose FP32 factorization met a
// non-positive or tiny pivot (pivot <= kRefactorTiny * injected diagonal): the
// block's stored (assembled and updated) values are factored by right-looking
// Cholesky in FP64 and inverted in place (lower-triangular inverse, columns from
// the last), then L, inv(L) (rounded for the tensor-core row solve when asked) and
// the 64 x 64 diagonal inverses are written as the FP32 pass would have. A pivot
// that stays non-positive in FP64 takes the refinement floor and is counted.
// Shared memory: the block as doubles (ld nb + 1) and one column of scratch.
template <typename T>
__device__ __noinline__ void refactor_block_fp64(const PanelTask &tk, T *blk, T *inv_scratch, T *factor,
                                                 const PivotCtl &pv, bool round_inv, unsigned char *smem) {
    const int nb = tk.nb, ld = tk.ld, LD = nb + 1;
    const int tid = threadIdx.x, nt = blockDim.x;
    double *F = reinterpret_cast<double *>(smem);          // (i, j) at F[j * LD + i]
    double *tmp = F + nb * LD;
    __shared__ double pivot;
    for (int q = tid; q < nb * nb; q += nt) {
        const int j = q / nb, i = q - j * nb;
        F[j * LD + i] = i >= j ? double(blk[int64_t(j) * ld + i]) : 0.0;
    }
    __syncthreads();
    for (int k = 0; k < nb; ++k) {
        if (tid == 0) {
            double p = F[k * LD + k];
            if (!(p > 0.0)) {
                const double fl = 1e-3 * fabs(pv.dorig[tk.col + k]);
                p = fabs(p) > fl ? fabs(p) : (fl > 0.0 ? fl : 1.0);
                atomicAdd(pv.perturbed, 1);
            }
            pivot = sqrt(p);
            F[k * LD + k] = pivot;
        }
        __syncthreads();
        const double rp = 1.0 / pivot;
        for (int i = k + 1 + tid; i < nb; i += nt) F[k * LD + i] *= rp;
        __syncthreads();
        const int m = nb - k - 1;
        for (int q = tid; q < m * m; q += nt) {
            const int j = k + 1 + q / m, i = k + 1 + q % m;
            if (i >= j) F[j * LD + i] -= F[k * LD + i] * F[k * LD + j];
        }
        __syncthreads();
    }
    for (int q = tid; q < nb * nb; q += nt) {
        const int j = q / nb, i = q - j * nb;
        if (i >= j) blk[int64_t(j) * ld + i] = T(F[j * LD + i]);
    }
    __syncthreads();
    // inv(L) in place: column j below the diagonal = -(1 / L_jj) inv(L_22) L(j+1:, j)
    for (int j = nb - 1; j >= 0; --j) {
        if (tid == 0) F[j * LD + j] = 1.0 / F[j * LD + j];
        __syncthreads();
        const double ajj = -F[j * LD + j];
        for (int i = j + 1 + tid; i < nb; i += nt) {
            double acc = 0.0;
            for (int k = j + 1; k <= i; ++k) acc += F[k * LD + i] * F[j * LD + k];
            tmp[i] = acc;
        }
        __syncthreads();
        for (int i = j + 1 + tid; i < nb; i += nt) F[j * LD + i] = tmp[i] * ajj;
        __syncthreads();
    }
    for (int q = tid; q < nb * nb; q += nt) {
        const int j = q / nb, i = q - j * nb;
        const T v = i >= j ? T(F[j * LD + i]) : T(0);
        inv_scratch[tk.inv_full + int64_t(j) * tk.ldi + i] = round_inv ? round_operand(v) : v;
    }
    if (tk.inv_out >= 0) {
        const int nb64 = (nb + 63) / 64;
        T *inv = factor + tk.inv_out;
        for (int q = tid; q < nb64 * 4096; q += nt) {
            const int b = q >> 12, e = q & 4095;
            const int j = e >> 6, i = e & 63;
            const int gi = b * 64 + i, gj = b * 64 + j;
            inv[q] = (gi < nb && gj < nb && gi >= gj) ? T(F[gj * LD + gi]) : T(0);
        }
    }
    if (tid == 0) atomicAdd(pv.refactored, 1);
}

template <typename T>
__global__ void __launch_bounds__(kPanelThreads, 1) panel_kernel(const PanelTask *__restrict__ tasks,
                                                                 T *__restrict__ factor, T *__restrict__ inv_scratch,
                                                                 PivotCtl pv, bool round_inv) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const PanelTask tk = tasks[blockIdx.x];
    const int nb = tk.nb, ld = tk.ld;
    const int nblk = (nb + 31) / 32, NBP = nblk * 32;
    const int LDD = NBP + 1;
    T *D = reinterpret_cast<T *>(smem_raw);          // L, column-major, ld LDD (identity-padded)
    T *Iv = D + NBP * LDD;                           // inv(L), column-major, ld LDD
    T *P = Iv + NBP * LDD;                           // 6 x [32][33] partial products
    T *rdiag = P + 6 * 32 * 33;                      // reciprocal diagonal of L
    T *Lrot = rdiag + NBP;                           // [32][32] rotated columns of a diagonal tile (16-byte aligned)
    const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    T *blk = factor + tk.off;
    __shared__ int refactor_flag;
    int *sflag = (std::is_same<T, float>::value && pv.refactored && pv.dorig) ? &refactor_flag : nullptr;
    if (tid == 0) refactor_flag = 0;
    // Load with 16-byte vectors (panel columns, the block's first row and ld are 16-byte
    // aligned), every load of a batch issued before the first shared-memory store.
    {
        using V = typename Vec16<T>::type;
        constexpr int E = 16 / int(sizeof(T));
        const int nvec = NBP / E, tot = NBP * nvec;
        for (int base = 0; base < tot; base += kPanelLoadVecs * nt) {
            V buf[kPanelLoadVecs];
#pragma unroll
            for (int u = 0; u < kPanelLoadVecs; ++u) {
                const int q = base + tid + u * nt;
                const int j = q / nvec, i0 = (q - j * nvec) * E;
                if (q < tot && j < nb && i0 + E <= nb)
                    buf[u] = *reinterpret_cast<const V *>(blk + int64_t(j) * ld + i0);
            }
#pragma unroll
            for (int u = 0; u < kPanelLoadVecs; ++u) {
                const int q = base + tid + u * nt;
                if (q >= tot) continue;
                const int j = q / nvec, i0 = (q - j * nvec) * E;
                const T *bv = reinterpret_cast<const T *>(&buf[u]);
                const bool full = j < nb && i0 + E <= nb;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const int i = i0 + e;
                    T v;
                    if (i < nb && j < nb) v = i >= j ? (full ? bv[e] : blk[int64_t(j) * ld + i]) : T(0);
                    else v = (i == j) ? T(1) : T(0);
                    D[j * LDD + i] = v;
                    Iv[j * LDD + i] = T(0);
                }
            }
        }
    }
    __syncthreads();
    if (warp == 0)
        warp_diag_tile(D, Iv, rdiag, Lrot, LDD, 0, nb, lane, tk.col, pv.fail_col, pv.perturbed, pv.dorig, sflag);
    __syncthreads();
    for (int I = 0; I < nblk; ++I) {
        const int c0 = 32 * I;
        // ---- phase A: tiles below (L_RI) and off-diagonal inverse tiles (inv(L)_IJ)
        {
            const int nbelow = nblk - 1 - I;
            for (int u = warp; u < nbelow + I; u += 8) {
                T c[4][8];
                tile_zero(c);
                if (u < nbelow) {
                    const int R = I + 1 + u;
                    // B(j, k) = inv(L_II)(j, k)
                    tile_mma(c, D + c0 * LDD + 32 * R, LDD, Iv + c0 * LDD + c0, 1, LDD, lane);
                    __syncwarp();
                    tile_store(D + c0 * LDD + 32 * R, LDD, c, T(1), false, lane);
                } else {
                    const int J = u - nbelow;
                    // T_IJ = sum_{K=J}^{I-1} P_IJK, gathered into the K = J slot; B(j, t) = T_IJ(t, j)
                    T *Pj = P + (J * (J + 1) / 2 + J) * 32 * 33;
                    for (int K = J + 1; K < I; ++K) {
                        const T *Pk = P + (K * (K + 1) / 2 + J) * 32 * 33;
                        for (int e = lane; e < 32 * 33; e += 32) Pj[e] += Pk[e];
                    }
                    __syncwarp();
                    tile_mma(c, Iv + c0 * LDD + c0, LDD, Pj, 33, 1, lane);
                    tile_store(Iv + (32 * J) * LDD + c0, LDD, c, T(-1), false, lane);
                }
            }
        }
        __syncthreads();
        if (I + 1 == nblk) break;
        // ---- phase B: trailing updates of tile column I; tile I+1 factored and inverted
        //      as soon as its update is in; products for the next inverse tiles
        {
            const int m = nblk - 1 - I;                          // trailing tile rows / columns
            const int ntrail = m * (m + 1) / 2;                  // u = 0 is tile (I+1, I+1)
            const int nterm = (I + 1) * (I + 2) / 2;             // P_{I+1,J,K}, J <= K <= I
            if (warp == 0) {
                T c[4][8];
                tile_zero(c);
                const int R = I + 1;
                tile_mma(c, D + c0 * LDD + 32 * R, LDD, D + c0 * LDD + 32 * R, 1, LDD, lane);
                tile_store(D + (32 * R) * LDD + 32 * R, LDD, c, T(-1), true, lane);
                __syncwarp();
                warp_diag_tile(D, Iv, rdiag, Lrot, LDD, 32 * R, nb, lane, tk.col, pv.fail_col, pv.perturbed,
                               pv.dorig, sflag);
            } else {
                for (int u = warp; u < ntrail + nterm; u += 7) {
                    T c[4][8];
                    tile_zero(c);
                    if (u < ntrail) {
                        int a = 0;
                        while ((a + 1) * (a + 2) / 2 <= u) ++a;
                        const int R = I + 1 + a, C = I + 1 + (u - a * (a + 1) / 2);   // R >= C
                        // B(j, k) = L_CI(j, k)
                        tile_mma(c, D + c0 * LDD + 32 * R, LDD, D + c0 * LDD + 32 * C, 1, LDD, lane);
                        tile_store(D + (32 * C) * LDD + 32 * R, LDD, c, T(-1), true, lane);
                    } else {
                        const int t = u - ntrail;                 // t = K (K + 1) / 2 + J
                        int K = 0;
                        while ((K + 1) * (K + 2) / 2 <= t) ++K;
                        const int J = t - K * (K + 1) / 2;
                        // B(j, k) = inv(L)_KJ(k, j)
                        tile_mma(c, D + (32 * K) * LDD + 32 * (I + 1), LDD, Iv + (32 * J) * LDD + 32 * K, LDD, 1,
                                 lane);
                        tile_store(P + t * 32 * 33, 33, c, T(1), false, lane);
                    }
                }
            }
        }
        __syncthreads();
    }
    if (sflag) {
        __syncthreads();
        if (refactor_flag) {
            // the block has not been written back: factor its stored values again in FP64
            refactor_block_fp64(tk, blk, inv_scratch, factor, pv, round_inv, smem_raw);
            return;
        }
    }
    // L (lower triangle only: the strict upper part keeps its stored values) and inv(L)
    // (zeros above the diagonal) with 16-byte vector stores where a vector is whole
    {
        using V = typename Vec16<T>::type;
        constexpr int E = 16 / int(sizeof(T));
        const int nvec = (nb + E - 1) / E, tot = nb * nvec;
        for (int q = tid; q < tot; q += nt) {
            const int j = q / nvec, i0 = (q - j * nvec) * E;
            V lv, iv;
            T *l = reinterpret_cast<T *>(&lv), *ivp = reinterpret_cast<T *>(&iv);
#pragma unroll
            for (int e = 0; e < E; ++e) {
                const int i = i0 + e;
                l[e] = D[j * LDD + i];
                const T v = i >= j ? Iv[j * LDD + i] : T(0);
                ivp[e] = round_inv ? round_operand(v) : v;
            }
            T *dl = blk + int64_t(j) * ld + i0;
            T *di = inv_scratch + tk.inv_full + int64_t(j) * tk.ldi + i0;
            if (i0 + E <= nb) {
                *reinterpret_cast<V *>(di) = iv;
                if (i0 >= j) {
                    *reinterpret_cast<V *>(dl) = lv;
                    continue;
                }
            } else {
                for (int e = 0; e < E && i0 + e < nb; ++e) di[e] = ivp[e];
            }
            for (int e = 0; e < E && i0 + e < nb; ++e)
                if (i0 + e >= j) dl[e] = l[e];
        }
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
    const size_t nbp = size_t((nb + 31) / 32) * 32;
    return (2 * nbp * (nbp + 1) + 6 * 32 * 33 + nbp + 32 * 32) * el;
}

template <typename T>
void launch_panel(const PanelTask *tasks, int ntasks, int max_nb, T *factor, T *inv_scratch, PivotCtl pv,
                  bool round_inv, cudaStream_t st) {
    if (ntasks <= 0) return;
    const size_t smem = panel_smem_bytes(max_nb, sizeof(T) == 8);
    // the opt-in limit counts static shared memory too
    static PerDeviceOnce once;
    once([] {
        cudaFuncAttributes fa{};
        cudaFuncGetAttributes(&fa, panel_kernel<T>);
        cudaFuncSetAttribute(panel_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kMaxSmemOptin - int(fa.sharedSizeBytes));
    });
    ++g_kernel_launches;
    panel_kernel<T><<<ntasks, kPanelThreads, smem, st>>>(tasks, factor, inv_scratch, pv, round_inv);
}

template void launch_panel<float>(const PanelTask *, int, int, float *, float *, PivotCtl, bool, cudaStream_t);
template void launch_panel<double>(const PanelTask *, int, int, double *, double *, PivotCtl, bool, cudaStream_t);

}  // namespace mfs
