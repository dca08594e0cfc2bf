// Learned preconditioner (K8): a message-passing network over the block graph
// of H emits a lower block-triangular G on H's pattern; PCG is preconditioned
// by M^{-1} = D^{-1/2} G^T G D^{-1/2} (D = diag(H)). No counterpart in the
// reference; it sits beside the Cholesky path, which stays the fallback.
//
// Graph: the permuted reduced block rows of the symmetric SpMV structure
// (3 x 3 blocks, one node per analysis variable). For row i the entries are
// sorted by column; the diagonal entry ends the lower part, so G's row i is the
// prefix [ptr_i, diag_i] and G^T's row j is the suffix [diag_j, ptr_{j+1}) read
// through `mirror` (entry (j, i) -> entry (i, j)).
//
// Network (weights BF16, every product accumulated in FP32):
//   input   x_i (16)  = [Hs_ii (9, row-major), sum_j a_ij, max_j a_ij, deg_i / 16, 0 x 4]
//                       Hs = D^{-1/2} H D^{-1/2}, a_ij = ||Hs_ij||_F, j != i
//   layer l h' = relu(W_l [h_i; s_i; e_i; 1]) (+ h_i for l > 1), s_i = sum_j a_ij h_j,
//                       e_i = sum_j Hs_ij (9); widths 16 -> 64 -> 64 -> 64 -> 64
//   head    q_i (24)  = V_h [h_i; 1] = [P_i (9) | Q_i (9) | R_i (6)]
//           G_ij (i > j) = P_i + Q_j + V_e [Hs_ij (9); 1]              (9 values, row-major)
//           G_ii       = lower triangle of R_i + V_d [Hs_ii; 1], diagonal through exp()
// With V_h = V_e = V_d = 0, G = I and PCG is Jacobi-preconditioned.
//
// Training loss for pairs (b, x = H^{-1} b), in the scaled variables
// bs = D^{-1/2} b, xs = D^{1/2} x:  L = mean_r e_r^T Hs e_r / (x_r^T b_r),
// e = G^T G bs - xs, i.e. the energy-norm error of M^{-1} b against x.
#include "device.h"
#include "learned.h"

#include <cuda_bf16.h>

#include <algorithm>

namespace mfs {

namespace {

constexpr int kT = 256;

int lgrid(int64_t work, int per_block = kT) {
    int64_t g = (work + per_block - 1) / per_block;
    return int(std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32)));
}

__device__ __forceinline__ int64_t lmin64(int64_t a, int64_t b) { return a < b ? a : b; }

// Block (r, c) of H(i, j) for SpMV entry e (orientation row i, column j).
__device__ __forceinline__ double hblock(const double *Ax, int64_t so, int fl, int r, int c) {
    if (fl & 2) return (r <= c) ? Ax[so + c * 3 + r] : Ax[so + r * 3 + c];
    if (fl & 1) return Ax[so + r * 3 + c];
    return Ax[so + c * 3 + r];
}

// ------------------------------------------------------------------ features
__global__ void dscale_kernel(const LGraph g, const double *__restrict__ Ax, double *__restrict__ dinv) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < g.nv; i += int64_t(gridDim.x) * blockDim.x) {
        const int64_t e = g.diag[i];
        const int64_t so = g.src[e];
        for (int c = 0; c < 3; ++c) {
            const double a = Ax[so + c * 3 + c];
            dinv[i * 3 + c] = a > 0.0 ? 1.0 / sqrt(a) : 1.0;
        }
    }
}

// one thread per node: scaled blocks of its row, aggregate features, input features
__global__ void features_kernel(const LGraph g, const double *__restrict__ Ax, const double *__restrict__ dinv,
                                float *__restrict__ eh, float *__restrict__ ea, float *__restrict__ esum,
                                float *__restrict__ x0) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < g.nv; i += int64_t(gridDim.x) * blockDim.x) {
        float es[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        float asum = 0.f, amax = 0.f;
        const double di[3] = {dinv[i * 3], dinv[i * 3 + 1], dinv[i * 3 + 2]};
        for (int64_t e = g.ptr[i]; e < g.ptr[i + 1]; ++e) {
            const int64_t j = g.col[e];
            const int64_t so = g.src[e];
            const int fl = g.flag[e];
            float n2 = 0.f;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) {
                    const float v = float(hblock(Ax, so, fl, r, c) * di[r] * dinv[j * 3 + c]);
                    eh[e * 9 + r * 3 + c] = v;
                    if (j != i) {
                        es[r * 3 + c] += v;
                        n2 += v * v;
                    }
                }
            const float a = j != i ? sqrtf(n2) : 0.f;
            ea[e] = a;
            asum += a;
            amax = fmaxf(amax, a);
        }
        const int64_t ed = g.diag[i];
        for (int k = 0; k < 9; ++k) {
            esum[i * 9 + k] = es[k];
            x0[i * kLIn + k] = eh[ed * 9 + k];
        }
        x0[i * kLIn + 9] = asum;
        x0[i * kLIn + 10] = amax;
        x0[i * kLIn + 11] = float(g.ptr[i + 1] - g.ptr[i]) * (1.f / 16.f);
        for (int k = 12; k < kLIn; ++k) x0[i * kLIn + k] = 0.f;
    }
}

// ------------------------------------------------------------------ dense node layers
// u_i = [h_i (din); s_i (din, if agg); e_i (9, if use_e); 1]; out = act(W u) (+ h_i).
// A CTA owns kNodeTile nodes: their u vectors and W^T (as float) sit in shared memory.
constexpr int kNodeTile = 32;

struct DenseArgs {
    const __nv_bfloat16 *W;   // dout x dtot, row-major
    const float *h;           // N x din
    const float *esum;        // N x 9
    float *s;                 // N x din (written by forward when agg, read by backward)
    float *pre;               // N x dout pre-activation (forward output when relu)
    float *out;               // N x dout
    int din, dout, agg, use_e, relu, resid;
};

__device__ __forceinline__ int dtot_of(int din, int agg, int use_e) { return din * (agg ? 2 : 1) + (use_e ? 9 : 0) + 1; }

// Fill u for the tile's nodes (aggregating neighbours when asked). One warp per node.
__device__ void load_u(const LGraph &g, const DenseArgs &a, int64_t n0, int nn, float *u, int dtot, bool write_s,
                       const float *s_in) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int t = warp; t < nn; t += nw) {
        const int64_t i = n0 + t;
        float *ui = u + t * dtot;
        for (int k = lane; k < a.din; k += 32) ui[k] = a.h[i * a.din + k];
        int o = a.din;
        if (a.agg) {
            if (s_in) {
                for (int k = lane; k < a.din; k += 32) ui[o + k] = s_in[i * a.din + k];
            } else {
                float acc0 = 0.f, acc1 = 0.f;
                for (int64_t e = g.ptr[i]; e < g.ptr[i + 1]; ++e) {
                    const int64_t j = g.col[e];
                    if (j == i) continue;
                    const float w = g.ea[e];
                    if (lane < a.din) acc0 += w * a.h[j * a.din + lane];
                    if (lane + 32 < a.din) acc1 += w * a.h[j * a.din + lane + 32];
                }
                if (lane < a.din) ui[o + lane] = acc0;
                if (lane + 32 < a.din) ui[o + lane + 32] = acc1;
                if (write_s) {
                    if (lane < a.din) a.s[i * a.din + lane] = acc0;
                    if (lane + 32 < a.din) a.s[i * a.din + lane + 32] = acc1;
                }
            }
            o += a.din;
        }
        if (a.use_e) {
            if (lane < 9) ui[o + lane] = a.esum[i * 9 + lane];
            o += 9;
        }
        if (lane == 0) ui[o] = 1.f;
    }
}

__global__ void __launch_bounds__(kT) dense_fwd_kernel(const LGraph g, DenseArgs a) {
    extern __shared__ float lsm[];
    const int dtot = dtot_of(a.din, a.agg, a.use_e);
    float *wt = lsm;                        // dtot x dout (W^T)
    float *u = wt + dtot * a.dout;          // kNodeTile x dtot
    for (int q = threadIdx.x; q < dtot * a.dout; q += blockDim.x) {
        const int k = q / dtot, m = q - k * dtot;
        wt[m * a.dout + k] = __bfloat162float(a.W[q]);
    }
    for (int64_t n0 = int64_t(blockIdx.x) * kNodeTile; n0 < g.nv; n0 += int64_t(gridDim.x) * kNodeTile) {
        const int nn = int(lmin64(kNodeTile, g.nv - n0));
        __syncthreads();
        load_u(g, a, n0, nn, u, dtot, true, nullptr);
        __syncthreads();
        for (int q = threadIdx.x; q < nn * a.dout; q += blockDim.x) {
            const int t = q / a.dout, k = q - t * a.dout;
            const float *ut = u + t * dtot;
            float acc = 0.f;
            for (int m = 0; m < dtot; ++m) acc += wt[m * a.dout + k] * ut[m];
            const int64_t i = n0 + t;
            float v = acc;
            if (a.relu) {
                a.pre[i * a.dout + k] = acc;
                v = fmaxf(acc, 0.f);
            }
            if (a.resid) v += ut[k];
            a.out[i * a.dout + k] = v;
        }
    }
}

// Backward of one dense layer: dpre = dout (.) [pre > 0]; per-CTA partials of
// dW = sum_i dpre_i u_i^T (fixed order, reduced later); dh_i = (W^T dpre_i)[0:din]
// (+ dout_i for a residual layer); ds_i = (W^T dpre_i)[din:2 din].
__global__ void __launch_bounds__(kT) dense_bwd_kernel(const LGraph g, DenseArgs a, const float *__restrict__ dout,
                                                        float *__restrict__ dh, float *__restrict__ ds,
                                                        float *__restrict__ wpart) {
    extern __shared__ float lsm[];
    const int dtot = dtot_of(a.din, a.agg, a.use_e);
    float *w = lsm;                         // dout x dtot (row-major)
    float *u = w + dtot * a.dout;           // kNodeTile x dtot
    float *dp = u + kNodeTile * dtot;       // kNodeTile x dout
    for (int q = threadIdx.x; q < dtot * a.dout; q += blockDim.x) w[q] = __bfloat162float(a.W[q]);
    // dW partial accumulators: each thread owns params q = tid + k * blockDim
    constexpr int kMaxOwn = 36;             // 64 x 138 / 256 rounded up
    float accw[kMaxOwn];
#pragma unroll
    for (int k = 0; k < kMaxOwn; ++k) accw[k] = 0.f;
    const int np = dtot * a.dout;
    for (int64_t n0 = int64_t(blockIdx.x) * kNodeTile; n0 < g.nv; n0 += int64_t(gridDim.x) * kNodeTile) {
        const int nn = int(lmin64(kNodeTile, g.nv - n0));
        __syncthreads();
        load_u(g, a, n0, nn, u, dtot, false, a.s);
        for (int q = threadIdx.x; q < kNodeTile * a.dout; q += blockDim.x) {
            const int t = q / a.dout, k = q - t * a.dout;
            float v = 0.f;
            if (t < nn) {
                const int64_t i = n0 + t;
                v = dout[i * a.dout + k];
                if (a.relu && a.pre[i * a.dout + k] <= 0.f) v = 0.f;
            }
            dp[q] = v;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kMaxOwn; ++k) {
            const int q = threadIdx.x + k * kT;
            if (q < np) {
                const int kk = q / dtot, m = q - kk * dtot;
                float acc = 0.f;
                for (int t = 0; t < nn; ++t) acc += dp[t * a.dout + kk] * u[t * dtot + m];
                accw[k] += acc;
            }
        }
        // du = W^T dpre for the h and s parts
        const int nin = a.din * (a.agg ? 2 : 1);
        for (int q = threadIdx.x; q < nn * nin; q += blockDim.x) {
            const int t = q / nin, m = q - t * nin;
            float acc = 0.f;
            for (int kk = 0; kk < a.dout; ++kk) acc += w[kk * dtot + m] * dp[t * a.dout + kk];
            const int64_t i = n0 + t;
            if (m < a.din) {
                if (a.resid) acc += dout[i * a.dout + m];
                dh[i * a.din + m] = acc;
            } else {
                ds[i * a.din + (m - a.din)] = acc;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < kMaxOwn; ++k) {
        const int q = threadIdx.x + k * kT;
        if (q < np) wpart[int64_t(blockIdx.x) * np + q] = accw[k];
    }
}

// dh_j += sum_{i in N(j)} a_ij ds_i (the aggregation's transpose; a is symmetric)
__global__ void agg_bwd_kernel(const LGraph g, const float *__restrict__ ds, float *__restrict__ dh, int din) {
    const int lane = threadIdx.x & 31;
    const int64_t w0 = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
    const int64_t nwarp = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t j = w0; j < g.nv; j += nwarp) {
        float acc0 = 0.f, acc1 = 0.f;
        for (int64_t e = g.ptr[j]; e < g.ptr[j + 1]; ++e) {
            const int64_t i = g.col[e];
            if (i == j) continue;
            const float w = g.ea[e];
            if (lane < din) acc0 += w * ds[i * din + lane];
            if (lane + 32 < din) acc1 += w * ds[i * din + lane + 32];
        }
        if (lane < din) dh[j * din + lane] += acc0;
        if (lane + 32 < din) dh[j * din + lane + 32] += acc1;
    }
}

// Fixed-order sum of per-CTA partials: grad[q] = sum_b part[b * np + q].
__global__ void reduce_parts_kernel(const float *__restrict__ part, int nparts, int np, float *__restrict__ grad) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < np; q += gridDim.x * blockDim.x) {
        float acc = 0.f;
        for (int b = 0; b < nparts; ++b) acc += part[int64_t(b) * np + q];
        grad[q] = acc;
    }
}

// ------------------------------------------------------------------ head: G from q and the scaled blocks
__device__ __forceinline__ float clampo(float x) { return fminf(fmaxf(x, -8.f), 8.f); }

__global__ void build_g_kernel(const LGraph g, const float *__restrict__ q, const float *__restrict__ eh,
                               const __nv_bfloat16 *__restrict__ Ve, const __nv_bfloat16 *__restrict__ Vd,
                               float *__restrict__ G) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < g.nv; i += int64_t(gridDim.x) * blockDim.x) {
        const float *qi = q + i * kLHead;
        for (int64_t e = g.ptr[i]; e < g.diag[i]; ++e) {
            const int64_t j = g.col[e];
            const float *qj = q + j * kLHead;
            const float *he = eh + e * 9;
            for (int k = 0; k < 9; ++k) {
                float o = qi[k] + qj[9 + k] + __bfloat162float(Ve[k * 10 + 9]);
                for (int m = 0; m < 9; ++m) o += __bfloat162float(Ve[k * 10 + m]) * he[m];
                G[e * 9 + k] = o;
            }
        }
        const int64_t e = g.diag[i];
        const float *he = eh + e * 9;
        float o[6];
        for (int k = 0; k < 6; ++k) {
            float v = qi[18 + k] + __bfloat162float(Vd[k * 10 + 9]);
            for (int m = 0; m < 9; ++m) v += __bfloat162float(Vd[k * 10 + m]) * he[m];
            o[k] = v;
        }
        // lower triangle, row-major: (0,0)=exp o0; (1,0)=o1, (1,1)=exp o2; (2,0)=o3, (2,1)=o4, (2,2)=exp o5
        float *Gd = G + e * 9;
        Gd[0] = expf(clampo(o[0]));
        Gd[1] = 0.f;
        Gd[2] = 0.f;
        Gd[3] = o[1];
        Gd[4] = expf(clampo(o[2]));
        Gd[5] = 0.f;
        Gd[6] = o[3];
        Gd[7] = o[4];
        Gd[8] = expf(clampo(o[5]));
    }
}

// ------------------------------------------------------------------ G products (FP64 vectors)
// Y = G X (trans = 0) or Y = G^T X (trans = 1); X, Y are n x nrhs (ld n), n = 3 nv.
// One thread per (node, rhs); scale (optional) multiplies X on the way in (pre)
// or Y on the way out (post).
__global__ void gmv_kernel(const LGraph g, const float *__restrict__ G, int trans, const double *__restrict__ X,
                           double *__restrict__ Y, int64_t ld, int nrhs, const double *__restrict__ pre,
                           const double *__restrict__ post) {
    const int64_t total = g.nv * nrhs;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t r = t / g.nv, i = t - r * g.nv;
        const double *x = X + r * ld;
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        const int64_t e0 = trans ? g.diag[i] : g.ptr[i];
        const int64_t e1 = trans ? g.ptr[i + 1] : g.diag[i] + 1;
        for (int64_t e = e0; e < e1; ++e) {
            const int64_t j = g.col[e];
            const float *b = G + (trans ? g.mirror[e] : e) * 9;
            double x0 = x[j * 3], x1 = x[j * 3 + 1], x2 = x[j * 3 + 2];
            if (pre) {
                x0 *= pre[j * 3];
                x1 *= pre[j * 3 + 1];
                x2 *= pre[j * 3 + 2];
            }
            if (!trans) {
                a0 += double(b[0]) * x0 + double(b[1]) * x1 + double(b[2]) * x2;
                a1 += double(b[3]) * x0 + double(b[4]) * x1 + double(b[5]) * x2;
                a2 += double(b[6]) * x0 + double(b[7]) * x1 + double(b[8]) * x2;
            } else {
                a0 += double(b[0]) * x0 + double(b[3]) * x1 + double(b[6]) * x2;
                a1 += double(b[1]) * x0 + double(b[4]) * x1 + double(b[7]) * x2;
                a2 += double(b[2]) * x0 + double(b[5]) * x1 + double(b[8]) * x2;
            }
        }
        if (post) {
            a0 *= post[i * 3];
            a1 *= post[i * 3 + 1];
            a2 *= post[i * 3 + 2];
        }
        double *y = Y + r * ld;
        y[i * 3] = a0;
        y[i * 3 + 1] = a1;
        y[i * 3 + 2] = a2;
    }
}

// elementwise: out = a * s (s per row, optional power)
__global__ void scale_rows_kernel(const double *__restrict__ in, const double *__restrict__ s, int inv,
                                  double *__restrict__ out, int64_t n, int nrhs, int64_t ld) {
    const int64_t total = n * nrhs;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total; t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t r = t / n, i = t - r * n;
        out[i + r * ld] = inv ? in[i + r * ld] / s[i] : in[i + r * ld] * s[i];
    }
}

// dG_e = sum_r z_i gy_j^T + gz_i bs_j^T for the lower entries (i >= j) of G.
__global__ void dg_kernel(const LGraph g, const double *__restrict__ Z, const double *__restrict__ GY,
                          const double *__restrict__ GZ, const double *__restrict__ BS, int64_t ld, int nrhs,
                          float *__restrict__ dG) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < g.nv; i += int64_t(gridDim.x) * blockDim.x) {
        for (int64_t e = g.ptr[i]; e <= g.diag[i]; ++e) {
            const int64_t j = g.col[e];
            double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            for (int r = 0; r < nrhs; ++r) {
                const int64_t o = r * ld;
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b)
                        acc[a * 3 + b] += Z[o + i * 3 + a] * GY[o + j * 3 + b] + GZ[o + i * 3 + a] * BS[o + j * 3 + b];
            }
            for (int k = 0; k < 9; ++k) dG[e * 9 + k] = float(acc[k]);
        }
    }
}

// Head backward, per node i: dq_i = [sum_{e in row i, lower} dG_e | sum_{e' in row i,
// upper} dG_{mirror e'} | d(diagonal head outputs)]; the latter also go to dod
// (6 per node) for the diagonal head's weight gradient.
__global__ void head_bwd_kernel(const LGraph g, const float *__restrict__ dG, const float *__restrict__ G,
                                float *__restrict__ dq, float *__restrict__ dod) {
    for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < g.nv; i += int64_t(gridDim.x) * blockDim.x) {
        float p[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, qq[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int64_t e = g.ptr[i]; e < g.diag[i]; ++e) {
            const float *d = dG + e * 9;
#pragma unroll
            for (int k = 0; k < 9; ++k) p[k] += d[k];
        }
        for (int64_t e = g.diag[i] + 1; e < g.ptr[i + 1]; ++e) {
            const float *d = dG + g.mirror[e] * 9;
#pragma unroll
            for (int k = 0; k < 9; ++k) qq[k] += d[k];
        }
        const int64_t ed = g.diag[i];
        const float *d = dG + ed * 9;
        const float *Gd = G + ed * 9;
        // o0 -> (0,0) exp, o1 -> (1,0), o2 -> (1,1) exp, o3 -> (2,0), o4 -> (2,1), o5 -> (2,2) exp;
        // the clamp to [-8, 8] blocks the gradient outside it
        const float lo = 3.3546e-4f, hi = 2980.95f;   // exp(-8), exp(8)
        float dout[6];
        dout[0] = (Gd[0] > lo && Gd[0] < hi) ? d[0] * Gd[0] : 0.f;
        dout[1] = d[3];
        dout[2] = (Gd[4] > lo && Gd[4] < hi) ? d[4] * Gd[4] : 0.f;
        dout[3] = d[6];
        dout[4] = d[7];
        dout[5] = (Gd[8] > lo && Gd[8] < hi) ? d[8] * Gd[8] : 0.f;
        float *dqi = dq + i * kLHead;
        for (int k = 0; k < 9; ++k) {
            dqi[k] = p[k];
            dqi[9 + k] = qq[k];
        }
        for (int k = 0; k < 6; ++k) {
            dqi[18 + k] = dout[k];
            dod[i * 6 + k] = dout[k];
        }
    }
}

// Per-CTA partials of the edge-head weights over a contiguous node range:
// thread t < 90: dVe[k][m] = sum over strictly lower entries of dG_e[k] [Hs_e; 1][m];
// thread 90 <= t < 150: dVd[k][m] = sum over nodes of dod_i[k] [Hs_ii; 1][m].
__global__ void head_param_kernel(const LGraph g, const float *__restrict__ dG, const float *__restrict__ dod,
                                  const float *__restrict__ eh, float *__restrict__ vpart) {
    const int64_t chunk = (g.nv + gridDim.x - 1) / gridDim.x;
    const int64_t n0 = blockIdx.x * chunk, n1 = lmin64(g.nv, n0 + chunk);
    const int t = threadIdx.x;
    if (t >= 150) return;
    float acc = 0.f;
    if (t < 90) {
        const int k = t / 10, m = t % 10;
        for (int64_t i = n0; i < n1; ++i)
            for (int64_t e = g.ptr[i]; e < g.diag[i]; ++e) acc += dG[e * 9 + k] * (m < 9 ? eh[e * 9 + m] : 1.f);
    } else {
        const int k = (t - 90) / 10, m = (t - 90) % 10;
        for (int64_t i = n0; i < n1; ++i) acc += dod[i * 6 + k] * (m < 9 ? eh[g.diag[i] * 9 + m] : 1.f);
    }
    vpart[int64_t(blockIdx.x) * 150 + t] = acc;
}

// Adam on the FP32 master copy; the BF16 copy is what the kernels read.
__global__ void adam_kernel(float *__restrict__ w, __nv_bfloat16 *__restrict__ wb, float *__restrict__ m,
                            float *__restrict__ v, const float *__restrict__ grad, int n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gr = grad[i];
        const float mi = b1 * m[i] + (1.f - b1) * gr;
        const float vi = b2 * v[i] + (1.f - b2) * gr * gr;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        wb[i] = __float2bfloat16_rn(wi);
    }
}

__global__ void to_bf16_kernel(const float *__restrict__ w, __nv_bfloat16 *__restrict__ wb, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        wb[i] = __float2bfloat16_rn(w[i]);
}

size_t dense_smem(int din, int dout, int agg, int use_e, bool bwd) {
    const int dtot = din * (agg ? 2 : 1) + (use_e ? 9 : 0) + 1;
    size_t f = size_t(dtot) * dout + size_t(kNodeTile) * dtot;
    if (bwd) f += size_t(kNodeTile) * dout;
    return f * sizeof(float);
}

}  // namespace

int lpc_layer_in(int l) { return l == 0 ? kLIn : kLHid; }

// Parameter offsets inside the flat weight array.
LParamLayout lpc_layout() {
    LParamLayout L{};
    int o = 0;
    for (int l = 0; l < kLLayers; ++l) {
        L.w[l] = o;
        o += kLHid * (2 * lpc_layer_in(l) + 10);
    }
    L.vh = o;
    o += kLHead * (kLHid + 1);
    L.ve = o;
    o += 90;
    L.vd = o;
    o += 60;
    L.total = o;
    return L;
}

int lpc_dense_parts() { return 148 * 4; }
int lpc_head_parts() { return 148 * 4; }

void lpc_features(const LGraph &g, const double *Ax, LWork &w, cudaStream_t st) {
    g_kernel_launches += 2;
    dscale_kernel<<<lgrid(g.nv), kT, 0, st>>>(g, Ax, w.dinv);
    features_kernel<<<lgrid(g.nv), kT, 0, st>>>(g, Ax, w.dinv, w.eh, g.ea, w.esum, w.h[0]);
}

void lpc_forward(const LGraph &g, const __nv_bfloat16 *wb, LWork &w, cudaStream_t st) {
    static PerDeviceOnce once;
    once([] {
        cudaFuncSetAttribute(dense_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmemOptin);
        cudaFuncSetAttribute(dense_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxSmemOptin);
    });
    const LParamLayout L = lpc_layout();
    const int grid = lpc_dense_parts();
    for (int l = 0; l < kLLayers; ++l) {
        DenseArgs a{wb + L.w[l], w.h[l], w.esum, w.s[l], w.pre[l], w.h[l + 1], lpc_layer_in(l), kLHid, 1, 1, 1, l > 0};
        ++g_kernel_launches;
        dense_fwd_kernel<<<grid, kT, dense_smem(a.din, a.dout, 1, 1, false), st>>>(g, a);
    }
    DenseArgs a{wb + L.vh, w.h[kLLayers], w.esum, nullptr, nullptr, w.q, kLHid, kLHead, 0, 0, 0, 0};
    ++g_kernel_launches;
    dense_fwd_kernel<<<grid, kT, dense_smem(kLHid, kLHead, 0, 0, false), st>>>(g, a);
    ++g_kernel_launches;
    build_g_kernel<<<lgrid(g.nv), kT, 0, st>>>(g, w.q, w.eh, wb + L.ve, wb + L.vd, w.G);
}

void lpc_gmv(const LGraph &g, const float *G, bool trans, const double *X, double *Y, int64_t ld, int nrhs,
             const double *pre, const double *post, cudaStream_t st) {
    ++g_kernel_launches;
    gmv_kernel<<<lgrid(g.nv * nrhs), kT, 0, st>>>(g, G, trans ? 1 : 0, X, Y, ld, nrhs, pre, post);
}

void lpc_scale_rows(const double *in, const double *s, bool inv, double *out, int64_t n, int nrhs, int64_t ld,
                    cudaStream_t st) {
    ++g_kernel_launches;
    scale_rows_kernel<<<lgrid(n * nrhs), kT, 0, st>>>(in, s, inv ? 1 : 0, out, n, nrhs, ld);
}

void lpc_dg(const LGraph &g, const double *Z, const double *GY, const double *GZ, const double *BS, int64_t ld,
            int nrhs, float *dG, cudaStream_t st) {
    ++g_kernel_launches;
    dg_kernel<<<lgrid(g.nv), kT, 0, st>>>(g, Z, GY, GZ, BS, ld, nrhs, dG);
}

void lpc_backward(const LGraph &g, const __nv_bfloat16 *wb, LWork &w, float *grad, cudaStream_t st) {
    const LParamLayout L = lpc_layout();
    const int grid = lpc_dense_parts();
    // head
    ++g_kernel_launches;
    head_bwd_kernel<<<lgrid(g.nv), kT, 0, st>>>(g, w.dG, w.G, w.dq, w.dod);
    ++g_kernel_launches;
    head_param_kernel<<<lpc_head_parts(), 160, 0, st>>>(g, w.dG, w.dod, w.eh, w.part);
    ++g_kernel_launches;
    reduce_parts_kernel<<<1, kT, 0, st>>>(w.part, lpc_head_parts(), 150, grad + L.ve);
    {
        DenseArgs a{wb + L.vh, w.h[kLLayers], w.esum, nullptr, nullptr, w.q, kLHid, kLHead, 0, 0, 0, 0};
        ++g_kernel_launches;
        dense_bwd_kernel<<<grid, kT, dense_smem(kLHid, kLHead, 0, 0, true), st>>>(g, a, w.dq, w.dh[1], nullptr,
                                                                                     w.part);
        const int np = kLHead * (kLHid + 1);
        ++g_kernel_launches;
        reduce_parts_kernel<<<lgrid(np), kT, 0, st>>>(w.part, grid, np, grad + L.vh);
    }
    int cur = 1;
    for (int l = kLLayers - 1; l >= 0; --l) {
        DenseArgs a{wb + L.w[l], w.h[l], w.esum, w.s[l], w.pre[l], w.h[l + 1], lpc_layer_in(l), kLHid, 1, 1, 1, l > 0};
        float *dh_out = w.dh[cur ^ 1];
        ++g_kernel_launches;
        dense_bwd_kernel<<<grid, kT, dense_smem(a.din, a.dout, 1, 1, true), st>>>(g, a, w.dh[cur], dh_out, w.ds,
                                                                                   w.part);
        const int np = kLHid * (2 * a.din + 10);
        ++g_kernel_launches;
        reduce_parts_kernel<<<lgrid(np), kT, 0, st>>>(w.part, grid, np, grad + L.w[l]);
        if (l > 0) {
            ++g_kernel_launches;
            agg_bwd_kernel<<<lgrid(g.nv * 32), kT, 0, st>>>(g, w.ds, dh_out, a.din);
        }
        cur ^= 1;
    }
}

void lpc_adam(float *w, __nv_bfloat16 *wb, float *m, float *v, const float *grad, int n, float lr, int step,
              cudaStream_t st) {
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, float(step)), c2 = 1.f - powf(b2, float(step));
    ++g_kernel_launches;
    adam_kernel<<<lgrid(n), kT, 0, st>>>(w, wb, m, v, grad, n, lr, b1, b2, 1e-8f, c1, c2);
}

void lpc_to_bf16(const float *w, __nv_bfloat16 *wb, int n, cudaStream_t st) {
    ++g_kernel_launches;
    to_bf16_kernel<<<lgrid(n), kT, 0, st>>>(w, wb, n);
}

}  // namespace mfs
