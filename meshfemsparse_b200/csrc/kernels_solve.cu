// Symmetric block SpMV (K7), the fused
// pin-removal/permutation gathers, element assembly (K1) and the FP64
// vector kernels of the refinement loop.
//
// Reference counterparts:
//   SparseLDL::Solve (forward L y = b, backward L^T x = y, multi-RHS column-major,
//   ld = n) ............................ Solvers/CatamariFactorizer.cc:54,70,838-907
//   removeFixedEntries / extractFullSolution with the permutation fused
//   ..................................... Solvers/CholeskyFactorizerBase.hh:299-363
//   BlockCSCHessianBase::applyRawColumnRangeAccum (upper blocks + transposes)
//   ..................................... BlockCSCHessian.hh:1080-1120
//   ElementHessianContribAssembler<true>::run + ColumnScanner::addBlockAtLoc
//   ..................................... SystemAssembler.hh:60-98, BlockCSCHessian.hh:371-381
// The triangular solves themselves live in kernels_trisolve.cu.
#include "device.h"

namespace mfs {

namespace {

constexpr int kReduceBlocks = 296;   // 2 x SM count; fixed so reductions are deterministic


__global__ void spmv_kernel(const int64_t *__restrict__ ptr, const int64_t *__restrict__ src,
                            const int32_t *__restrict__ col, const int32_t *__restrict__ flag, int64_t nrows, int vb,
                            int ld, const double *__restrict__ Ax, const double *__restrict__ X,
                            double *__restrict__ Y, int64_t ldx, int nrhs) {
    const int64_t total = nrows * vb * nrhs;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t rr = t / (nrows * vb);
        const int64_t q = t - rr * nrows * vb;
        const int64_t i = q / vb;
        const int r = int(q - i * vb);
        double acc = 0.0;
        for (int64_t e = ptr[i]; e < ptr[i + 1]; ++e) {
            const int64_t so = src[e];
            const int64_t xb = int64_t(col[e]) * vb + rr * ldx;
            const int fl = flag[e];
            for (int c = 0; c < vb; ++c) {
                double a;
                if (fl & 2) a = (r <= c) ? Ax[so + int64_t(c) * ld + r] : Ax[so + int64_t(r) * ld + c];
                else if (fl & 1) a = Ax[so + int64_t(r) * ld + c];
                else a = Ax[so + int64_t(c) * ld + r];
                acc += a * X[xb + c];
            }
        }
        Y[i * vb + r + rr * ldx] = acc;
    }
}

__global__ void gather_rows_kernel(const int64_t *__restrict__ map, int64_t n_in, const double *__restrict__ in,
                                   int64_t ld_in, double *__restrict__ out, int64_t ld_out, int nrhs) {
    const int64_t total = n_in * nrhs;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t r = t / n_in, i = t - r * n_in;
        const int64_t q = map ? map[i] : i;
        if (q >= 0) out[q + r * ld_out] = in[i + r * ld_in];
    }
}

__global__ void scatter_rows_kernel(const int64_t *__restrict__ map, int64_t n_out, const double *__restrict__ in,
                                    int64_t ld_in, double *__restrict__ out, int64_t ld_out, int nrhs) {
    const int64_t total = n_out * nrhs;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t r = t / n_out, i = t - r * n_out;
        const int64_t q = map ? map[i] : i;
        out[i + r * ld_out] = q >= 0 ? in[q + r * ld_in] : 0.0;
    }
}

// K1: one thread per (slot, component); contributions are summed in element order.
// contrib = (offset into Ke of the 3x3 block's upper-left) << 2 | kind,
// kind 0: O(r,c) = Ke[o + 12 r + c]; 1: O(r,c) = Ke[o + 12 c + r]; 2: diagonal, r <= c only.
__global__ void assemble_elements_kernel(const int64_t *__restrict__ slot_ptr, const int64_t *__restrict__ contrib,
                                         int64_t nslots, const double *__restrict__ Ke, double *__restrict__ Ax) {
    const int64_t total = nslots * 9;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int64_t slot = t / 9;
        const int comp = int(t - slot * 9);
        const int c = comp / 3, r = comp - 3 * c;
        double acc = 0.0;
        for (int64_t k = slot_ptr[slot]; k < slot_ptr[slot + 1]; ++k) {
            const int64_t code = contrib[k];
            const int kind = int(code & 3);
            const int64_t o = code >> 2;
            if (kind == 1) acc += Ke[o + 12 * c + r];
            else if (kind == 0 || r <= c) acc += Ke[o + 12 * r + c];
        }
        Ax[t] = acc;
    }
}

__global__ void residual_kernel(const double *__restrict__ B, const double *__restrict__ AX, double *__restrict__ R,
                                int64_t total) {
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x)
        R[t] = B[t] - AX[t];
}

// Deterministic column dot products: fixed grid, per-block partial sums, ordered final sum.
__global__ void __launch_bounds__(256) coldot_partial_kernel(const double *__restrict__ X,
                                                             const double *__restrict__ Y, int64_t n, int nrhs,
                                                             double *__restrict__ partials) {
    __shared__ double red[256];
    for (int r = 0; r < nrhs; ++r) {
        double acc = 0.0;
        for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
            acc += X[i + r * n] * Y[i + r * n];
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int h = 128; h > 0; h >>= 1) {
            if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
            __syncthreads();
        }
        if (threadIdx.x == 0) partials[r * gridDim.x + blockIdx.x] = red[0];
        __syncthreads();
    }
}

__global__ void coldot_final_kernel(const double *__restrict__ partials, int nparts, int nrhs,
                                    double *__restrict__ out) {
    const int r = threadIdx.x;
    if (r >= nrhs) return;
    double acc = 0.0;
    for (int k = 0; k < nparts; ++k) acc += partials[r * nparts + k];
    out[r] = acc;
}

// x += alpha p, r -= alpha Ap with alpha = rz / pAp per column (columns with active == 0 untouched)
__global__ void pcg_xr_kernel(double *__restrict__ X, double *__restrict__ R, const double *__restrict__ P,
                              const double *__restrict__ AP, const double *__restrict__ rz,
                              const double *__restrict__ pap, const int *__restrict__ active, int64_t n, int nrhs) {
    const int64_t total = n * nrhs;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int r = int(t / n);
        if (!active[r]) continue;
        const double alpha = pap[r] != 0.0 ? rz[r] / pap[r] : 0.0;
        X[t] += alpha * P[t];
        R[t] -= alpha * AP[t];
    }
}

__global__ void pcg_p_kernel(double *__restrict__ P, const double *__restrict__ Z, const double *__restrict__ rz_new,
                             const double *__restrict__ rz_old, const int *__restrict__ active, int64_t n, int nrhs) {
    const int64_t total = n * nrhs;
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < total;
         t += int64_t(gridDim.x) * blockDim.x) {
        const int r = int(t / n);
        if (!active[r]) continue;
        const double beta = rz_old[r] != 0.0 ? rz_new[r] / rz_old[r] : 0.0;
        P[t] = Z[t] + beta * P[t];
    }
}

__global__ void copy_kernel(double *__restrict__ dst, const double *__restrict__ src, int64_t count) {
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < count;
         t += int64_t(gridDim.x) * blockDim.x)
        dst[t] = src[t];
}

__global__ void axpy_kernel(double *__restrict__ y, const double *__restrict__ x, double alpha, int64_t count) {
    for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < count;
         t += int64_t(gridDim.x) * blockDim.x)
        y[t] += alpha * x[t];
}

inline int grid_for(int64_t n, int threads) {
    int64_t g = (n + threads - 1) / threads;
    if (g > 148 * 32) g = 148 * 32;
    if (g < 1) g = 1;
    return int(g);
}

}  // namespace

int reduce_partials_count() { return kReduceBlocks; }

void launch_spmv(const int64_t *ptr, const int64_t *src, const int32_t *col, const int32_t *flag, int64_t nrows,
                 int vb, int src_ld, const double *Ax, const double *X, double *Y, int64_t ld, int nrhs,
                 cudaStream_t st) {
    if (nrows <= 0) return;
    ++g_kernel_launches;
    spmv_kernel<<<grid_for(nrows * vb * nrhs, 256), 256, 0, st>>>(ptr, src, col, flag, nrows, vb, src_ld, Ax, X, Y,
                                                                   ld, nrhs);
}

void launch_gather_rows(const int64_t *map, int64_t n_in, const double *in, int64_t ld_in, double *out,
                        int64_t ld_out, int nrhs, cudaStream_t st) {
    if (n_in <= 0) return;
    ++g_kernel_launches;
    gather_rows_kernel<<<grid_for(n_in * nrhs, 256), 256, 0, st>>>(map, n_in, in, ld_in, out, ld_out, nrhs);
}

void launch_scatter_rows(const int64_t *map, int64_t n_out, const double *in, int64_t ld_in, double *out,
                         int64_t ld_out, int nrhs, cudaStream_t st) {
    if (n_out <= 0) return;
    ++g_kernel_launches;
    scatter_rows_kernel<<<grid_for(n_out * nrhs, 256), 256, 0, st>>>(map, n_out, in, ld_in, out, ld_out, nrhs);
}

void launch_assemble_elements(const int64_t *slot_ptr, const int64_t *contrib, int64_t nslots, const double *Ke,
                              double *Ax, cudaStream_t st) {
    if (nslots <= 0) return;
    ++g_kernel_launches;
    assemble_elements_kernel<<<grid_for(nslots * 9, 256), 256, 0, st>>>(slot_ptr, contrib, nslots, Ke, Ax);
}

void launch_residual(const double *B, const double *AX, double *R, int64_t n, int nrhs, cudaStream_t st) {
    if (n * nrhs <= 0) return;
    ++g_kernel_launches;
    residual_kernel<<<grid_for(n * nrhs, 256), 256, 0, st>>>(B, AX, R, n * nrhs);
}

void launch_coldot(const double *X, const double *Y, int64_t n, int nrhs, double *partials, double *out,
                   cudaStream_t st) {
    ++g_kernel_launches;
    coldot_partial_kernel<<<kReduceBlocks, 256, 0, st>>>(X, Y, n, nrhs, partials);
    ++g_kernel_launches;
    coldot_final_kernel<<<1, 64, 0, st>>>(partials, kReduceBlocks, nrhs, out);
}

void launch_colnorm2(const double *X, int64_t n, int nrhs, double *partials, double *out, cudaStream_t st) {
    launch_coldot(X, X, n, nrhs, partials, out, st);
}

void launch_pcg_update_x_r(double *X, double *R, const double *P, const double *AP, const double *rz,
                           const double *pap, const int *active, int64_t n, int nrhs, cudaStream_t st) {
    ++g_kernel_launches;
    pcg_xr_kernel<<<grid_for(n * nrhs, 256), 256, 0, st>>>(X, R, P, AP, rz, pap, active, n, nrhs);
}

void launch_pcg_update_p(double *P, const double *Z, const double *rz_new, const double *rz_old, const int *active,
                         int64_t n, int nrhs, cudaStream_t st) {
    ++g_kernel_launches;
    pcg_p_kernel<<<grid_for(n * nrhs, 256), 256, 0, st>>>(P, Z, rz_new, rz_old, active, n, nrhs);
}

void launch_copy(double *dst, const double *src, int64_t count, cudaStream_t st) {
    if (count <= 0) return;
    ++g_kernel_launches;
    copy_kernel<<<grid_for(count, 256), 256, 0, st>>>(dst, src, count);
}

void launch_axpy(double *y, const double *x, double alpha, int64_t count, cudaStream_t st) {
    if (count <= 0) return;
    ++g_kernel_launches;
    axpy_kernel<<<grid_for(count, 256), 256, 0, st>>>(y, x, alpha, count);
}

}  // namespace mfs
