// Test hooks (include/mfs_b200_testing.h): single kernels of the numeric
// factorization on caller device arrays, with every access bounds-checked on the
// host before the launch.
#include "../../include/mfs_b200_testing.h"
#include "device.h"
#include "host_symbolic.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace mfs;

namespace {

void put_error(char *buf, size_t len, const std::string &msg) {
    if (buf && len > 0) {
        std::snprintf(buf, len, "%s", msg.c_str());
    }
}

}  // namespace

extern "C" mfs_status mfs_debug_gemm(int32_t device, int32_t precision, int32_t kernel, int64_t ntasks,
                                     const int64_t *tasks, const void *A, int64_t a_len, const void *B,
                                     int64_t b_len, void *C, int64_t c_len, char *err_buf, size_t err_len) {
    const bool f64 = precision == MFS_PREC_FP64;
    if (precision != MFS_PREC_FP64 && precision != MFS_PREC_FP32) {
        put_error(err_buf, err_len, "unknown precision");
        return MFS_INVALID_ARG;
    }
    if (ntasks <= 0 || !tasks || !A || !B || !C) {
        put_error(err_buf, err_len, "empty task list or null array");
        return MFS_INVALID_ARG;
    }
    if (!f64 && (kernel < 0 || kernel > 7 || kernel == 2)) {
        put_error(err_buf, err_len, "kernel must be 0, 1, 3, 4, 5, 6 or 7");
        return MFS_INVALID_ARG;
    }
    const bool tma = !f64 && (kernel == 4 || kernel == 5 || kernel == 6);
    const bool split16 = !f64 && kernel == 6;           // A and B: FP16 hi array, then FP16 lo array
    const bool half = !f64 && (kernel == 5 || kernel == 6);   // A and B are FP16
    const bool split32 = !f64 && kernel == 7;           // tcgen05 split TF32 (FP32 operands)
    if (split16 && ((a_len & 1) || (b_len & 1))) {
        put_error(err_buf, err_len, "kernel 6: A and B hold two equal halves (hi, lo)");
        return MFS_INVALID_ARG;
    }
    // element count of one operand copy (kernel 6: each half)
    const int64_t a_ext = split16 ? a_len / 2 : a_len, b_ext = split16 ? b_len / 2 : b_len;
    std::vector<TensorMapBlob> maps;
    const int TM = gemm_tile_m(f64), TN = gemm_tile_n(f64);
    std::vector<GemmTask> gt(static_cast<size_t>(ntasks));
    int base = 0;
    for (int64_t t = 0; t < ntasks; ++t) {
        const int64_t *q = tasks + t * MFS_GEMM_TASK_FIELDS;
        const int64_t a_off = q[0], b_off = q[1], c_off = q[2], lda = q[3], ldb = q[4], ldc = q[5];
        const int64_t m = q[6], n = q[7], k = q[8], lower = q[9], mode = q[10], scale_exp = q[11];
        const std::string id = "task " + std::to_string(t) + ": ";
        if (m <= 0 || n <= 0 || k <= 0 || m > (1 << 30) || n > (1 << 30) || k > (1 << 30)) {
            put_error(err_buf, err_len, id + "m, n, k must be positive");
            return MFS_INVALID_ARG;
        }
        if ((mode != 0 && mode != 1) || (lower != 0 && lower != 1)) {
            put_error(err_buf, err_len, id + "mode and lower must be 0 or 1");
            return MFS_INVALID_ARG;
        }
        if (lda < m || ldb < n || ldc < m || lda > INT32_MAX || ldb > INT32_MAX || ldc > INT32_MAX) {
            put_error(err_buf, err_len, id + "leading dimension below the extent");
            return MFS_INVALID_ARG;
        }
        int da = 0, db = 0;
        if (!f64) {
            // 16-byte aligned columns; tiles start at the 8-element boundary at or before
            // the operand, as in the factorization
            const int64_t al = half ? 7 : 3;
            if ((lda & al) || (ldb & al)) {
                put_error(err_buf, err_len, id + "leading dimensions must span whole 16-byte units");
                return MFS_INVALID_ARG;
            }
            da = int(a_off & 7);
            db = int(b_off & 7);
        }
        if (scale_exp < -60 || scale_exp > 60 || (scale_exp != 0 && !half)) {
            put_error(err_buf, err_len, id + "scale_exp applies to FP16 operands only (|scale_exp| <= 60)");
            return MFS_INVALID_ARG;
        }
        // the kernels read A rows [a_off - da, a_off + m) of columns 0..k-1, B likewise,
        // and write C rows [0, m) of columns 0..n-1
        if (a_off - da < 0 || b_off - db < 0 || c_off < 0 || a_off + (k - 1) * lda + m > a_ext ||
            b_off + (k - 1) * ldb + n > b_ext || c_off + (n - 1) * ldc + m > c_len) {
            put_error(err_buf, err_len, id + "an access falls outside the arrays");
            return MFS_INVALID_ARG;
        }
        GemmTask &g = gt[size_t(t)];
        g.a_off = a_off; g.b_off = b_off; g.c_off = c_off;
        g.lda = int32_t(lda); g.ldb = int32_t(ldb); g.ldc = int32_t(ldc);
        g.m = int32_t(m); g.n = int32_t(n); g.k = int32_t(k);
        g.shift = da | (db << 8);
        g.tiles_m = int32_t((m + da + TM - 1) / TM);
        g.tiles_n = int32_t((n + db + TN - 1) / TN);
        g.tile_base = base;
        g.lower = int32_t(lower);
        g.mode = int32_t(mode);
        g.amap = g.bmap = -1;
        g.ax = g.ay = g.bx = g.by = 0;
        g.scale_exp = int32_t(scale_exp);
        g.sn = split32 ? 0 : -1;
        if (tma) {
            // one tensor map per operand, starting at the shifted (16-byte aligned) operand
            if (mode != 0) {
                put_error(err_buf, err_len, id + "the TMA-fed kernel runs mode 0 only");
                return MFS_INVALID_ARG;
            }
            maps.resize(maps.size() + 2);
            TensorMapBlob *ma = &maps[maps.size() - 2], *mb = &maps[maps.size() - 1];
            const size_t es = half ? 2 : 4;
            const char *Af = static_cast<const char *>(A) + size_t(a_off - da) * es;
            const char *Bf = static_cast<const char *>(B) + size_t(b_off - db) * es;
            if ((reinterpret_cast<uintptr_t>(Af) & 15) || (reinterpret_cast<uintptr_t>(Bf) & 15)) {
                put_error(err_buf, err_len, id + "arrays must be 16-byte aligned");
                return MFS_INVALID_ARG;
            }
            const int ops = split16 ? 2 : half ? 1 : 0;
            if (!encode_operand_map(ma, Af, ops, uint64_t(m + da), uint64_t(k), uint64_t(lda)) ||
                !encode_operand_map(mb, Bf, ops, uint64_t(n + db), uint64_t(k), uint64_t(ldb))) {
                put_error(err_buf, err_len, id + "tensor map refused by the driver");
                return MFS_INVALID_ARG;
            }
            g.amap = int32_t(maps.size() - 2);
            g.bmap = int32_t(maps.size() - 1);
        }
        if (split32 && lower && mode == 1) {
            put_error(err_buf, err_len, id + "row solves (mode 1) are not lower");
            return MFS_INVALID_ARG;
        }
        if (int64_t(base) + int64_t(g.tiles_m) * g.tiles_n > INT32_MAX / 2) {
            put_error(err_buf, err_len, "too many tiles");
            return MFS_INVALID_ARG;
        }
        base += g.tiles_m * g.tiles_n;
    }
    if (split16) {
        // the lo copies' maps, in the same order, 2 ntasks entries after the hi ones
        const size_t nh = maps.size();
        maps.resize(2 * nh);
        for (int64_t t = 0; t < ntasks; ++t) {
            const GemmTask &g = gt[size_t(t)];
            const int da = g.shift & 255, db = g.shift >> 8;
            const char *Al = static_cast<const char *>(A) + size_t(a_ext + g.a_off - da) * 2;
            const char *Bl = static_cast<const char *>(B) + size_t(b_ext + g.b_off - db) * 2;
            if ((reinterpret_cast<uintptr_t>(Al) & 15) || (reinterpret_cast<uintptr_t>(Bl) & 15) ||
                !encode_operand_map(&maps[nh + size_t(g.amap)], Al, 2, uint64_t(g.m + da), uint64_t(g.k),
                                    uint64_t(g.lda)) ||
                !encode_operand_map(&maps[nh + size_t(g.bmap)], Bl, 2, uint64_t(g.n + db), uint64_t(g.k),
                                    uint64_t(g.ldb))) {
                put_error(err_buf, err_len, "kernel 6: lo tensor map refused (alignment or driver)");
                return MFS_INVALID_ARG;
            }
        }
    }
    GemmTask *dt = nullptr;
    int *derr = nullptr;
    TensorMapBlob *dmaps = nullptr;
    void *h16s = nullptr, *h16l = nullptr;
    int32_t *dsexp = nullptr;
    auto fail = [&](cudaError_t e) {
        put_error(err_buf, err_len, cudaGetErrorString(e));
        if (dt) cudaFree(dt);
        if (derr) cudaFree(derr);
        if (dmaps) cudaFree(dmaps);
        if (h16s) cudaFree(h16s);
        if (h16l) cudaFree(h16l);
        if (dsexp) cudaFree(dsexp);
        return MFS_CUDA_ERROR;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&dt, gt.size() * sizeof(GemmTask))) != cudaSuccess) return fail(e);
    if ((e = cudaMalloc(&derr, sizeof(int))) != cudaSuccess) return fail(e);
    if ((e = cudaMemcpy(dt, gt.data(), gt.size() * sizeof(GemmTask), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e);
    if ((e = cudaMemset(derr, 0, sizeof(int))) != cudaSuccess) return fail(e);
    if (tma) {
        if ((e = cudaMalloc(&dmaps, maps.size() * sizeof(TensorMapBlob))) != cudaSuccess) return fail(e);
        if ((e = cudaMemcpy(dmaps, maps.data(), maps.size() * sizeof(TensorMapBlob), cudaMemcpyHostToDevice)) !=
            cudaSuccess)
            return fail(e);
        launch_gemm_tma(split16 ? 2 : half ? 1 : 0, dt, int(ntasks), base, dmaps, static_cast<float *>(C), nullptr,
                        derr, nullptr, int(maps.size() / 2));
    } else if (split32) {
        // the row solves' half-copy outputs go to scratch (scale exponent 0)
        if ((e = cudaMalloc(&h16s, size_t(c_len) * 2)) != cudaSuccess) return fail(e);
        if ((e = cudaMalloc(&h16l, size_t(c_len) * 2)) != cudaSuccess) return fail(e);
        if ((e = cudaMalloc(&dsexp, sizeof(int32_t))) != cudaSuccess) return fail(e);
        if ((e = cudaMemset(dsexp, 0, sizeof(int32_t))) != cudaSuccess) return fail(e);
        launch_gemm_tc(dt, int(ntasks), base, static_cast<const float *>(A), static_cast<const float *>(B),
                       static_cast<float *>(C), derr, nullptr, h16s, dsexp, h16l);
    } else if (f64)
        launch_gemm<double>(dt, int(ntasks), base, static_cast<const double *>(A), static_cast<const double *>(B),
                            static_cast<double *>(C), 0, derr, nullptr);
    else
        launch_gemm<float>(dt, int(ntasks), base, static_cast<const float *>(A), static_cast<const float *>(B),
                           static_cast<float *>(C), kernel, derr, nullptr);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(e);
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return fail(e);
    int herr = 0;
    if ((e = cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess) return fail(e);
    cudaFree(dt);
    cudaFree(derr);
    if (dmaps) cudaFree(dmaps);
    if (h16s) cudaFree(h16s);
    if (h16l) cudaFree(h16l);
    if (dsexp) cudaFree(dsexp);
    if (herr) {
        put_error(err_buf, err_len, "a tensor-core pipeline wait timed out");
        return MFS_TIMEOUT;
    }
    return MFS_OK;
}

extern "C" mfs_status mfs_debug_dirty_subtrees(int64_t n, const int64_t *xadj, const int64_t *adj, int64_t ncomp,
                                               const int64_t *cparent, const int64_t *cmember,
                                               int32_t *full_rebuild, int64_t *roots, int64_t *nroots) {
    if (n < 0 || ncomp < 0 || !xadj || !full_rebuild || !nroots || (ncomp > 0 && (!cparent || !roots)) ||
        (n > 0 && !cmember))
        return MFS_INVALID_ARG;
    const int64_t ne = xadj[n];
    if (ne < 0 || (ne > 0 && !adj)) return MFS_INVALID_ARG;
    for (int64_t v = 0; v < n; ++v)
        if (xadj[v] > xadj[v + 1] || cmember[v] < 0 || cmember[v] >= ncomp) return MFS_INVALID_ARG;
    for (int64_t k = 0; k < ne; ++k)
        if (adj[k] < 0 || adj[k] >= n) return MFS_INVALID_ARG;
    for (int64_t c = 0; c < ncomp; ++c)
        if (cparent[c] != -1 && (cparent[c] <= c || cparent[c] >= ncomp)) return MFS_INVALID_ARG;
    try {
        const std::vector<idx> x(xadj, xadj + n + 1), a(adj, adj + ne), p(cparent, cparent + ncomp),
            m(cmember, cmember + n);
        const DirtySubtrees d = dirty_subtrees(n, x, a, p, m);
        *full_rebuild = d.full ? 1 : 0;
        *nroots = int64_t(d.roots.size());
        for (size_t r = 0; r < d.roots.size(); ++r) roots[r] = d.roots[r];
        return MFS_OK;
    } catch (const std::bad_alloc &) {
        return MFS_OOM;
    }
}

extern "C" mfs_status mfs_debug_hierarchical_order(int64_t n, const int64_t *xadj, const int64_t *adj,
                                                   int64_t ncomp, const int64_t *cparent, const int64_t *cmember,
                                                   int32_t cut_depth, int64_t *perm, int64_t *stats) {
    if (n < 0 || ncomp < 0 || !xadj || !stats || cut_depth < 0 || (n > 0 && (!cmember || !perm)) ||
        (ncomp > 0 && !cparent))
        return MFS_INVALID_ARG;
    const int64_t ne = xadj[n];
    if (ne < 0 || (ne > 0 && !adj)) return MFS_INVALID_ARG;
    for (int64_t v = 0; v < n; ++v)
        if (xadj[v] > xadj[v + 1] || cmember[v] < 0 || cmember[v] >= ncomp) return MFS_INVALID_ARG;
    for (int64_t k = 0; k < ne; ++k)
        if (adj[k] < 0 || adj[k] >= n) return MFS_INVALID_ARG;
    for (int64_t c = 0; c < ncomp; ++c)
        if (cparent[c] != -1 && (cparent[c] <= c || cparent[c] >= ncomp)) return MFS_INVALID_ARG;
    try {
        NDResult nd;
        nd.ncomp = ncomp;
        nd.cparent.assign(cparent, cparent + ncomp);
        nd.cmember.assign(cmember, cmember + n);
        nd.iperm.resize(size_t(n));
        for (int64_t v = 0; v < n; ++v) nd.iperm[size_t(v)] = v;
        // every edge joins a component to itself or to an ancestor or descendant
        std::vector<int64_t> depth(size_t(ncomp), 0);
        for (int64_t c = ncomp - 1; c >= 0; --c)
            if (cparent[c] >= 0) depth[size_t(c)] = depth[size_t(cparent[c])] + 1;
        for (int64_t v = 0; v < n; ++v)
            for (int64_t k = xadj[v]; k < xadj[v + 1]; ++k) {
                int64_t a = cmember[v], b = cmember[adj[k]];
                if (depth[size_t(a)] < depth[size_t(b)]) std::swap(a, b);
                while (depth[size_t(a)] > depth[size_t(b)]) a = cparent[a];
                if (a != b) return MFS_INVALID_ARG;
            }
        const std::vector<idx> x(xadj, xadj + n + 1), a(adj, adj + ne);
        HierarchicalMDStats st;
        const std::vector<idx> p = hierarchical_constrained_md(n, x, a, nd, cut_depth, &st);
        if (!st.applied && n > 0) return MFS_INVALID_ARG;
        for (int64_t k = 0; k < n; ++k) perm[k] = p[size_t(k)];
        stats[0] = st.cut_depth;
        stats[1] = st.tasks;
        stats[2] = st.upper_vertices;
        stats[3] = st.upper_elements;
        return MFS_OK;
    } catch (const std::bad_alloc &) {
        return MFS_OOM;
    }
}
