// GPU construction of the symbolic structures that change with the mesh pattern:
//
//   block sparsity pattern from element stencils (SystemAssembler.hh:252-465):
//     per element the stencil is sorted; every column counts the stencil entries
//     at or above its own position (k + 1 for position k), the counts are scanned,
//     the (row, column) pairs are bucketed with atomic cursors, and each column's
//     bucket is sorted and de-duplicated (one thread per column). The buckets hold
//     the same multiset as the host construction's, so Ap / Ai are identical.
//   element -> slot map of the assembly (SystemAssembler.hh:60-98, 524-543): ten
//     contributions per tet located by binary search in their column, counted,
//     scanned, bucketed, and each slot's list sorted by contribution index so that
//     slots sum in element order as the host map does.
//   block conversion plan (CatamariConversionPlan.hh:402-541): the full symmetric
//     adjacency of the reduced pattern (own upper entries first, then the mirrored
//     entries of later columns in column order, as the host builds it), then per
//     permuted column one thread walks that adjacency and writes each entry into
//     its bucket (2j: source from the lower triangle, transposed; 2j + 1: strict
//     upper, copied) in the host's order, in the catamari panel layout and in the
//     device panel layout.
// Scans use CUB; everything else is written here. Invalid input (an index out of
// range, an element block missing from the pattern) sets an error code that the
// host turns into MFS_INVALID_ARG.
#include "device.h"
#include "handle.h"

#include <cub/cub.cuh>

#include <algorithm>
#include <cstdint>
#include <vector>

namespace mfs {

namespace {

constexpr int kMaxStencil = 32;

inline int grid_of(int64_t n, int threads) {
    return int(std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 148 * 64)));
}

// In place: a[0..n) := inclusive prefix sums (a[0] is left as is).
void inclusive_scan(int64_t *a, int64_t n, cudaStream_t st) {
    if (n <= 1) return;
    DBuf<int64_t> out;
    out.ensure(size_t(n));
    size_t tmp = 0;
    MFS_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, a, out.p, n, st));
    DBuf<unsigned char> t;
    t.ensure(std::max<size_t>(tmp, 1));
    MFS_CUDA(cub::DeviceScan::InclusiveSum(t.p, tmp, a, out.p, n, st));
    MFS_CUDA(cudaMemcpyAsync(a, out.p, size_t(n) * sizeof(int64_t), cudaMemcpyDeviceToDevice, st));
    MFS_CUDA(cudaStreamSynchronize(st));
}

__device__ __forceinline__ void sort_small(int64_t *v, int n) {
    for (int i = 1; i < n; ++i) {
        const int64_t x = v[i];
        int j = i - 1;
        while (j >= 0 && v[j] > x) {
            v[j + 1] = v[j];
            --j;
        }
        v[j + 1] = x;
    }
}
__device__ __forceinline__ void sort_segment(int64_t *v, int64_t n) {
    for (int64_t i = 1; i < n; ++i) {
        const int64_t x = v[i];
        int64_t j = i - 1;
        while (j >= 0 && v[j] > x) {
            v[j + 1] = v[j];
            --j;
        }
        v[j + 1] = x;
    }
}

// ---------------------------------------------------------------- pattern
__global__ void pattern_count_kernel(int64_t nelem, int npe, const int64_t *__restrict__ conn, int64_t nvars,
                                     unsigned long long *cnt, int *err) {
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < nelem; e += int64_t(gridDim.x) * blockDim.x) {
        int64_t s[kMaxStencil];
        for (int k = 0; k < npe; ++k) s[k] = conn[e * npe + k];
        sort_small(s, npe);
        if (s[0] < 0 || s[npe - 1] >= nvars) {
            atomicExch(err, 1);
            continue;
        }
        for (int k = 0; k < npe; ++k) atomicAdd(&cnt[s[k] + 1], (unsigned long long)(k + 1));
    }
}

__global__ void pattern_fill_kernel(int64_t nelem, int npe, const int64_t *__restrict__ conn,
                                    unsigned long long *back, int64_t *__restrict__ buckets) {
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < nelem; e += int64_t(gridDim.x) * blockDim.x) {
        int64_t s[kMaxStencil];
        for (int k = 0; k < npe; ++k) s[k] = conn[e * npe + k];
        sort_small(s, npe);
        for (int b = 0; b < npe; ++b)
            for (int a = 0; a <= b; ++a) {
                const unsigned long long p = atomicAdd(&back[s[b]], 1ull);
                buckets[p] = s[a];
            }
    }
}

// Sort and de-duplicate each column's bucket in place; cnt[j + 1] = unique rows.
__global__ void pattern_unique_kernel(int64_t nvars, const int64_t *__restrict__ start, int64_t *buckets,
                                      int64_t *cnt) {
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < nvars; j += int64_t(gridDim.x) * blockDim.x) {
        int64_t *b = buckets + start[j];
        const int64_t n = start[j + 1] - start[j];
        sort_segment(b, n);
        int64_t u = 0;
        for (int64_t i = 0; i < n; ++i)
            if (i == 0 || b[i] != b[i - 1]) b[u++] = b[i];
        cnt[j + 1] = u;
    }
}

__global__ void pattern_emit_kernel(int64_t nvars, const int64_t *__restrict__ start,
                                    const int64_t *__restrict__ buckets, const int64_t *__restrict__ Ap,
                                    int64_t *__restrict__ Ai) {
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < nvars; j += int64_t(gridDim.x) * blockDim.x) {
        const int64_t *b = buckets + start[j];
        for (int64_t k = Ap[j]; k < Ap[j + 1]; ++k) Ai[k] = b[k - Ap[j]];
    }
}

// --------------------------------------------------------------- slot map
__device__ __forceinline__ int64_t find_row(const int64_t *Ap, const int64_t *Ai, int64_t j, int64_t i) {
    int64_t lo = Ap[j], hi = Ap[j + 1];
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (Ai[mid] < i) lo = mid + 1;
        else hi = mid;
    }
    return (lo < Ap[j + 1] && Ai[lo] == i) ? lo : -1;
}

// Ten contributions per tet, in the host map's order: columns by ascending node
// (ties keep the local order), the upper blocks of a column, then its diagonal.
__global__ void slot_compute_kernel(int64_t nelem, const int64_t *__restrict__ conn, int64_t nb,
                                    const int64_t *__restrict__ Ap, const int64_t *__restrict__ Ai,
                                    int64_t *__restrict__ slots, int64_t *__restrict__ codes, unsigned long long *cnt,
                                    int *err) {
    for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < nelem; e += int64_t(gridDim.x) * blockDim.x) {
        int64_t v[4];
        bool ok = true;
        for (int k = 0; k < 4; ++k) {
            v[k] = conn[4 * e + k];
            if (v[k] < 0 || v[k] >= nb) ok = false;
        }
        if (!ok) {
            atomicExch(err, 1);
            for (int q = 0; q < 10; ++q) slots[e * 10 + q] = -1;
            continue;
        }
        int order[4] = {0, 1, 2, 3};
        for (int i = 1; i < 4; ++i) {                       // stable insertion sort by node
            const int x = order[i];
            int j = i - 1;
            while (j >= 0 && v[order[j]] > v[x]) {
                order[j + 1] = order[j];
                --j;
            }
            order[j + 1] = x;
        }
        int q = 0;
        for (int jj = 0; jj < 4; ++jj) {
            const int lj = order[jj];
            const int64_t bj = v[lj];
            for (int ii = 0; ii < jj; ++ii) {
                const int li = order[ii];
                const int64_t slot = find_row(Ap, Ai, bj, v[li]);
                const int64_t code = li < lj ? (((e * 144 + (3 * li) * 12 + 3 * lj) << 2) | 0)
                                             : (((e * 144 + (3 * lj) * 12 + 3 * li) << 2) | 1);
                slots[e * 10 + q] = slot;
                codes[e * 10 + q] = code;
                if (slot < 0) atomicExch(err, 2);
                else atomicAdd(&cnt[slot + 1], 1ull);
                ++q;
            }
            const int64_t slot = find_row(Ap, Ai, bj, bj);
            slots[e * 10 + q] = slot;
            codes[e * 10 + q] = ((e * 144 + (3 * lj) * 12 + 3 * lj) << 2) | 2;
            if (slot < 0) atomicExch(err, 2);
            else atomicAdd(&cnt[slot + 1], 1ull);
            ++q;
        }
    }
}

__global__ void slot_fill_kernel(int64_t ncontrib, const int64_t *__restrict__ slots, unsigned long long *back,
                                 int64_t *__restrict__ kidx) {
    for (int64_t k = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; k < ncontrib;
         k += int64_t(gridDim.x) * blockDim.x) {
        const int64_t s = slots[k];
        if (s < 0) continue;
        kidx[atomicAdd(&back[s], 1ull)] = k;
    }
}

__global__ void slot_order_kernel(int64_t nslots, const int64_t *__restrict__ slot_ptr, int64_t *kidx,
                                  const int64_t *__restrict__ codes, int64_t *__restrict__ contrib) {
    for (int64_t s = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; s < nslots; s += int64_t(gridDim.x) * blockDim.x) {
        int64_t *b = kidx + slot_ptr[s];
        const int64_t n = slot_ptr[s + 1] - slot_ptr[s];
        sort_segment(b, n);
        for (int64_t p = 0; p < n; ++p) contrib[slot_ptr[s] + p] = codes[b[p]];
    }
}

// ------------------------------------------------------- conversion plan
// Mirrored entries (i, j), i < j, of the reduced upper pattern go to column i.
__global__ void mirror_count_kernel(int64_t nv, const int64_t *__restrict__ Ap, const int64_t *__restrict__ Ai,
                                    unsigned long long *cnt) {
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < nv; j += int64_t(gridDim.x) * blockDim.x) {
        atomicAdd(&cnt[j + 1], (unsigned long long)(Ap[j + 1] - Ap[j]));
        for (int64_t k = Ap[j]; k < Ap[j + 1]; ++k)
            if (Ai[k] != j) atomicAdd(&cnt[Ai[k] + 1], 1ull);
    }
}
// Own entries first (in pattern order), mirrored ones appended by atomic cursor.
__global__ void mirror_fill_kernel(int64_t nv, const int64_t *__restrict__ Ap, const int64_t *__restrict__ Ai,
                                   const int64_t *__restrict__ fptr, unsigned long long *back,
                                   int64_t *__restrict__ fent) {
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < nv; j += int64_t(gridDim.x) * blockDim.x) {
        for (int64_t k = Ap[j]; k < Ap[j + 1]; ++k) {
            fent[fptr[j] + (k - Ap[j])] = k;
            if (Ai[k] != j) fent[atomicAdd(&back[Ai[k]], 1ull)] = k;
        }
    }
}
// The mirrored part of every column in entry order (= the order of their columns).
__global__ void mirror_sort_kernel(int64_t nv, const int64_t *__restrict__ Ap, const int64_t *__restrict__ fptr,
                                   int64_t *fent) {
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < nv; j += int64_t(gridDim.x) * blockDim.x) {
        const int64_t own = Ap[j + 1] - Ap[j];
        sort_segment(fent + fptr[j] + own, fptr[j + 1] - fptr[j] - own);
    }
}

struct PlanArgs {
    int64_t nv;
    int vb;
    const int64_t *Ap, *Ai, *src_off, *fptr, *fent, *perm, *iperm;
    const int64_t *sn_start, *struct_ptr, *struct_rows, *w, *f, *pan_off, *dpan;
    const int32_t *dld;
    int64_t nsn;
};
__device__ __forceinline__ int64_t entry_column(const PlanArgs &a, int64_t k) {
    int64_t lo = 0, hi = a.nv;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (a.Ap[mid + 1] <= k) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}
// The other end of adjacency entry p of column oj (entry k = fent[p]).
__device__ __forceinline__ int64_t adj_of(const PlanArgs &a, int64_t oj, int64_t p) {
    const int64_t k = a.fent[p];
    const int64_t own = a.Ap[oj + 1] - a.Ap[oj];
    return (p - a.fptr[oj] < own) ? a.Ai[k] : entry_column(a, k);
}

__global__ void plan_count_kernel(PlanArgs a, int64_t *__restrict__ cnt) {
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < a.nv; j += int64_t(gridDim.x) * blockDim.x) {
        const int64_t oj = a.iperm[j];
        int64_t c0 = 0, c1 = 0;
        for (int64_t p = a.fptr[oj]; p < a.fptr[oj + 1]; ++p) {
            const int64_t oi = adj_of(a, oj, p);
            if (a.perm[oi] < j) continue;
            if (oi >= oj) ++c0;
            else ++c1;
        }
        cnt[2 * j + 1] = c0;
        cnt[2 * j + 2] = c1;
    }
}

__global__ void plan_fill_kernel(PlanArgs a, const int64_t *__restrict__ plan_ptr, PlanEntryDev *__restrict__ cat,
                                 PlanEntryDev *__restrict__ dev, int *err) {
    for (int64_t j = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; j < a.nv; j += int64_t(gridDim.x) * blockDim.x) {
        const int64_t oj = a.iperm[j];
        int64_t lo = 0, hi = a.nsn;                     // supernode of column j
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (a.sn_start[mid + 1] <= j) lo = mid + 1;
            else hi = mid;
        }
        const int64_t s = lo;
        const int64_t jr = int64_t(a.vb) * (j - a.sn_start[s]);
        const int64_t *pb = a.struct_rows + a.struct_ptr[s];
        const int64_t nst = a.struct_ptr[s + 1] - a.struct_ptr[s];
        int64_t b0 = plan_ptr[2 * j], b1 = plan_ptr[2 * j + 1];
        for (int64_t p = a.fptr[oj]; p < a.fptr[oj + 1]; ++p) {
            const int64_t oi = adj_of(a, oj, p);
            const int64_t i = a.perm[oi];
            if (i < j) continue;
            int64_t ir;
            if (i < a.sn_start[s + 1]) {
                ir = int64_t(a.vb) * (i - a.sn_start[s]);
            } else {
                int64_t l = 0, h = nst;
                while (l < h) {
                    const int64_t m = (l + h) >> 1;
                    if (pb[m] < i) l = m + 1;
                    else h = m;
                }
                if (l >= nst || pb[l] != i) {
                    atomicExch(err, 3);
                    continue;
                }
                ir = a.w[s] + int64_t(a.vb) * l;
            }
            PlanEntryDev e;
            e.dst = a.pan_off[s] + jr * a.f[s] + ir;
            e.src = a.src_off[a.fent[p]];
            e.ld = int32_t(a.f[s]);
            e.flags = (oi >= oj ? 1 : 0) | (i == j ? 2 : 0);
            const int64_t pos = oi >= oj ? b0++ : b1++;
            cat[pos] = e;
            e.dst = a.dpan[s] + jr * a.dld[s] + ir;
            e.ld = a.dld[s];
            dev[pos] = e;
        }
    }
}

}  // namespace

int64_t gpu_build_pattern(int64_t nvars, int64_t nelem, int npe, const int64_t *conn, int64_t *Ap, int64_t *Ai,
                          cudaStream_t st) {
    if (npe <= 0 || npe > kMaxStencil) throw StatusError(MFS_INVALID_ARG, "stencil size must be 1 .. 32");
    DBuf<int> err;
    err.ensure(1);
    MFS_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), st));
    DBuf<int64_t> start, back, buckets, cnt;
    start.ensure(size_t(nvars + 1));
    MFS_CUDA(cudaMemsetAsync(start.p, 0, size_t(nvars + 1) * sizeof(int64_t), st));
    if (nelem > 0) {
        pattern_count_kernel<<<grid_of(nelem, 256), 256, 0, st>>>(nelem, npe, conn, nvars,
                                                                  reinterpret_cast<unsigned long long *>(start.p),
                                                                  err.p);
        MFS_LAUNCHED();
    }
    int herr = 0;
    MFS_CUDA(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MFS_CUDA(cudaStreamSynchronize(st));
    if (herr) throw StatusError(MFS_INVALID_ARG, "Stencil index exceeds the number of block variables");
    inclusive_scan(start.p, nvars + 1, st);
    int64_t total = 0;
    MFS_CUDA(cudaMemcpy(&total, start.p + nvars, sizeof(int64_t), cudaMemcpyDeviceToHost));
    buckets.ensure(size_t(std::max<int64_t>(total, 1)));
    back.ensure(size_t(nvars + 1));
    MFS_CUDA(cudaMemcpyAsync(back.p, start.p, size_t(nvars + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, st));
    if (nelem > 0) {
        pattern_fill_kernel<<<grid_of(nelem, 256), 256, 0, st>>>(
            nelem, npe, conn, reinterpret_cast<unsigned long long *>(back.p), buckets.p);
        MFS_LAUNCHED();
    }
    MFS_CUDA(cudaMemsetAsync(Ap, 0, size_t(nvars + 1) * sizeof(int64_t), st));
    if (nvars > 0) {
        pattern_unique_kernel<<<grid_of(nvars, 128), 128, 0, st>>>(nvars, start.p, buckets.p, Ap);
        MFS_LAUNCHED();
    }
    inclusive_scan(Ap, nvars + 1, st);
    int64_t nnz = 0;
    MFS_CUDA(cudaMemcpy(&nnz, Ap + nvars, sizeof(int64_t), cudaMemcpyDeviceToHost));
    if (Ai && nvars > 0) {
        pattern_emit_kernel<<<grid_of(nvars, 128), 128, 0, st>>>(nvars, start.p, buckets.p, Ap, Ai);
        MFS_LAUNCHED();
        MFS_CUDA(cudaStreamSynchronize(st));
    }
    return nnz;
}

void gpu_build_slot_map(int64_t nelem, const int64_t *conn, int64_t nb, const int64_t *Ap, const int64_t *Ai,
                        int64_t nslots, DBuf<int64_t> &slot_ptr, DBuf<int64_t> &contrib, cudaStream_t st) {
    const int64_t ncontrib = nelem * 10;
    DBuf<int> err;
    err.ensure(1);
    MFS_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), st));
    DBuf<int64_t> slots, codes, kidx, back;
    slots.ensure(size_t(std::max<int64_t>(ncontrib, 1)));
    codes.ensure(size_t(std::max<int64_t>(ncontrib, 1)));
    slot_ptr.ensure(size_t(nslots + 1));
    MFS_CUDA(cudaMemsetAsync(slot_ptr.p, 0, size_t(nslots + 1) * sizeof(int64_t), st));
    if (nelem > 0) {
        slot_compute_kernel<<<grid_of(nelem, 256), 256, 0, st>>>(
            nelem, conn, nb, Ap, Ai, slots.p, codes.p, reinterpret_cast<unsigned long long *>(slot_ptr.p), err.p);
        MFS_LAUNCHED();
    }
    int herr = 0;
    MFS_CUDA(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MFS_CUDA(cudaStreamSynchronize(st));
    if (herr == 1) throw StatusError(MFS_INVALID_ARG, "element node out of range");
    if (herr) throw StatusError(MFS_INVALID_ARG, "element block not in the pattern");
    inclusive_scan(slot_ptr.p, nslots + 1, st);
    back.ensure(size_t(nslots + 1));
    MFS_CUDA(cudaMemcpyAsync(back.p, slot_ptr.p, size_t(nslots + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, st));
    kidx.ensure(size_t(std::max<int64_t>(ncontrib, 1)));
    contrib.ensure(size_t(std::max<int64_t>(ncontrib, 1)));
    if (ncontrib > 0) {
        slot_fill_kernel<<<grid_of(ncontrib, 256), 256, 0, st>>>(
            ncontrib, slots.p, reinterpret_cast<unsigned long long *>(back.p), kidx.p);
        MFS_LAUNCHED();
    }
    if (nslots > 0) {
        slot_order_kernel<<<grid_of(nslots, 128), 128, 0, st>>>(nslots, slot_ptr.p, kidx.p, codes.p, contrib.p);
        MFS_LAUNCHED();
    }
    MFS_CUDA(cudaStreamSynchronize(st));
}

void gpu_build_plan(const Symbolic &S, const std::vector<int64_t> &dpan, const std::vector<int32_t> &dld,
                    DBuf<PlanEntryDev> &plan_dev, DBuf<PlanEntryDev> &plan_cat, DBuf<int64_t> &plan_ptr,
                    cudaStream_t st) {
    const int64_t nv = S.nv;
    DBuf<int64_t> Ap, Ai, src, perm, iperm, sn_start, sptr, srows, w, f, pan, dp, fptr, back, fent;
    DBuf<int32_t> dl;
    Ap.upload(S.A.Ap, st);
    Ai.upload(S.A.Ai, st);
    src.upload(S.src_off, st);
    perm.upload(S.perm, st);
    iperm.upload(S.iperm, st);
    sn_start.upload(S.sn_start, st);
    sptr.upload(S.struct_ptr, st);
    srows.upload(S.struct_rows, st);
    w.upload(S.w, st);
    f.upload(S.f, st);
    pan.upload(S.pan_off, st);
    dp.upload(dpan, st);
    dl.upload(dld, st);
    // full symmetric adjacency
    fptr.ensure(size_t(nv + 1));
    MFS_CUDA(cudaMemsetAsync(fptr.p, 0, size_t(nv + 1) * sizeof(int64_t), st));
    if (nv > 0) {
        mirror_count_kernel<<<grid_of(nv, 128), 128, 0, st>>>(nv, Ap.p, Ai.p,
                                                              reinterpret_cast<unsigned long long *>(fptr.p));
        MFS_LAUNCHED();
    }
    inclusive_scan(fptr.p, nv + 1, st);
    int64_t nadj = 0;
    MFS_CUDA(cudaMemcpy(&nadj, fptr.p + nv, sizeof(int64_t), cudaMemcpyDeviceToHost));
    fent.ensure(size_t(std::max<int64_t>(nadj, 1)));
    // cursors of the mirrored part: after each column's own entries
    std::vector<int64_t> hf(size_t(nv + 1));
    MFS_CUDA(cudaMemcpy(hf.data(), fptr.p, size_t(nv + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost));
    std::vector<int64_t> hb(size_t(std::max<int64_t>(nv, 1)));
    for (int64_t j = 0; j < nv; ++j) hb[size_t(j)] = hf[size_t(j)] + (S.A.Ap[size_t(j) + 1] - S.A.Ap[size_t(j)]);
    back.upload(hb, st);
    if (nv > 0) {
        mirror_fill_kernel<<<grid_of(nv, 128), 128, 0, st>>>(nv, Ap.p, Ai.p, fptr.p,
                                                             reinterpret_cast<unsigned long long *>(back.p), fent.p);
        MFS_LAUNCHED();
        mirror_sort_kernel<<<grid_of(nv, 128), 128, 0, st>>>(nv, Ap.p, fptr.p, fent.p);
        MFS_LAUNCHED();
    }
    PlanArgs a{nv, S.vb, Ap.p, Ai.p, src.p, fptr.p, fent.p, perm.p, iperm.p, sn_start.p, sptr.p, srows.p,
               w.p, f.p, pan.p, dp.p, dl.p, S.nsn};
    plan_ptr.ensure(size_t(2 * nv + 1));
    MFS_CUDA(cudaMemsetAsync(plan_ptr.p, 0, size_t(2 * nv + 1) * sizeof(int64_t), st));
    if (nv > 0) {
        plan_count_kernel<<<grid_of(nv, 128), 128, 0, st>>>(a, plan_ptr.p);
        MFS_LAUNCHED();
    }
    inclusive_scan(plan_ptr.p, 2 * nv + 1, st);
    int64_t nplan = 0;
    MFS_CUDA(cudaMemcpy(&nplan, plan_ptr.p + 2 * nv, sizeof(int64_t), cudaMemcpyDeviceToHost));
    plan_dev.ensure(size_t(std::max<int64_t>(nplan, 1)));
    plan_cat.ensure(size_t(std::max<int64_t>(nplan, 1)));
    DBuf<int> err;
    err.ensure(1);
    MFS_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), st));
    if (nv > 0) {
        plan_fill_kernel<<<grid_of(nv, 128), 128, 0, st>>>(a, plan_ptr.p, plan_cat.p, plan_dev.p, err.p);
        MFS_LAUNCHED();
    }
    int herr = 0;
    MFS_CUDA(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MFS_CUDA(cudaStreamSynchronize(st));
    if (herr) throw StatusError(MFS_INTERNAL, "GPU conversion plan: entry outside the factor structure");
    if (nplan != int64_t(S.plan.size()))
        throw StatusError(MFS_INTERNAL, "GPU conversion plan size differs from the analysis");
}

}  // namespace mfs
