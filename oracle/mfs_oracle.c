/*
 * CPU oracle for the MeshFEMSparse numeric path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker, never the product: it is loaded only by tests/,
 * __graft_entry__.smoke() and the CPU-baseline / reference legs of bench.py.
 * It restates, in plain C and independently of the GPU implementation:
 *
 *   orc_build_pattern   SystemAssembler<N>::blockSparsityPattern
 *                       (src/lib/MeshFEMSparse/SystemAssembler.hh:252-465)
 *   orc_assemble        ElementHessianContribAssembler<true>::run, sequential in
 *                       element order (SystemAssembler.hh:60-98; block add
 *                       BlockCSCHessian.hh:371-381; diagonal upper triangle :88-93)
 *   orc_symbolic        elimination structure by explicit symbolic elimination,
 *                       fundamental supernodes, relaxation restricted to contiguous
 *                       merges (the BlockCatamari symbolic stage called at
 *                       Solvers/CatamariFactorizer.cc:286,516 with relax_supernodes,
 *                       :105, and preserve_ordering for Native, :284)
 *   orc_inject          conversion-plan injection (CatamariConversionPlan.hh:524-525)
 *   orc_mf_factor       supernodal right-looking (multifrontal) Cholesky over the
 *                       given supernode partition (SparseLDL::RefactorWithFixedSparsityPattern,
 *                       called at CatamariFactorizer.cc:660; failure rule :701-705)
 *   orc_mf_solve        forward / backward substitution, multi-RHS column-major
 *                       (SparseLDL::Solve, CatamariFactorizer.cc:54,70); plain loops
 *                       for the checker, per-supernode TRSM / GEMM for the timed baseline
 *
 * Dense kernels optionally go through OpenBLAS (the copy bundled with scipy,
 * loaded with dlopen) so the oracle can double as the timed CPU baseline;
 * without it, plain loops are used.
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef int64_t i64;

/* ------------------------------------------------------------------ BLAS -- */
typedef void (*dgemm_t)(int, int, int, int, int, int, double, const double *, int, const double *, int, double,
                        double *, int);
typedef void (*dsyrk_t)(int, int, int, int, int, double, const double *, int, double, double *, int);
typedef void (*dtrsm_t)(int, int, int, int, int, int, int, double, const double *, int, double *, int);
typedef void (*dpotrf_t)(const char *, const int *, double *, const int *, int *);
typedef void (*setthreads_t)(int);

static dgemm_t p_dgemm;
static dsyrk_t p_dsyrk;
static dtrsm_t p_dtrsm;
static dpotrf_t p_dpotrf;
static setthreads_t p_setthreads;

enum { ColMajor = 102, NoTrans = 111, Trans = 112, Lower = 122, Left = 141, Right = 142, NonUnit = 131 };

int orc_blas_load(const char *path) {
    void *hdl = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!hdl) return 0;
    p_dgemm = (dgemm_t)dlsym(hdl, "scipy_cblas_dgemm");
    p_dsyrk = (dsyrk_t)dlsym(hdl, "scipy_cblas_dsyrk");
    p_dtrsm = (dtrsm_t)dlsym(hdl, "scipy_cblas_dtrsm");
    p_dpotrf = (dpotrf_t)dlsym(hdl, "scipy_dpotrf_");
    p_setthreads = (setthreads_t)dlsym(hdl, "scipy_openblas_set_num_threads");
    if (!p_dgemm || !p_dsyrk || !p_dtrsm || !p_dpotrf) {
        p_dgemm = 0; p_dsyrk = 0; p_dtrsm = 0; p_dpotrf = 0;
        return 0;
    }
    return 1;
}

int orc_blas_loaded(void) { return p_dpotrf != 0; }

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* --------------------------------------------------------------- pattern -- */
static int cmp_i64(const void *a, const void *b) {
    i64 x = *(const i64 *)a, y = *(const i64 *)b;
    return (x > y) - (x < y);
}

/* Upper block pattern: column j holds every i <= j sharing an element with j.
 * Returns nnz; Ai may be NULL (count only). */
i64 orc_build_pattern(i64 nvars, i64 nelem, int npe, const i64 *conn, i64 *Ap, i64 *Ai) {
    i64 *deg = calloc((size_t)nvars + 1, sizeof(i64));
    for (i64 e = 0; e < nelem; ++e)
        for (int a = 0; a < npe; ++a) deg[conn[e * npe + a]] += npe;
    i64 *start = malloc(((size_t)nvars + 1) * sizeof(i64));
    start[0] = 0;
    for (i64 j = 0; j < nvars; ++j) start[j + 1] = start[j] + deg[j];
    i64 *buf = malloc((size_t)(start[nvars] + 1) * sizeof(i64));
    i64 *fill = calloc((size_t)nvars, sizeof(i64));
    for (i64 e = 0; e < nelem; ++e)
        for (int b = 0; b < npe; ++b) {
            i64 j = conn[e * npe + b];
            for (int a = 0; a < npe; ++a) {
                i64 i = conn[e * npe + a];
                if (i <= j) buf[start[j] + fill[j]++] = i;
            }
        }
    i64 nnz = 0;
    Ap[0] = 0;
    for (i64 j = 0; j < nvars; ++j) {
        i64 *col = buf + start[j];
        qsort(col, (size_t)fill[j], sizeof(i64), cmp_i64);
        i64 u = 0;
        for (i64 k = 0; k < fill[j]; ++k)
            if (k == 0 || col[k] != col[k - 1]) {
                if (Ai) Ai[nnz + u] = col[k];
                ++u;
            }
        nnz += u;
        Ap[j + 1] = nnz;
    }
    free(deg); free(start); free(buf); free(fill);
    return nnz;
}

static i64 find_row(const i64 *Ap, const i64 *Ai, i64 j, i64 i) {
    for (i64 k = Ap[j]; k < Ap[j + 1]; ++k)
        if (Ai[k] == i) return k;
    return -1;
}

/* Sequential assembly of 4-node elements with 12x12 row-major element matrices
 * into the contiguous 3x3 block layout; Ax is overwritten. Returns -1 when an
 * element block is missing from the pattern, 0 on success. */
int orc_assemble(i64 nb, const i64 *Ap, const i64 *Ai, i64 nelem, const i64 *conn, const double *Ke, double *Ax) {
    memset(Ax, 0, (size_t)Ap[nb] * 9 * sizeof(double));
    for (i64 e = 0; e < nelem; ++e) {
        const i64 *v = conn + 4 * e;
        const double *K = Ke + 144 * e;
        int order[4] = {0, 1, 2, 3};
        for (int a = 1; a < 4; ++a)   /* stable insertion sort by global index */
            for (int b = a; b > 0 && v[order[b - 1]] > v[order[b]]; --b) {
                int t = order[b]; order[b] = order[b - 1]; order[b - 1] = t;
            }
        for (int jj = 0; jj < 4; ++jj) {
            int lj = order[jj];
            i64 bj = v[lj];
            for (int ii = 0; ii < jj; ++ii) {
                int li = order[ii];
                i64 k = find_row(Ap, Ai, bj, v[li]);
                if (k < 0) return -1;
                double *O = Ax + 9 * k;
                for (int c = 0; c < 3; ++c)
                    for (int r = 0; r < 3; ++r) {
                        if (li < lj) O[3 * c + r] += K[(3 * li + r) * 12 + 3 * lj + c];
                        else O[3 * c + r] += K[(3 * lj + c) * 12 + 3 * li + r];
                    }
            }
            i64 k = find_row(Ap, Ai, bj, bj);
            if (k < 0) return -1;
            double *O = Ax + 9 * k;
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r <= c; ++r) O[3 * c + r] += K[(3 * lj + r) * 12 + 3 * lj + c];
        }
    }
    return 0;
}

/* -------------------------------------------------------------- symbolic -- */
/* Explicit symbolic elimination on the permuted graph. Input: upper pattern over
 * nv analysis variables, iperm (new -> old). Output: parent (etree), cc (column
 * counts incl. diagonal), sn_start (relaxed supernodes; returns their count).
 * Relaxation: a supernode may absorb the child group that ends immediately
 * before it, if the explicit zeros of the merged supernode (scalar units, vb
 * scalars per variable) stay <= relax_zeros or <= relax_ratio of its entries. */
i64 orc_symbolic(i64 nv, const i64 *Ap, const i64 *Ai, const i64 *iperm, int vb, int relax, i64 relax_zeros,
                 double relax_ratio, i64 *parent, i64 *cc, i64 *sn_start, i64 *L_ptr, i64 *L_rows, i64 L_cap) {
    i64 *perm = malloc((size_t)nv * sizeof(i64));
    for (i64 k = 0; k < nv; ++k) perm[iperm[k]] = k;
    /* lower adjacency in permuted numbering: rows > j of column j */
    i64 *cnt = calloc((size_t)nv + 1, sizeof(i64));
    for (i64 j = 0; j < nv; ++j)
        for (i64 k = Ap[j]; k < Ap[j + 1]; ++k) {
            i64 i = Ai[k];
            if (i == j) continue;
            i64 a = perm[i], b = perm[j];
            cnt[(a < b ? a : b) + 1]++;
        }
    for (i64 j = 0; j < nv; ++j) cnt[j + 1] += cnt[j];
    i64 *rows = malloc((size_t)(cnt[nv] + 1) * sizeof(i64));
    i64 *fillp = calloc((size_t)nv, sizeof(i64));
    for (i64 j = 0; j < nv; ++j)
        for (i64 k = Ap[j]; k < Ap[j + 1]; ++k) {
            i64 i = Ai[k];
            if (i == j) continue;
            i64 a = perm[i], b = perm[j];
            i64 lo = a < b ? a : b, hi = a < b ? b : a;
            rows[cnt[lo] + fillp[lo]++] = hi;
        }
    /* L structure column by column: struct(j) = A rows U struct(children) \ {j} */
    i64 **Ls = calloc((size_t)nv, sizeof(i64 *));
    i64 *Ln = calloc((size_t)nv, sizeof(i64));
    i64 *mark = malloc((size_t)nv * sizeof(i64));
    for (i64 j = 0; j < nv; ++j) mark[j] = -1;
    i64 *tmp = malloc((size_t)nv * sizeof(i64));
    i64 *kids_head = malloc((size_t)nv * sizeof(i64));
    i64 *kids_next = malloc((size_t)nv * sizeof(i64));
    for (i64 j = 0; j < nv; ++j) kids_head[j] = -1;
    for (i64 j = 0; j < nv; ++j) {
        i64 t = 0;
        for (i64 k = cnt[j]; k < cnt[j + 1]; ++k) {
            i64 i = rows[k];
            if (mark[i] != j) { mark[i] = j; tmp[t++] = i; }
        }
        for (i64 c = kids_head[j]; c >= 0; c = kids_next[c])
            for (i64 k = 0; k < Ln[c]; ++k) {
                i64 i = Ls[c][k];
                if (i > j && mark[i] != j) { mark[i] = j; tmp[t++] = i; }
            }
        qsort(tmp, (size_t)t, sizeof(i64), cmp_i64);
        Ls[j] = malloc((size_t)(t + 1) * sizeof(i64));
        memcpy(Ls[j], tmp, (size_t)t * sizeof(i64));
        Ln[j] = t;
        parent[j] = t > 0 ? tmp[0] : -1;
        cc[j] = t + 1;
        if (parent[j] >= 0) { kids_next[j] = kids_head[parent[j]]; kids_head[parent[j]] = j; }
    }
    /* fundamental supernodes */
    i64 *nchild = calloc((size_t)nv, sizeof(i64));
    for (i64 j = 0; j < nv; ++j) if (parent[j] >= 0) nchild[parent[j]]++;
    i64 nf = 0;
    i64 *fs = malloc(((size_t)nv + 1) * sizeof(i64));
    for (i64 j = 0; j < nv; ++j) {
        int join = j > 0 && parent[j - 1] == j && cc[j - 1] == cc[j] + 1;
        if (!join) fs[nf++] = j;
    }
    fs[nf] = nv;
    /* relaxation over fundamental supernodes in column order */
    i64 *gfirst = malloc(((size_t)nf + 1) * sizeof(i64));
    i64 *gw = malloc(((size_t)nf + 1) * sizeof(i64));
    i64 *gd = malloc(((size_t)nf + 1) * sizeof(i64));
    double *gz = calloc((size_t)nf + 1, sizeof(double));
    char *absorbed = calloc((size_t)nf + 1, 1);
    i64 *fsn_of = malloc((size_t)nv * sizeof(i64) + 8);
    for (i64 s = 0; s < nf; ++s) {
        gfirst[s] = fs[s];
        gw[s] = fs[s + 1] - fs[s];
        gd[s] = cc[fs[s + 1] - 1] - 1;
        for (i64 j = fs[s]; j < fs[s + 1]; ++j) fsn_of[j] = s;
    }
    if (relax) {
        for (i64 s = 0; s < nf; ++s) {
            i64 pc = parent[fs[s + 1] - 1];
            if (pc < 0) continue;
            i64 p = fsn_of[pc];
            if (fs[s + 1] != gfirst[p]) continue;
            double w1 = (double)(vb * gw[s]), d1 = (double)(vb * gd[s]);
            double w2 = (double)(vb * gw[p]), d2 = (double)(vb * gd[p]);
            double merged = (w1 + w2) * (w1 + w2 + 1) / 2 + (w1 + w2) * d2;
            double z = gz[s] + gz[p] + merged - (w1 * (w1 + 1) / 2 + w1 * d1) - (w2 * (w2 + 1) / 2 + w2 * d2);
            if (z <= (double)relax_zeros || z <= relax_ratio * merged) {
                gfirst[p] = gfirst[s];
                gw[p] += gw[s];
                gz[p] = z;
                absorbed[s] = 1;
            }
        }
    }
    i64 nsn = 0;
    for (i64 j = 0; j < nv; ++j) {
        /* a final supernode starts at column j if j is the group start of an unabsorbed group */
        (void)j;
    }
    /* groups are contiguous column ranges [gfirst[s], fs[s+1]) for unabsorbed s, in column order */
    for (i64 s = 0; s < nf; ++s)
        if (!absorbed[s]) sn_start[nsn++] = gfirst[s];
    /* sort (they are already increasing because unabsorbed groups are disjoint ranges ordered by s) */
    qsort(sn_start, (size_t)nsn, sizeof(i64), cmp_i64);
    sn_start[nsn] = nv;
    /* optional: below-diagonal structure of every column of L (fundamental, before relaxation) */
    if (L_ptr) {
        L_ptr[0] = 0;
        for (i64 j = 0; j < nv; ++j) {
            L_ptr[j + 1] = L_ptr[j] + Ln[j];
            if (L_rows && L_ptr[j + 1] <= L_cap) memcpy(L_rows + L_ptr[j], Ls[j], (size_t)Ln[j] * sizeof(i64));
        }
    }
    for (i64 j = 0; j < nv; ++j) free(Ls[j]);
    free(Ls); free(Ln); free(mark); free(tmp); free(kids_head); free(kids_next); free(nchild); free(fs);
    free(gfirst); free(gw); free(gd); free(gz); free(absorbed); free(fsn_of); free(perm); free(cnt); free(rows);
    free(fillp);
    return nsn;
}

/* ------------------------------------------------------------- injection -- */
/* entries: 4 int64 per plan entry (dst, src, ld, flags); see the product's plan. */
void orc_inject(i64 nplan, const i64 *entries, int vb, int src_ld, const double *Ax, const double *Bx, double sigma_b,
                double *factor, i64 factor_size) {
    memset(factor, 0, (size_t)factor_size * sizeof(double));
    for (i64 e = 0; e < nplan; ++e) {
        i64 dst = entries[4 * e], src = entries[4 * e + 1], ld = entries[4 * e + 2], fl = entries[4 * e + 3];
        for (int c = 0; c < vb; ++c)
            for (int r = 0; r < vb; ++r) {
                if ((fl & 2) && r < c) continue;
                i64 so = (fl & 1) ? src + (i64)r * src_ld + c : src + (i64)c * src_ld + r;
                double v = Ax[so];
                if (Bx) v += sigma_b * Bx[so];
                factor[dst + (i64)c * ld + r] = v;
            }
    }
}

/* ------------------------------------------------------------- numeric --- */
typedef struct {
    i64 nsn;
    int vb;
    const i64 *sn_start, *parent, *struct_ptr, *struct_rows;
    i64 *w, *d, *f, *pan_off, *col0;
    i64 *level, nlevels, *level_ptr, *level_list;
    i64 *child_ptr, *child_list;
} Tree;

static void tree_build(Tree *T) {
    i64 nsn = T->nsn;
    T->w = malloc(((size_t)nsn + 1) * sizeof(i64));
    T->d = malloc(((size_t)nsn + 1) * sizeof(i64));
    T->f = malloc(((size_t)nsn + 1) * sizeof(i64));
    T->col0 = malloc(((size_t)nsn + 1) * sizeof(i64));
    T->pan_off = malloc(((size_t)nsn + 1) * sizeof(i64));
    T->pan_off[0] = 0;
    for (i64 s = 0; s < nsn; ++s) {
        T->w[s] = T->vb * (T->sn_start[s + 1] - T->sn_start[s]);
        T->d[s] = T->vb * (T->struct_ptr[s + 1] - T->struct_ptr[s]);
        T->f[s] = T->w[s] + T->d[s];
        T->col0[s] = T->vb * T->sn_start[s];
        T->pan_off[s + 1] = T->pan_off[s] + T->f[s] * T->w[s];
    }
    T->level = calloc((size_t)nsn + 1, sizeof(i64));
    T->nlevels = 0;
    for (i64 s = 0; s < nsn; ++s) {
        i64 p = T->parent[s];
        if (p >= 0 && T->level[p] < T->level[s] + 1) T->level[p] = T->level[s] + 1;
    }
    for (i64 s = 0; s < nsn; ++s) if (T->level[s] + 1 > T->nlevels) T->nlevels = T->level[s] + 1;
    T->level_ptr = calloc((size_t)T->nlevels + 2, sizeof(i64));
    for (i64 s = 0; s < nsn; ++s) T->level_ptr[T->level[s] + 1]++;
    for (i64 l = 0; l < T->nlevels; ++l) T->level_ptr[l + 1] += T->level_ptr[l];
    T->level_list = malloc(((size_t)nsn + 1) * sizeof(i64));
    i64 *back = malloc(((size_t)T->nlevels + 1) * sizeof(i64));
    for (i64 l = 0; l < T->nlevels; ++l) back[l] = T->level_ptr[l];
    for (i64 s = 0; s < nsn; ++s) T->level_list[back[T->level[s]]++] = s;
    free(back);
    T->child_ptr = calloc((size_t)nsn + 2, sizeof(i64));
    for (i64 s = 0; s < nsn; ++s) if (T->parent[s] >= 0) T->child_ptr[T->parent[s] + 1]++;
    for (i64 s = 0; s < nsn; ++s) T->child_ptr[s + 1] += T->child_ptr[s];
    T->child_list = malloc(((size_t)nsn + 1) * sizeof(i64));
    back = malloc(((size_t)nsn + 1) * sizeof(i64));
    for (i64 s = 0; s < nsn; ++s) back[s] = T->child_ptr[s];
    for (i64 s = 0; s < nsn; ++s) if (T->parent[s] >= 0) T->child_list[back[T->parent[s]]++] = s;
    free(back);
}

static void tree_free(Tree *T) {
    free(T->w); free(T->d); free(T->f); free(T->col0); free(T->pan_off); free(T->level); free(T->level_ptr);
    free(T->level_list); free(T->child_ptr); free(T->child_list);
}

/* scalar row of entry i of the (scalar) structure of supernode s */
static inline i64 struct_scalar(const Tree *T, i64 s, i64 i) {
    return T->struct_rows[T->struct_ptr[s] + i / T->vb] * T->vb + i % T->vb;
}

/* front position of global scalar row r inside supernode p (binary search) */
static i64 front_pos(const Tree *T, i64 p, i64 r) {
    if (r >= T->col0[p] && r < T->col0[p] + T->w[p]) return r - T->col0[p];
    i64 vr = r / T->vb, c = r % T->vb;
    i64 lo = T->struct_ptr[p], hi = T->struct_ptr[p + 1];
    while (lo < hi) {
        i64 mid = (lo + hi) / 2;
        if (T->struct_rows[mid] < vr) lo = mid + 1; else hi = mid;
    }
    if (lo >= T->struct_ptr[p + 1] || T->struct_rows[lo] != vr) return -1;
    return T->w[p] + (lo - T->struct_ptr[p]) * T->vb + c;
}

/* dense partial Cholesky of an f x f front (ld f): w pivots; returns the first failing pivot or -1 */
static i64 dense_partial(double *F, i64 f, i64 w, int use_blas) {
    i64 d = f - w;
    if (use_blas && p_dpotrf && w > 0) {
        int iw = (int)w, ld = (int)f, info = 0;
        p_dpotrf("L", &iw, F, &ld, &info);
        if (info > 0) return info - 1;
        if (d > 0) {
            p_dtrsm(ColMajor, Right, Lower, Trans, NonUnit, (int)d, (int)w, 1.0, F, (int)f, F + w, (int)f);
            p_dsyrk(ColMajor, Lower, NoTrans, (int)d, (int)w, -1.0, F + w, (int)f, 1.0, F + w * f + w, (int)f);
        }
        return -1;
    }
    for (i64 k = 0; k < w; ++k) {
        double *ck = F + k * f;
        double a = ck[k];
        if (!(a > 0)) return k;
        a = sqrt(a);
        ck[k] = a;
        for (i64 i = k + 1; i < f; ++i) ck[i] /= a;
        for (i64 j = k + 1; j < f; ++j) {
            double ljk = ck[j];
            double *cj = F + j * f;
            for (i64 i = j; i < f; ++i) cj[i] -= ck[i] * ljk;
        }
    }
    return -1;
}

/* Optional restriction to the supernodes [lo, hi] (a subtree in postorder is a
 * contiguous range): used to time a bounded sample of a large factorization. */
static i64 g_range_lo = 0, g_range_hi = -1;
void orc_set_range(i64 lo, i64 hi) {
    g_range_lo = lo;
    g_range_hi = hi;
}

/* Multifrontal factorization in place on injected panels (factor, catamari
 * layout). Returns -1 on success or the first failing scalar column. threads:
 * 0 = sequential without BLAS (pure oracle), >0 = level-parallel with BLAS. */
i64 orc_mf_factor(i64 nsn, int vb, const i64 *sn_start, const i64 *parent, const i64 *struct_ptr,
                  const i64 *struct_rows, double *factor, int threads) {
    Tree T = {0};
    T.nsn = nsn; T.vb = vb; T.sn_start = sn_start; T.parent = parent; T.struct_ptr = struct_ptr;
    T.struct_rows = struct_rows;
    tree_build(&T);
    double **U = calloc((size_t)nsn + 1, sizeof(double *));
    i64 fail = -1;
    const int use_blas = threads > 0 && p_dpotrf != 0;
    /* one dense front buffer per host thread, reused across fronts (grown on demand) */
    const int nbuf = threads > 0 ? threads : 1;
    double **ws = calloc((size_t)nbuf, sizeof(double *));
    size_t *wcap = calloc((size_t)nbuf, sizeof(size_t));
    /* Per level, two passes: fronts with more than kBigFront dense flops one after
     * another with all BLAS threads, then the rest concurrently with one BLAS thread
     * each (a large front on one thread would stall its level). */
    const double kBigFront = 2e9;
    for (i64 l = 0; l < T.nlevels; ++l)
    for (int pass = 0; pass < 2; ++pass) {
        i64 lo = T.level_ptr[l], hi = T.level_ptr[l + 1];
        int par = use_blas && pass == 1 && (hi - lo) >= 2;
        if (use_blas && p_setthreads) p_setthreads(par ? 1 : threads);
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(par ? threads : 1) if (par)
#endif
        for (i64 q = lo; q < hi; ++q) {
            i64 s = T.level_list[q];
            if (s < g_range_lo || (g_range_hi >= 0 && s > g_range_hi)) continue;
            {
                double fw = (double)T.w[s], fd = (double)T.d[s];
                if (use_blas) {
                    int big = (fw * fw * fw / 3 + fw * fw * fd + fw * fd * fd) > kBigFront;
                    if (big != (pass == 0)) continue;
                } else if (pass == 1) {
                    continue;                      /* the checker: one pass in level order */
                }
            }
            i64 w = T.w[s], d = T.d[s], f = T.f[s];
#ifdef _OPENMP
            int tid = par ? omp_get_thread_num() : 0;
#else
            int tid = 0;
#endif
            if ((size_t)(f * f) > wcap[tid]) {
                free(ws[tid]);
                ws[tid] = malloc((size_t)(f * f) * sizeof(double));
                wcap[tid] = (size_t)(f * f);
            }
            double *F = ws[tid];
            double *pan = factor + T.pan_off[s];
            /* the panel's w columns, then the lower triangle of the update block zeroed
             * (the only part the extend-add, SYRK and the update copy touch) */
            memcpy(F, pan, (size_t)(f * w) * sizeof(double));
            for (i64 j = w; j < f; ++j) memset(F + j * f + j, 0, (size_t)(f - j) * sizeof(double));
            for (i64 k = T.child_ptr[s]; k < T.child_ptr[s + 1]; ++k) {
                i64 c = T.child_list[k];
                i64 dc = T.d[c];
                i64 *pos = malloc((size_t)(dc + 1) * sizeof(i64));
                for (i64 i = 0; i < dc; ++i) pos[i] = front_pos(&T, s, struct_scalar(&T, c, i));
                /* columns of one child go to distinct front columns: with one front per
                 * level (the top of the tree) the host threads split them */
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads) if (use_blas && !par && dc > 512)
#endif
                for (i64 j = 0; j < dc; ++j)
                    for (i64 i = j; i < dc; ++i) F[pos[j] * f + pos[i]] += U[c][j * dc + i];
                free(pos);
                free(U[c]);
                U[c] = 0;
            }
            i64 bad = dense_partial(F, f, w, use_blas);
            if (bad >= 0) {
#ifdef _OPENMP
#pragma omp critical
#endif
                {
                    i64 col = T.col0[s] + bad;
                    if (fail < 0 || col < fail) fail = col;
                }
            }
            memcpy(pan, F, (size_t)(f * w) * sizeof(double));
            if (d > 0 && parent[s] >= 0) {
                U[s] = malloc((size_t)(d * d) * sizeof(double));
                for (i64 j = 0; j < d; ++j)
                    memcpy(U[s] + j * d + j, F + (w + j) * f + w + j, (size_t)(d - j) * sizeof(double));
            }
        }
    }
    for (int t = 0; t < nbuf; ++t) free(ws[t]);
    free(ws);
    free(wcap);
    for (i64 s = 0; s < nsn; ++s) free(U[s]);
    free(U);
    tree_free(&T);
    return fail;
}

/* Supernodal substitution with dense BLAS kernels per supernode (the timed CPU
 * baseline): forward  X[cols] = L11^{-1} X[cols], X[struct] -= L21 X[cols];
 * backward X[cols] -= L21^T X[struct], X[cols] = L11^{-T} X[cols]. */
static void mf_solve_blas(const Tree *T, const double *factor, double *X, i64 n, int nrhs, int threads) {
    if (p_setthreads) p_setthreads(threads);
    i64 dmax = 0;
    for (i64 s = 0; s < T->nsn; ++s) if (T->d[s] > dmax) dmax = T->d[s];
    double *tmp = malloc((size_t)(dmax * nrhs + 1) * sizeof(double));
    i64 *rows = malloc((size_t)(dmax + 1) * sizeof(i64));
    for (i64 s = 0; s < T->nsn; ++s) {
        if (s < g_range_lo || (g_range_hi >= 0 && s > g_range_hi)) continue;
        i64 w = T->w[s], d = T->d[s], f = T->f[s], c0 = T->col0[s];
        const double *pan = factor + T->pan_off[s];
        p_dtrsm(ColMajor, Left, Lower, NoTrans, NonUnit, (int)w, nrhs, 1.0, pan, (int)f, X + c0, (int)n);
        if (d > 0) {
            p_dgemm(ColMajor, NoTrans, NoTrans, (int)d, nrhs, (int)w, 1.0, pan + w, (int)f, X + c0, (int)n, 0.0, tmp,
                    (int)d);
            for (i64 i = 0; i < d; ++i) rows[i] = struct_scalar(T, s, i);
            for (int r = 0; r < nrhs; ++r)
                for (i64 i = 0; i < d; ++i) X[rows[i] + (i64)r * n] -= tmp[i + (i64)r * d];
        }
    }
    for (i64 s = T->nsn - 1; s >= 0; --s) {
        if (s < g_range_lo || (g_range_hi >= 0 && s > g_range_hi)) continue;
        i64 w = T->w[s], d = T->d[s], f = T->f[s], c0 = T->col0[s];
        const double *pan = factor + T->pan_off[s];
        if (d > 0) {
            for (i64 i = 0; i < d; ++i) rows[i] = struct_scalar(T, s, i);
            for (int r = 0; r < nrhs; ++r)
                for (i64 i = 0; i < d; ++i) tmp[i + (i64)r * d] = X[rows[i] + (i64)r * n];
            p_dgemm(ColMajor, Trans, NoTrans, (int)w, nrhs, (int)d, -1.0, pan + w, (int)f, tmp, (int)d, 1.0, X + c0,
                    (int)n);
        }
        p_dtrsm(ColMajor, Left, Lower, Trans, NonUnit, (int)w, nrhs, 1.0, pan, (int)f, X + c0, (int)n);
    }
    free(tmp);
    free(rows);
}

/* Forward then backward substitution on X (n x nrhs, ld n, permuted order).
 * threads > 0 with OpenBLAS loaded: the dense per-supernode form above;
 * otherwise plain loops (the checker). */
void orc_mf_solve(i64 nsn, int vb, const i64 *sn_start, const i64 *parent, const i64 *struct_ptr,
                  const i64 *struct_rows, const double *factor, double *X, i64 n, int nrhs, int threads) {
    Tree T = {0};
    T.nsn = nsn; T.vb = vb; T.sn_start = sn_start; T.parent = parent; T.struct_ptr = struct_ptr;
    T.struct_rows = struct_rows;
    tree_build(&T);
    if (threads > 0 && p_dpotrf) {
        mf_solve_blas(&T, factor, X, n, nrhs, threads);
        tree_free(&T);
        return;
    }
    /* forward: X[cols] = L11^{-1} X[cols]; X[struct] -= L21 X[cols] (sequential column order) */
    for (i64 s = 0; s < nsn; ++s) {
        if (s < g_range_lo || (g_range_hi >= 0 && s > g_range_hi)) continue;
        i64 w = T.w[s], d = T.d[s], f = T.f[s], c0 = T.col0[s];
        const double *pan = factor + T.pan_off[s];
        i64 *rows = malloc((size_t)(d + 1) * sizeof(i64));
        for (i64 i = 0; i < d; ++i) rows[i] = struct_scalar(&T, s, i);
        for (int r = 0; r < nrhs; ++r) {
            double *x = X + (i64)r * n;
            for (i64 k = 0; k < w; ++k) {
                const double *lk = pan + k * f;
                double xk = x[c0 + k] / lk[k];
                x[c0 + k] = xk;
                for (i64 i = k + 1; i < w; ++i) x[c0 + i] -= lk[i] * xk;
                for (i64 i = 0; i < d; ++i) x[rows[i]] -= lk[w + i] * xk;
            }
        }
        free(rows);
    }
    for (i64 s = nsn - 1; s >= 0; --s) {
        if (s < g_range_lo || (g_range_hi >= 0 && s > g_range_hi)) continue;
        i64 w = T.w[s], d = T.d[s], f = T.f[s], c0 = T.col0[s];
        const double *pan = factor + T.pan_off[s];
        i64 *rows = malloc((size_t)(d + 1) * sizeof(i64));
        for (i64 i = 0; i < d; ++i) rows[i] = struct_scalar(&T, s, i);
        for (int r = 0; r < nrhs; ++r) {
            double *x = X + (i64)r * n;
            for (i64 k = w - 1; k >= 0; --k) {
                const double *lk = pan + k * f;
                double acc = x[c0 + k];
                for (i64 i = k + 1; i < w; ++i) acc -= lk[i] * x[c0 + i];
                for (i64 i = 0; i < d; ++i) acc -= lk[w + i] * x[rows[i]];
                x[c0 + k] = acc / lk[k];
            }
        }
        free(rows);
    }
    tree_free(&T);
}
