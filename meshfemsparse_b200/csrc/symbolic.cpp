// Host symbolic analysis: pattern construction, pin removal, ordering,
// elimination tree, relaxed supernodes, factor layout, assembly-tree relative
// indices, level schedule, update-matrix memory plan, conversion plan and the
// symmetric SpMV structure.
//
// Reference steps restated here (file:line in the reference project):
//   block pattern from element stencils ........ SystemAssembler.hh:252-465
//   whole-block pin removal .................... CatamariFactorizer.cc:187-246,
//                                                CholeskyFactorizerBase.hh:402-426
//   partial-block pins -> scalar analysis ...... CatamariFactorizer.cc:208-216
//   full symmetric pattern for ordering ........ CatamariConverter.hh:47-146
//   ordering dispatch (ND / native / AMD) ...... CatamariFactorizer.cc:275-516
//   native ordering keeps the input order ...... CatamariFactorizer.cc:275-287
//   factor storage, compact row indices ........ CatamariConversionPlan.hh:366,
//                                                tests/test_catamari_factorizer.cc:299-343
//   child_rel_indices / num_child_diag_indices . tests/test_catamari_factorizer.cc:330-343
//   block conversion plan (two buckets/column) . CatamariConversionPlan.hh:402-541
//   factor nnz / flop estimate ................. CatamariFactorizer.cc:724-732
// The supernodal symbolic factorization itself (etree, column counts,
// fundamental and relaxed supernodes) lives in the external BlockCatamari
// library in the reference; it is restated from the published algorithms
// (Liu's elimination tree, row-subtree column counts, Ashcraft-Grimes style
// relaxation with catamari's allowance of 128 zeros or a 1% zero ratio) with
// merges restricted to a supernode and its immediately preceding child, so
// that relaxation never permutes columns.
#include "host_symbolic.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <stdexcept>
#include <string>

namespace mfs {

Pattern build_block_pattern(idx nvars, idx nelem, int npe, const idx *conn) {
    Pattern P;
    P.n = nvars;
    std::vector<idx> start(nvars + 1, 0);
    std::vector<idx> s(npe);
    for (idx e = 0; e < nelem; ++e) {
        for (int k = 0; k < npe; ++k) s[k] = conn[e * npe + k];
        std::sort(s.begin(), s.end());
        for (int k = 0; k < npe; ++k) {
            if (s[k] < 0 || s[k] >= nvars)
                throw std::invalid_argument("Stencil index exceeds the number of block variables");
            start[s[k] + 1] += k + 1;
        }
    }
    for (idx j = 0; j < nvars; ++j) start[j + 1] += start[j];
    std::vector<uint32_t> buckets(start[nvars]);
    std::vector<idx> back(start.begin(), start.end() - 1);
    for (idx e = 0; e < nelem; ++e) {
        for (int k = 0; k < npe; ++k) s[k] = conn[e * npe + k];
        std::sort(s.begin(), s.end());
        for (int b = 0; b < npe; ++b) {
            idx col = s[b];
            for (int a = 0; a <= b; ++a) buckets[back[col]++] = uint32_t(s[a]);
        }
    }
    P.Ap.assign(nvars + 1, 0);
    std::vector<idx> flag(nvars, -1);
    std::vector<idx> cnt(nvars, 0);
    for (idx j = 0; j < nvars; ++j) {
        uint32_t *b0 = buckets.data() + start[j], *b1 = buckets.data() + start[j + 1];
        uint32_t *out = b0;
        for (uint32_t *p = b0; p < b1; ++p) {
            if (flag[*p] != j) { flag[*p] = j; *out++ = *p; }
        }
        std::sort(b0, out);
        cnt[j] = out - b0;
    }
    for (idx j = 0; j < nvars; ++j) P.Ap[j + 1] = P.Ap[j] + cnt[j];
    P.Ai.resize(P.Ap[nvars]);
    for (idx j = 0; j < nvars; ++j)
        for (idx k = 0; k < cnt[j]; ++k) P.Ai[P.Ap[j] + k] = buckets[start[j] + k];
    return P;
}

namespace {

inline double entries_of(double w, double d) { return w * (w + 1) / 2 + w * d; }

// First-fit arena allocator used for the static update-matrix memory plan.
struct Arena {
    struct Block { idx off, size; };
    std::vector<Block> free_list;   // sorted by offset, coalesced
    idx top = 0;
    static idx align(idx x) { return (x + 63) & ~idx(63); }
    idx alloc(idx size) {
        size = align(std::max<idx>(size, 1));
        for (size_t k = 0; k < free_list.size(); ++k) {
            if (free_list[k].size >= size) {
                idx off = free_list[k].off;
                free_list[k].off += size;
                free_list[k].size -= size;
                if (free_list[k].size == 0) free_list.erase(free_list.begin() + k);
                return off;
            }
        }
        // extend the top (merging a trailing free block when present)
        if (!free_list.empty() && free_list.back().off + free_list.back().size == top) {
            idx off = free_list.back().off;
            free_list.pop_back();
            top = off + size;
            return off;
        }
        idx off = top;
        top += size;
        return off;
    }
    void release(idx off, idx size) {
        size = align(std::max<idx>(size, 1));
        Block b{off, size};
        auto it = std::lower_bound(free_list.begin(), free_list.end(), b,
                                   [](const Block &a, const Block &c) { return a.off < c.off; });
        it = free_list.insert(it, b);
        size_t k = size_t(it - free_list.begin());
        if (k + 1 < free_list.size() && free_list[k].off + free_list[k].size == free_list[k + 1].off) {
            free_list[k].size += free_list[k + 1].size;
            free_list.erase(free_list.begin() + k + 1);
        }
        if (k > 0 && free_list[k - 1].off + free_list[k - 1].size == free_list[k].off) {
            free_list[k - 1].size += free_list[k].size;
            free_list.erase(free_list.begin() + k);
        }
    }
};

}  // namespace

std::string analyze(idx nblocks, const idx *Ap, const idx *Ai, int bs, const idx *pinned, idx npinned,
                    const SymbolicOptions &opt, const idx *user_perm, Symbolic &S, const idx *user_sn_sizes,
                    idx n_user_sn) {
    S = Symbolic();
    if (bs < 1 || bs > 8) return "block size must be in [1, 8]";
    if (nblocks < 0) return "negative matrix size";
    if (Ap[0] != 0) return "Ap[0] must be 0";
    for (idx j = 0; j < nblocks; ++j) {
        if (Ap[j + 1] < Ap[j]) return "Ap must be non-decreasing";
        for (idx k = Ap[j]; k < Ap[j + 1]; ++k) {
            if (Ai[k] < 0 || Ai[k] > j) return "pattern must be upper triangular with rows in range";
            if (k > Ap[j] && Ai[k] <= Ai[k - 1]) return "row indices must be sorted and unique per column";
        }
    }
    S.bs = bs;
    S.n_full = idx(bs) * nblocks;

    // ---- pins: scalar -> sorted unique; detect partially pinned blocks.
    std::vector<char> scalar_fixed(S.n_full, 0);
    for (idx k = 0; k < npinned; ++k) {
        idx v = pinned[k];
        if (v < 0 || v >= S.n_full) return "Fixed variable index out of range";
        if (!scalar_fixed[v]) { scalar_fixed[v] = 1; S.fixed_vars.push_back(v); }
    }
    std::sort(S.fixed_vars.begin(), S.fixed_vars.end());
    bool partial = false;
    if (bs > 1) {
        for (idx b = 0; b < nblocks && !partial; ++b) {
            int c = 0;
            for (int r = 0; r < bs; ++r) c += scalar_fixed[b * bs + r];
            if (c != 0 && c != bs) partial = true;
        }
    }
    const int vb = partial ? 1 : bs;
    S.vb = vb;
    S.src_ld = bs;
    const idx nv_full = S.n_full / vb;
    S.nv_full = nv_full;

    // ---- analysis pattern over nv_full variables with Ax source offsets.
    Pattern P;
    std::vector<idx> src;
    if (vb == bs) {
        P.n = nblocks;
        P.Ap.assign(Ap, Ap + nblocks + 1);
        P.Ai.assign(Ai, Ai + Ap[nblocks]);
        src.resize(P.Ai.size());
        for (size_t k = 0; k < src.size(); ++k) src[k] = idx(k) * bs * bs;
    } else {
        // Scalar expansion of the contiguous-block layout (the reference's
        // toScalar + dataOffsetsForScalarCSCDataOffsets, BlockCSCHessian.hh).
        P.n = S.n_full;
        P.Ap.assign(P.n + 1, 0);
        for (idx bj = 0; bj < nblocks; ++bj) {
            for (int c = 0; c < bs; ++c) {
                idx j = bj * bs + c;
                for (idx k = Ap[bj]; k < Ap[bj + 1]; ++k) {
                    idx bi = Ai[k];
                    int rmax = (bi == bj) ? c : bs - 1;
                    for (int r = 0; r <= rmax; ++r) {
                        P.Ai.push_back(bi * bs + r);
                        src.push_back(k * bs * bs + idx(c) * bs + r);
                    }
                }
                P.Ap[j + 1] = idx(P.Ai.size());
            }
        }
    }

    // ---- row/column removal at analysis granularity.
    std::vector<idx> rr(nv_full, 0);
    {
        idx next = 0;
        for (idx v = 0; v < nv_full; ++v) {
            bool fixed = scalar_fixed[v * vb] != 0;
            rr[v] = fixed ? -1 : next++;
        }
        S.nv = next;
    }
    const idx nv = S.nv;
    S.n = nv * vb;
    S.A.n = nv;
    S.A.Ap.assign(nv + 1, 0);
    for (idx j = 0; j < nv_full; ++j) {
        if (rr[j] < 0) continue;
        for (idx k = P.Ap[j]; k < P.Ap[j + 1]; ++k) {
            if (rr[P.Ai[k]] < 0) continue;
            S.A.Ai.push_back(rr[P.Ai[k]]);
            S.src_off.push_back(src[k]);
        }
        S.A.Ap[rr[j] + 1] = idx(S.A.Ai.size());
    }
    S.reduced_row_for_row.assign(S.n_full, -1);
    for (idx v = 0; v < nv_full; ++v)
        if (rr[v] >= 0)
            for (int c = 0; c < vb; ++c) S.reduced_row_for_row[v * vb + c] = rr[v] * vb + c;

    // ---- full symmetric adjacency (with the entry index of every pair).
    std::vector<idx> fptr(nv + 1, 0), fadj, fent;
    for (idx j = 0; j < nv; ++j)
        for (idx k = S.A.Ap[j]; k < S.A.Ap[j + 1]; ++k) {
            idx i = S.A.Ai[k];
            fptr[j + 1]++;
            if (i != j) fptr[i + 1]++;
        }
    for (idx j = 0; j < nv; ++j) fptr[j + 1] += fptr[j];
    fadj.resize(fptr[nv]); fent.resize(fptr[nv]);
    {
        std::vector<idx> back(fptr.begin(), fptr.end() - 1);
        for (idx j = 0; j < nv; ++j)
            for (idx k = S.A.Ap[j]; k < S.A.Ap[j + 1]; ++k) {
                idx i = S.A.Ai[k];
                fadj[back[j]] = i; fent[back[j]++] = k;
                if (i != j) { fadj[back[i]] = j; fent[back[i]++] = k; }
            }
    }
    std::vector<idx> gx(nv + 1, 0), ga;   // graph without self loops
    for (idx j = 0; j < nv; ++j) {
        for (idx k = fptr[j]; k < fptr[j + 1]; ++k) if (fadj[k] != j) ga.push_back(fadj[k]);
        gx[j + 1] = idx(ga.size());
    }

    // ---- ordering
    std::vector<idx> iperm(nv);
    bool postorder = true;
    if (opt.ordering == ORDER_NATIVE) {
        std::iota(iperm.begin(), iperm.end(), 0);
        postorder = false;
    } else if (opt.ordering == ORDER_USER) {
        if (!user_perm) return "user ordering requested without a permutation";
        // user_perm is new -> old over reduced analysis variables
        std::vector<char> seen(nv, 0);
        for (idx k = 0; k < nv; ++k) {
            idx v = user_perm[k];
            if (v < 0 || v >= nv || seen[v]) return "user permutation is not a permutation of the reduced variables";
            seen[v] = 1;
            iperm[k] = v;
        }
        postorder = false;
    } else if (opt.ordering == ORDER_MD) {
        iperm = minimum_degree(nv, gx, ga);
    } else {
        idx rebuilt = -1;
        NDResult nd = opt.nd_prev ? nested_dissection_reuse(nv, gx, ga, *opt.nd_prev, opt.nd, &rebuilt)
                                  : nested_dissection(nv, gx, ga, opt.nd);
        const int cut = camd_cut_depth_from_env();
        if (cut >= 0) nd.iperm = hierarchical_constrained_md(nv, gx, ga, nd, cut);
        iperm = nd.iperm;
        S.nd_cparent = nd.cparent;
        S.nd_cmember = nd.cmember;
        S.nd_ncomp = nd.ncomp;
        S.nd_rebuilt = rebuilt;
    }
    std::vector<idx> perm(nv);
    for (idx k = 0; k < nv; ++k) perm[iperm[k]] = k;

    // ---- elimination tree (Liu) on the permuted pattern
    std::vector<idx> parent(nv, -1), anc(nv, -1);
    for (idx j = 0; j < nv; ++j) {
        idx oj = iperm[j];
        for (idx k = gx[oj]; k < gx[oj + 1]; ++k) {
            idx i = perm[ga[k]];
            if (i >= j) continue;
            while (i != -1 && i < j) {
                idx nxt = anc[i];
                anc[i] = j;
                if (nxt == -1) parent[i] = j;
                i = nxt;
            }
        }
    }
    if (postorder) {
        // depth-first postorder, children visited in increasing order
        std::vector<idx> head(nv, -1), nextc(nv, -1);
        for (idx j = nv - 1; j >= 0; --j) {
            if (parent[j] >= 0) { nextc[j] = head[parent[j]]; head[parent[j]] = j; }
        }
        std::vector<idx> post; post.reserve(nv);
        std::vector<idx> stack;
        for (idx r = 0; r < nv; ++r) {
            if (parent[r] != -1) continue;
            stack.push_back(r);
            while (!stack.empty()) {
                idx p = stack.back();
                idx c = head[p];
                if (c == -1) { stack.pop_back(); post.push_back(p); }
                else { head[p] = nextc[c]; stack.push_back(c); }
            }
        }
        std::vector<idx> ipost(nv);
        for (idx k = 0; k < nv; ++k) ipost[post[k]] = k;
        std::vector<idx> iperm2(nv), parent2(nv);
        for (idx k = 0; k < nv; ++k) {
            iperm2[k] = iperm[post[k]];
            idx p = parent[post[k]];
            parent2[k] = p < 0 ? -1 : ipost[p];
        }
        iperm.swap(iperm2);
        parent.swap(parent2);
        for (idx k = 0; k < nv; ++k) perm[iperm[k]] = k;
    }
    S.perm = perm;
    S.iperm = iperm;

    // ---- column counts (row-subtree traversal), including the diagonal
    std::vector<idx> cc(nv, 1), mark(nv, -1), nchild(nv, 0);
    for (idx j = 0; j < nv; ++j) if (parent[j] >= 0) nchild[parent[j]]++;
    for (idx i = 0; i < nv; ++i) {
        mark[i] = i;
        idx oi = iperm[i];
        for (idx k = gx[oi]; k < gx[oi + 1]; ++k) {
            idx j = perm[ga[k]];
            if (j >= i) continue;
            while (j != -1 && j < i && mark[j] != i) {
                mark[j] = i;
                cc[j]++;
                j = parent[j];
            }
        }
    }

    // ---- fundamental supernodes
    std::vector<idx> fstart{0};
    // Column j+1 continues j's supernode when it is j's parent and the column
    // structures nest exactly (no single-child requirement: the reference's
    // native-ordering known answer, tests/test_native_ordering.cc:141, needs
    // the two-child column pair {3,4} of its example to form one supernode).
    (void)nchild;
    for (idx j = 0; j + 1 < nv; ++j) {
        bool join = parent[j] == j + 1 && cc[j] == cc[j + 1] + 1;
        if (!join) fstart.push_back(j + 1);
    }
    if (nv > 0) fstart.push_back(nv);
    else fstart.assign(1, 0);
    const idx nf = idx(fstart.size()) - 1;
    std::vector<idx> fsn_of(nv);
    for (idx s = 0; s < nf; ++s) for (idx j = fstart[s]; j < fstart[s + 1]; ++j) fsn_of[j] = s;
    std::vector<idx> fparent(nf, -1);
    for (idx s = 0; s < nf; ++s) {
        idx p = parent[fstart[s + 1] - 1];
        fparent[s] = p < 0 ? -1 : fsn_of[p];
    }

    // ---- relaxation: merge a group into its parent when it ends right
    // before the parent's group starts and the explicit-zero allowance holds.
    std::vector<idx> gfirst(nf), gw(nf), gd(nf), absorbed(nf, -1);
    std::vector<double> gz(nf, 0.0);
    for (idx s = 0; s < nf; ++s) {
        gfirst[s] = fstart[s];
        gw[s] = fstart[s + 1] - fstart[s];
        gd[s] = cc[fstart[s + 1] - 1] - 1;
    }
    if (user_sn_sizes) {
        // Caller-supplied partition (the reference's ordering.supernode_sizes,
        // CatamariFactorizer.cc:311-324): each supernode must be an etree chain.
        if (opt.ordering != ORDER_NATIVE && opt.ordering != ORDER_USER)
            return "a supernode partition can only be supplied with the native or user ordering";
        idx tot = 0;
        for (idx t = 0; t < n_user_sn; ++t) {
            if (user_sn_sizes[t] <= 0) return "supernode sizes must be positive";
            for (idx j = tot; j + 1 < tot + user_sn_sizes[t]; ++j)
                if (j + 1 >= nv || parent[j] != j + 1) return "supplied supernode is not a chain of the elimination tree";
            tot += user_sn_sizes[t];
        }
        if (tot != nv) return "supernode sizes must sum to the number of reduced variables";
        fstart.assign(1, 0);
        for (idx t = 0; t < n_user_sn; ++t) fstart.push_back(fstart.back() + user_sn_sizes[t]);
    }
    const idx nf2 = idx(fstart.size()) - 1;
    if (user_sn_sizes) {
        gfirst.assign(nf2, 0); gw.assign(nf2, 0); gd.assign(nf2, 0); absorbed.assign(nf2, -1); gz.assign(nf2, 0.0);
        for (idx s = 0; s < nf2; ++s) {
            gfirst[s] = fstart[s];
            gw[s] = fstart[s + 1] - fstart[s];
        }
    }
    if (opt.relax && !user_sn_sizes) {
        for (idx s = 0; s < nf; ++s) {
            idx p = fparent[s];
            if (p < 0) continue;
            if (fstart[s + 1] != gfirst[p]) continue;
            double w1 = double(vb * gw[s]), d1 = double(vb * gd[s]);
            double w2 = double(vb * gw[p]), d2 = double(vb * gd[p]);
            double merged = entries_of(w1 + w2, d2);
            double z = gz[s] + gz[p] + (merged - entries_of(w1, d1) - entries_of(w2, d2));
            if (z <= double(opt.relax_zeros) || z <= opt.relax_ratio * merged) {
                gfirst[p] = gfirst[s];
                gw[p] += gw[s];
                gz[p] = z;
                absorbed[s] = p;
            }
        }
    }
    // final supernodes: the groups that were not absorbed, in column order
    std::vector<idx> sn_of(nv, -1);
    S.sn_start.clear();
    {
        std::vector<idx> reps;
        for (idx s = 0; s < nf2; ++s) if (absorbed[s] < 0) reps.push_back(s);
        std::sort(reps.begin(), reps.end(), [&](idx a, idx b) { return gfirst[a] < gfirst[b]; });
        S.nsn = idx(reps.size());
        S.sn_start.resize(S.nsn + 1);
        for (idx t = 0; t < S.nsn; ++t) {
            S.sn_start[t] = gfirst[reps[t]];
            for (idx j = gfirst[reps[t]]; j < fstart[reps[t] + 1]; ++j) sn_of[j] = t;
        }
        S.sn_start[S.nsn] = nv;
    }
    const idx nsn = S.nsn;
    for (idx j = 0; j < nv; ++j) if (sn_of[j] < 0) return "internal error: column without supernode";
    S.sn_parent.assign(nsn, -1);
    for (idx s = 0; s < nsn; ++s) {
        idx p = parent[S.sn_start[s + 1] - 1];
        S.sn_parent[s] = p < 0 ? -1 : sn_of[p];
        if (S.sn_parent[s] >= 0 && S.sn_parent[s] <= s) return "internal error: supernode tree not topological";
    }
    S.child_ptr.assign(nsn + 1, 0);
    for (idx s = 0; s < nsn; ++s) if (S.sn_parent[s] >= 0) S.child_ptr[S.sn_parent[s] + 1]++;
    for (idx s = 0; s < nsn; ++s) S.child_ptr[s + 1] += S.child_ptr[s];
    S.child_list.resize(S.child_ptr[nsn]);
    {
        std::vector<idx> back(S.child_ptr.begin(), S.child_ptr.end() - 1);
        for (idx s = 0; s < nsn; ++s) if (S.sn_parent[s] >= 0) S.child_list[back[S.sn_parent[s]]++] = s;
    }

    // ---- supernode row structures
    S.struct_ptr.assign(nsn + 1, 0);
    S.struct_rows.clear();
    {
        std::vector<idx> flag(nv, -1), rows;
        for (idx s = 0; s < nsn; ++s) {
            rows.clear();
            const idx last = S.sn_start[s + 1] - 1;
            for (idx j = S.sn_start[s]; j <= last; ++j) {
                idx oj = iperm[j];
                for (idx k = gx[oj]; k < gx[oj + 1]; ++k) {
                    idx i = perm[ga[k]];
                    if (i > last && flag[i] != s) { flag[i] = s; rows.push_back(i); }
                }
            }
            for (idx k = S.child_ptr[s]; k < S.child_ptr[s + 1]; ++k) {
                idx c = S.child_list[k];
                for (idx t = S.struct_ptr[c]; t < S.struct_ptr[c + 1]; ++t) {
                    idx i = S.struct_rows[t];
                    if (i > last && flag[i] != s) { flag[i] = s; rows.push_back(i); }
                }
            }
            std::sort(rows.begin(), rows.end());
            S.struct_rows.insert(S.struct_rows.end(), rows.begin(), rows.end());
            S.struct_ptr[s + 1] = idx(S.struct_rows.size());
        }
    }

    // ---- scalar layout, nnz and flop estimates
    S.w.resize(nsn); S.d.resize(nsn); S.f.resize(nsn); S.pan_off.resize(nsn + 1);
    S.pan_off[0] = 0;
    S.factor_nnz = 0;
    S.flops = 0;
    for (idx s = 0; s < nsn; ++s) {
        S.w[s] = vb * (S.sn_start[s + 1] - S.sn_start[s]);
        S.d[s] = vb * (S.struct_ptr[s + 1] - S.struct_ptr[s]);
        S.f[s] = S.w[s] + S.d[s];
        S.pan_off[s + 1] = S.pan_off[s] + S.f[s] * S.w[s];
        double w = double(S.w[s]), d = double(S.d[s]);
        S.factor_nnz += S.w[s] * (S.w[s] + 1) / 2 + S.w[s] * S.d[s];
        S.flops += w * w * w / 3.0 + w * w * d + w * d * d;
    }
    S.factor_size = S.pan_off[nsn];

    // ---- relative indices of every child's structure inside its parent's front
    S.rel.assign(S.struct_rows.size(), 0);
    S.num_child_diag.assign(nsn, 0);
    for (idx c = 0; c < nsn; ++c) {
        idx p = S.sn_parent[c];
        if (p < 0) continue;
        const idx *pb = S.struct_rows.data() + S.struct_ptr[p];
        const idx *pe = S.struct_rows.data() + S.struct_ptr[p + 1];
        idx ndiag = 0;
        for (idx t = S.struct_ptr[c]; t < S.struct_ptr[c + 1]; ++t) {
            idx r = S.struct_rows[t];
            if (r >= S.sn_start[p] && r < S.sn_start[p + 1]) {
                S.rel[t] = int32_t(vb * (r - S.sn_start[p]));
                ++ndiag;
            } else {
                const idx *it = std::lower_bound(pb, pe, r);
                if (it == pe || *it != r) return "internal error: child structure not contained in parent";
                S.rel[t] = int32_t(S.w[p] + vb * (it - pb));
            }
        }
        S.num_child_diag[c] = vb * ndiag;
    }

    // ---- level schedule
    S.level.assign(nsn, 0);
    for (idx s = 0; s < nsn; ++s) {
        idx p = S.sn_parent[s];
        if (p >= 0) S.level[p] = std::max(S.level[p], S.level[s] + 1);
    }
    S.nlevels = 0;
    for (idx s = 0; s < nsn; ++s) S.nlevels = std::max<idx>(S.nlevels, S.level[s] + 1);
    S.level_ptr.assign(S.nlevels + 1, 0);
    for (idx s = 0; s < nsn; ++s) S.level_ptr[S.level[s] + 1]++;
    for (idx l = 0; l < S.nlevels; ++l) S.level_ptr[l + 1] += S.level_ptr[l];
    S.level_list.resize(nsn);
    {
        std::vector<idx> back(S.level_ptr.begin(), S.level_ptr.end() - 1);
        for (idx s = 0; s < nsn; ++s) S.level_list[back[S.level[s]]++] = s;
    }

    // ---- static memory plan for update matrices
    auto plan_arena = [&](bool square, std::vector<idx> &off, idx &total) {
        off.assign(nsn, -1);
        Arena arena;
        // free at the start of level h every buffer whose parent sits at level < h
        std::vector<std::vector<idx>> release_at(S.nlevels + 1);
        for (idx l = 0; l < S.nlevels; ++l) {
            for (idx s : release_at[l]) arena.release(off[s], square ? S.d[s] * S.d[s] : S.d[s]);
            for (idx k = S.level_ptr[l]; k < S.level_ptr[l + 1]; ++k) {
                idx s = S.level_list[k];
                if (S.d[s] == 0 || S.sn_parent[s] < 0) continue;
                off[s] = arena.alloc(square ? S.d[s] * S.d[s] : S.d[s]);
                release_at[S.level[S.sn_parent[s]] + 1].push_back(s);
            }
        }
        total = arena.top;
    };
    plan_arena(true, S.upd_off, S.upd_size);

    // ---- subtree solve cut: the highest level whose subtrees are many and small
    // (fronts <= kSubFmax rows). One CTA walks a subtree sequentially, so the
    // largest subtree bounds the phase: aim for kManySubtrees (16 per SM of a
    // 148-SM B200, the measured optimum on the 811k-DOF cube; for a forest of many
    // independent meshes 48 per tree, measured on a batch of 256: the solve 103.5 ->
    // 87.9 ms against 2368), else settle for kMinSubtrees (one per SM).
    {
        idx nroots = 0;
        for (idx s = 0; s < nsn; ++s) nroots += S.sn_parent[s] < 0 ? 1 : 0;
        const idx kManySubtrees = opt.solve_subtrees > 0 ? opt.solve_subtrees : std::max<idx>(2368, 48 * nroots);
        constexpr idx kMinSubtrees = 148, kSubFmax = 2048;
        S.solve_cut = -1;
        std::vector<idx> fmax_le(S.nlevels, 0);           // max front at levels <= l
        for (idx s = 0; s < nsn; ++s) fmax_le[S.level[s]] = std::max(fmax_le[S.level[s]], S.f[s]);
        for (idx l = 1; l < S.nlevels; ++l) fmax_le[l] = std::max(fmax_le[l], fmax_le[l - 1]);
        std::vector<idx> roots_at(S.nlevels, 0);           // subtree count for a cut at level l
        for (idx s = 0; s < nsn; ++s)
            for (idx l = S.level[s]; l < (S.sn_parent[s] < 0 ? S.nlevels : S.level[S.sn_parent[s]]); ++l)
                ++roots_at[l];
        for (idx want : {kManySubtrees, kMinSubtrees}) {
            for (idx l = S.nlevels - 2; l >= 0; --l) {
                if (fmax_le[l] > kSubFmax || roots_at[l] < want) continue;
                S.solve_cut = l;
                S.sub_fmax = fmax_le[l];
                break;
            }
            if (S.solve_cut >= 0) break;
        }
        if (S.solve_cut >= 0) {
            // subtree of root s = [s - size(s) + 1, s] in postorder
            std::vector<idx> size(nsn, 1);
            for (idx s = 0; s < nsn; ++s)
                if (S.sn_parent[s] >= 0) size[S.sn_parent[s]] += size[s];
            std::vector<std::pair<double, idx>> work;
            for (idx s = 0; s < nsn; ++s) {
                if (S.level[s] > S.solve_cut) continue;
                if (S.sn_parent[s] >= 0 && S.level[S.sn_parent[s]] <= S.solve_cut) continue;
                double wk = 0;
                for (idx t = s - size[s] + 1; t <= s; ++t) wk += double(S.f[t]) * double(S.w[t]);
                work.push_back({wk, s});
            }
            std::sort(work.begin(), work.end(), [](const auto &a, const auto &b) {
                return a.first > b.first || (a.first == b.first && a.second < b.second);
            });
            for (const auto &pw : work) {
                S.sub_lo.push_back(pw.second - size[pw.second] + 1);
                S.sub_hi.push_back(pw.second);
            }
        }
    }
    // ---- solve arena: as the update arena, except that subtree supernodes are
    // allocated up front and kept at least until the levels above the cut
    {
        S.sol_off.assign(nsn, -1);
        Arena arena;
        std::vector<std::vector<idx>> release_at(S.nlevels + 2);
        auto alloc_level = [&](idx s) { return S.level[s] <= S.solve_cut ? 0 : idx(S.level[s]); };
        for (idx l = 0; l < S.nlevels; ++l) {
            for (idx s : release_at[l]) arena.release(S.sol_off[s], S.d[s]);
            for (idx s = 0; s < nsn; ++s) {
                if (alloc_level(s) != l || S.d[s] == 0 || S.sn_parent[s] < 0) continue;
                S.sol_off[s] = arena.alloc(S.d[s]);
                release_at[std::max<idx>(S.level[S.sn_parent[s]] + 1, S.solve_cut + 1)].push_back(s);
            }
        }
        S.sol_size = arena.top;
    }

    // ---- conversion plan
    S.plan_ptr.assign(2 * nv + 1, 0);
    for (idx j = 0; j < nv; ++j) {
        idx oj = iperm[j];
        for (idx k = fptr[oj]; k < fptr[oj + 1]; ++k) {
            idx oi = fadj[k];
            if (perm[oi] < j) continue;
            if (oi >= oj) S.plan_ptr[2 * j + 1]++;
            else S.plan_ptr[2 * j + 2]++;
        }
    }
    for (idx b = 0; b < 2 * nv; ++b) S.plan_ptr[b + 1] += S.plan_ptr[b];
    S.plan.resize(S.plan_ptr[2 * nv]);
    {
        std::vector<idx> back(S.plan_ptr.begin(), S.plan_ptr.end() - 1);
        for (idx j = 0; j < nv; ++j) {
            idx oj = iperm[j];
            idx s = sn_of[j];
            idx jr = vb * (j - S.sn_start[s]);
            const idx *pb = S.struct_rows.data() + S.struct_ptr[s];
            const idx *pe = S.struct_rows.data() + S.struct_ptr[s + 1];
            for (idx k = fptr[oj]; k < fptr[oj + 1]; ++k) {
                idx oi = fadj[k];
                idx i = perm[oi];
                if (i < j) continue;
                idx ir;
                if (i < S.sn_start[s + 1]) ir = vb * (i - S.sn_start[s]);
                else {
                    const idx *it = std::lower_bound(pb, pe, i);
                    if (it == pe || *it != i) return "internal error: plan entry outside the factor structure";
                    ir = S.w[s] + vb * (it - pb);
                }
                PlanEntry e;
                e.dst = S.pan_off[s] + jr * S.f[s] + ir;
                e.src = S.src_off[fent[k]];
                e.ld = int32_t(S.f[s]);
                e.flags = (oi >= oj ? 1 : 0) | (i == j ? 2 : 0);
                idx bucket = oi >= oj ? 2 * j : 2 * j + 1;
                S.plan[back[bucket]++] = e;
            }
        }
    }

    // ---- symmetric SpMV structure over permuted rows
    S.spmv_ptr.assign(nv + 1, 0);
    for (idx i = 0; i < nv; ++i) S.spmv_ptr[i + 1] = S.spmv_ptr[i] + (fptr[iperm[i] + 1] - fptr[iperm[i]]);
    S.spmv_src.resize(S.spmv_ptr[nv]);
    S.spmv_col.resize(S.spmv_ptr[nv]);
    S.spmv_flag.resize(S.spmv_ptr[nv]);
    {
        std::vector<std::pair<idx, idx>> row;
        for (idx i = 0; i < nv; ++i) {
            idx oi = iperm[i];
            row.clear();
            for (idx k = fptr[oi]; k < fptr[oi + 1]; ++k) row.push_back({perm[fadj[k]], k});
            std::sort(row.begin(), row.end());
            idx o = S.spmv_ptr[i];
            for (auto &pr : row) {
                idx k = pr.second;
                idx oj = fadj[k];
                S.spmv_src[o] = S.src_off[fent[k]];
                S.spmv_col[o] = int32_t(pr.first);
                S.spmv_flag[o] = (oi > oj ? 1 : 0) | (oi == oj ? 2 : 0);
                ++o;
            }
        }
    }

    // ---- scalar permutations and the fused pin+permutation map
    S.scalar_perm.resize(S.n);
    S.scalar_iperm.resize(S.n);
    for (idx v = 0; v < nv; ++v)
        for (int c = 0; c < vb; ++c) {
            S.scalar_perm[v * vb + c] = perm[v] * vb + c;
            S.scalar_iperm[v * vb + c] = iperm[v] * vb + c;
        }
    S.permuted_reduced_row_for_row.assign(S.n_full, -1);
    for (idx r = 0; r < S.n_full; ++r) {
        idx q = S.reduced_row_for_row[r];
        if (q >= 0) S.permuted_reduced_row_for_row[r] = S.scalar_perm[q];
    }
    return std::string();
}

}  // namespace mfs
