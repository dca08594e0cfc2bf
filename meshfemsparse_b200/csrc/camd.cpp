// Final ordering of a nested dissection: constrained minimum degree over the
// separator forest, split hierarchically at a cut depth.
//
// The reference orders the vertices of its separator forest with CAMD
// (constrained approximate minimum degree, SuiteSparse; not part of the
// reference tree), one call per subtree rooted at the cut depth (default 4) plus
// one call for the separators above it (Solvers/ParallelNestedDissection/
// hierarchical_camd.cc:165-333, hierarchical_camd.md). This file restates that
// structure with its own minimum-degree engine:
//   * constraint sets are the forest's components; a component's vertices are
//     eliminated after every vertex of a lower-numbered (postorder) component of
//     the same problem, so descendants precede ancestors and every component stays
//     contiguous;
//   * inside a constraint set the next pivot is the vertex of least approximate
//     external degree on a quotient graph (variables, and elements = cliques of
//     eliminated vertices), with AMD's degree bound and element absorption;
//     ties go to the lower vertex id, so the order is deterministic; variables
//     left adjacent to nothing but the new element are simplicial and are
//     eliminated with the pivot (mass elimination, no fill);
//   * the subtrees below the cut are independent problems (no edge joins two of
//     them) and run on separate host threads; the upper vertices next to a subtree
//     are kept in its problem as a halo that is never eliminated, so degrees count
//     the separators the subtree's vertices touch (the reference's local problems
//     omit them; with the halo the fill stays within 1% of the dissection's own
//     order on cubes of side 6-64, without it small cubes lost 3.5%); each connected part of a subtree
//     leaves the separators above it one clique, which enters the upper problem as
//     an initial element, so the upper ordering sees the fill the subtrees make.
// Exact AMD/CAMD tie-breaking, supervariable detection and dense-row handling are
// not reproduced: the orders differ from SuiteSparse's in detail.
#include "host_symbolic.h"

#include <algorithm>
#include <cstdlib>
#include <exception>
#include <limits>
#include <numeric>
#include <queue>
#include <thread>

namespace mfs {

namespace {

struct QuotientMD {
    idx nv;
    std::vector<std::vector<idx>> A;      // variable neighbours (may hold stale entries)
    std::vector<std::vector<idx>> E;      // adjacent elements (may hold dead ones)
    std::vector<std::vector<idx>> L;      // element variable lists (live variables only)
    std::vector<char> alive, elim;
    std::vector<idx> deg, mark, wmark, w;
    idx stamp = 0, wstamp = 0;

    idx next_stamp() { return ++stamp; }

    // |A_i U (union of L_e, e in E_i)| \ {i}, exactly
    idx exact_degree(idx i) {
        const idx s = next_stamp();
        mark[i] = s;
        idx cnt = 0;
        for (idx j : A[i])
            if (!elim[j] && mark[j] != s) { mark[j] = s; ++cnt; }
        for (idx e : E[i]) {
            if (!alive[e]) continue;
            for (idx j : L[e])
                if (mark[j] != s) { mark[j] = s; ++cnt; }
        }
        return cnt;
    }
};

// Constrained minimum degree. label[v] orders the constraint sets (ascending);
// `elements` are cliques already present (their variables are live). Sets with a
// label >= stop_label are never eliminated: they are halo vertices that only count
// in the degrees of the others.
std::vector<idx> constrained_md(idx nv, const std::vector<idx> &xadj, const std::vector<idx> &adj,
                                const std::vector<std::vector<idx>> &elements, const std::vector<idx> &label,
                                idx stop_label = std::numeric_limits<idx>::max()) {
    QuotientMD q;
    q.nv = nv;
    q.A.resize(nv);
    q.E.resize(nv);
    q.elim.assign(nv, 0);
    q.deg.assign(nv, 0);
    q.mark.assign(nv, 0);
    for (idx v = 0; v < nv; ++v)
        for (idx k = xadj[v]; k < xadj[v + 1]; ++k)
            if (adj[k] != v) q.A[v].push_back(adj[k]);
    for (const auto &el : elements) {
        const idx e = idx(q.L.size());
        q.L.push_back(el);
        for (idx v : el) q.E[v].push_back(e);
    }
    q.alive.assign(q.L.size(), 1);
    q.w.assign(q.L.size(), 0);
    q.wmark.assign(q.L.size(), 0);

    std::vector<idx> byset(nv);
    std::iota(byset.begin(), byset.end(), 0);
    std::stable_sort(byset.begin(), byset.end(), [&](idx a, idx b) { return label[a] < label[b]; });
    std::vector<idx> order;
    order.reserve(nv);
    idx remaining = nv;
    using Entry = std::pair<idx, idx>;    // (degree, vertex)
    std::vector<idx> Lp, keep;
    for (size_t g0 = 0; g0 < byset.size();) {
        size_t g1 = g0;
        while (g1 < byset.size() && label[byset[g1]] == label[byset[g0]]) ++g1;
        const idx cur = label[byset[g0]];
        if (cur >= stop_label) break;
        std::priority_queue<Entry, std::vector<Entry>, std::greater<Entry>> heap;
        for (size_t t = g0; t < g1; ++t) {
            const idx v = byset[t];
            q.deg[v] = q.exact_degree(v);
            heap.push({q.deg[v], v});
        }
        for (idx todo = idx(g1 - g0); todo > 0; --todo) {
            idx p = -1;
            while (!heap.empty()) {
                const Entry top = heap.top();
                heap.pop();
                if (!q.elim[top.second] && q.deg[top.second] == top.first) { p = top.second; break; }
            }
            if (p < 0) break;   // cannot happen: every member of the set is in the heap
            // the new element: p's variable neighbours and the members of its elements
            const idx s = q.next_stamp();
            q.mark[p] = s;
            Lp.clear();
            for (idx j : q.A[p])
                if (!q.elim[j] && q.mark[j] != s) { q.mark[j] = s; Lp.push_back(j); }
            for (idx e : q.E[p]) {
                if (!q.alive[e]) continue;
                for (idx j : q.L[e])
                    if (q.mark[j] != s) { q.mark[j] = s; Lp.push_back(j); }
                q.alive[e] = 0;                                   // absorbed into the new element
                std::vector<idx>().swap(q.L[e]);
            }
            q.elim[p] = 1;
            order.push_back(p);
            --remaining;
            std::vector<idx>().swap(q.A[p]);
            std::vector<idx>().swap(q.E[p]);
            const idx ne = idx(q.L.size());
            q.L.push_back(Lp);
            q.alive.push_back(1);
            q.w.push_back(0);
            q.wmark.push_back(0);
            // |L_e \ L_p| for every live element meeting L_p (AMD's w(e))
            const idx ws = ++q.wstamp;
            for (idx i : Lp)
                for (idx e : q.E[i]) {
                    if (!q.alive[e]) continue;
                    if (q.wmark[e] != ws) { q.wmark[e] = ws; q.w[e] = idx(q.L[e].size()); }
                    --q.w[e];
                }
            const idx lp = idx(Lp.size());
            for (idx i : Lp) {
                // elements: drop dead and fully covered ones (absorbed), add the new one
                keep.clear();
                for (idx e : q.E[i]) {
                    if (!q.alive[e]) continue;
                    if (q.w[e] == 0 && q.wmark[e] == ws) { q.alive[e] = 0; std::vector<idx>().swap(q.L[e]); continue; }
                    keep.push_back(e);
                }
                keep.push_back(ne);
                q.E[i].swap(keep);
                // variable neighbours now reached through the new element leave A_i
                keep.clear();
                for (idx j : q.A[i])
                    if (!q.elim[j] && q.mark[j] != s) keep.push_back(j);
                q.A[i].swap(keep);
                if (label[i] != cur) continue;          // later sets get exact degrees when they start
                idx d = idx(q.A[i].size()) + lp - 1;
                for (idx e : q.E[i])
                    if (e != ne && q.alive[e]) d += (q.wmark[e] == ws) ? q.w[e] : idx(q.L[e].size());
                d = std::min(d, q.deg[i] + lp);
                d = std::min(d, remaining - 1);
                d = std::max<idx>(d, 0);
                if (d != q.deg[i]) {
                    q.deg[i] = d;
                    heap.push({d, i});
                }
            }
            // Mass elimination: a variable of the current set whose only neighbour is the
            // new element is simplicial (its neighbourhood is already a clique), so
            // eliminating it now adds no fill; it leaves the element and the order.
            idx nsimp = 0;
            for (idx i : Lp) {
                if (label[i] != cur || !q.A[i].empty() || q.E[i].size() != 1 || todo - 1 - nsimp <= 0) continue;
                q.elim[i] = 1;
                order.push_back(i);
                --remaining;
                ++nsimp;
                std::vector<idx>().swap(q.E[i]);
            }
            if (nsimp > 0) {
                todo -= nsimp;
                auto &le = q.L[ne];
                le.erase(std::remove_if(le.begin(), le.end(), [&](idx j) { return q.elim[j] != 0; }), le.end());
            }
        }
        g0 = g1;
    }
    return order;
}

}  // namespace

std::vector<idx> quotient_minimum_degree(idx n, const std::vector<idx> &xadj, const std::vector<idx> &adj) {
    return constrained_md(n, xadj, adj, {}, std::vector<idx>(size_t(n), 0));
}

int camd_cut_depth_from_env() {
    const char *e = std::getenv("MFS_ND_CAMD_CUT_DEPTH");
    if (!e || !*e) return 4;
    char *end = nullptr;
    const long v = std::strtol(e, &end, 10);
    if (end == e) return 4;
    return int(v);
}

std::vector<idx> hierarchical_constrained_md(idx n, const std::vector<idx> &xadj, const std::vector<idx> &adj,
                                             const NDResult &nd, int cut_depth, HierarchicalMDStats *stats) {
    const idx nc = nd.ncomp;
    if (cut_depth < 0 || nc <= 0 || idx(nd.cmember.size()) != n) return nd.iperm;
    // depths (parents follow children in postorder), the cut, task roots
    std::vector<int> depth(nc, 0);
    int max_depth = 0;
    for (idx c = nc - 1; c >= 0; --c) {
        const idx p = nd.cparent[c];
        if (p >= 0) {
            if (p <= c || p >= nc) return nd.iperm;     // not a postordered forest
            depth[c] = depth[p] + 1;
        }
        max_depth = std::max(max_depth, depth[c]);
    }
    const int cut = std::min(cut_depth, max_depth);
    std::vector<idx> root(nc, -1), task_of_root(nc, -1);
    for (idx c = nc - 1; c >= 0; --c) {
        if (depth[c] == cut) root[c] = c;
        else if (depth[c] > cut) root[c] = root[nd.cparent[c]];
    }
    idx nt = 0;
    for (idx c = 0; c < nc; ++c)
        if (root[c] == c) task_of_root[c] = nt++;
    std::vector<std::vector<idx>> verts(nt);
    std::vector<idx> upper, owner(n), local(n);
    for (idx v = 0; v < n; ++v) {
        const idx c = nd.cmember[v];
        owner[v] = root[c] < 0 ? -1 : task_of_root[root[c]];
        auto &list = owner[v] < 0 ? upper : verts[owner[v]];
        local[v] = idx(list.size());
        list.push_back(v);
    }
    for (idx v = 0; v < n; ++v)                      // a subtree edge into another subtree: not a dissection
        for (idx k = xadj[v]; k < xadj[v + 1]; ++k) {
            const idx u = adj[k];
            if (owner[v] >= 0 && owner[u] >= 0 && owner[u] != owner[v]) return nd.iperm;
        }

    std::vector<std::vector<idx>> perms(nt);
    std::vector<std::vector<std::vector<idx>>> bounds(nt);
    // per-worker maps over the upper vertices, set up once and reset after each task
    // (a forest of many trees has thousands of subtrees at the cut)
    struct Scratch {
        std::vector<idx> hid, umark;
        idx stamp = 0;
    };
    auto run_task = [&](idx t, Scratch &sc) {
        if (sc.hid.size() != upper.size()) {
            sc.hid.assign(upper.size(), -1);
            sc.umark.assign(upper.size(), 0);
        }
        const auto &vs = verts[t];
        const idx m = idx(vs.size());
        // local graph: the subtree's vertices, then its halo (the upper vertices next to
        // it, labelled after every component and never eliminated: they count in the
        // degrees, as the separators above will be eliminated later)
        std::vector<idx> &hid = sc.hid, halo;
        std::vector<std::vector<idx>> hadj;
        std::vector<idx> lx(m + 1, 0), la, lab(m);
        for (idx a = 0; a < m; ++a) {
            const idx v = vs[a];
            lab[a] = nd.cmember[v];
            for (idx k = xadj[v]; k < xadj[v + 1]; ++k) {
                const idx u = adj[k];
                if (u == v) continue;
                if (owner[u] == t) {
                    la.push_back(local[u]);
                } else if (owner[u] < 0) {
                    idx &h = hid[local[u]];
                    if (h < 0) { h = idx(halo.size()); halo.push_back(u); hadj.emplace_back(); }
                    la.push_back(m + h);
                    hadj[h].push_back(a);
                }
            }
            lx[a + 1] = idx(la.size());
        }
        const idx nh = idx(halo.size());
        lx.resize(m + nh + 1);
        for (idx h = 0; h < nh; ++h) {
            la.insert(la.end(), hadj[h].begin(), hadj[h].end());
            lx[m + h + 1] = idx(la.size());
        }
        for (idx u : halo) hid[local[u]] = -1;
        lab.resize(m + nh, nc);
        std::vector<idx> ord = constrained_md(m + nh, lx, la, {}, lab, nc);
        for (idx &a : ord) a = vs[a];
        perms[t] = std::move(ord);
        // every connected part of the subtree leaves its upper neighbours one clique
        std::vector<char> seen(m, 0);
        std::vector<idx> stack, b;
        std::vector<idx> &umark = sc.umark;
        for (idx s0 = 0; s0 < m; ++s0) {
            if (seen[s0]) continue;
            seen[s0] = 1;
            const idx part = ++sc.stamp;             // marks this connected part's boundary
            stack.assign(1, s0);
            b.clear();
            while (!stack.empty()) {
                const idx a = stack.back();
                stack.pop_back();
                const idx v = vs[a];
                for (idx k = xadj[v]; k < xadj[v + 1]; ++k) {
                    const idx u = adj[k];
                    if (owner[u] < 0) {
                        if (umark[local[u]] != part) { umark[local[u]] = part; b.push_back(local[u]); }
                    } else if (!seen[local[u]]) {
                        seen[local[u]] = 1;
                        stack.push_back(local[u]);
                    }
                }
            }
            if (b.size() >= 2) {
                std::sort(b.begin(), b.end());
                bounds[t].push_back(b);
            }
        }
    };
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const idx nthreads = std::min<idx>(idx(hw), nt);
    if (nthreads <= 1) {
        Scratch sc;
        for (idx t = 0; t < nt; ++t) run_task(t, sc);
    } else {
        // an exception must not leave a worker thread (that would terminate the
        // process): the first one is kept and rethrown on this thread after the join
        std::vector<std::exception_ptr> errors(static_cast<size_t>(nthreads));
        std::vector<std::thread> pool;
        for (idx th = 0; th < nthreads; ++th)
            pool.emplace_back([&, th] {
                try {
                    Scratch sc;
                    for (idx t = th; t < nt; t += nthreads) run_task(t, sc);
                } catch (...) {
                    errors[size_t(th)] = std::current_exception();
                }
            });
        for (auto &th : pool) th.join();
        for (auto &e : errors)
            if (e) std::rethrow_exception(e);
    }

    // the separators above the cut, with the subtrees' cliques as initial elements
    const idx nu = idx(upper.size());
    std::vector<idx> ux(nu + 1, 0), ua, ulab(nu);
    for (idx a = 0; a < nu; ++a) {
        const idx v = upper[a];
        ulab[a] = nd.cmember[v];
        for (idx k = xadj[v]; k < xadj[v + 1]; ++k)
            if (owner[adj[k]] < 0 && adj[k] != v) ua.push_back(local[adj[k]]);
        ux[a + 1] = idx(ua.size());
    }
    std::vector<std::vector<idx>> elements;
    for (auto &tb : bounds)
        for (auto &b : tb) elements.push_back(std::move(b));
    std::vector<idx> uord = constrained_md(nu, ux, ua, elements, ulab);

    std::vector<idx> iperm;
    iperm.reserve(n);
    for (auto &p : perms) iperm.insert(iperm.end(), p.begin(), p.end());
    for (idx a : uord) iperm.push_back(upper[a]);
    if (idx(iperm.size()) != n) return nd.iperm;
    if (stats) {
        stats->applied = true;
        stats->cut_depth = cut;
        stats->tasks = nt;
        stats->upper_vertices = nu;
        stats->upper_elements = idx(elements.size());
    }
    return iperm;
}

}  // namespace mfs
