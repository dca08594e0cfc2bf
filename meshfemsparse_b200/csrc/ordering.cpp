// Fill-reducing orderings for the host symbolic stage.
//
// The reference orders the reduced block graph with its parallel nested
// dissection driver (Solvers/ParallelNestedDissection/cholmod_nesdis_parallel.cc:
// 299-560, entry nested_dissection_from_graph :1546) around METIS node
// bisection (nesdis_bisector.cc:110-186) and finishes every subtree with
// constrained minimum degree (hierarchical_camd.cc:165). METIS and CAMD are
// third-party code that is not part of the reference tree, so this file is a
// self-contained restatement of the same structure:
//   * connected components are ordered independently (forest roots);
//   * each component is bisected by a multilevel edge bisection (heavy-edge
//     matching coarsening, region-growing initial cut, Fiduccia-Mattheyses
//     refinement while uncoarsening) that is turned into a vertex separator by
//     a minimum vertex cover of the cut edges (Koenig's theorem);
//   * both halves recurse; separator vertices are numbered after them;
//   * pieces below `leaf_size` vertices get a minimum-degree order that also
//     counts their (later eliminated) outside neighbours ("halo").
// The separator tree (CParent/CMember, postordered) is reported like
// cholmod_ordering.hh:222-258 expects it.
#include "host_symbolic.h"

#include <algorithm>
#include <cstdint>
#include <functional>
#include <numeric>
#include <queue>
#include <stdexcept>

namespace mfs {
namespace {

struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(seed ? seed : 0x9E3779B97F4A7C15ull) {}
    uint64_t next() {
        s ^= s << 13; s ^= s >> 7; s ^= s << 17;
        return s;
    }
    idx below(idx n) { return n <= 1 ? 0 : idx(next() % uint64_t(n)); }
};

// Weighted undirected graph in adjacency (CSR) form.
struct WGraph {
    idx n = 0;
    std::vector<idx> xadj, adj, ew, vw;
    idx totw = 0;
};

// ------------------------------------------------------------ coarsening --
// Heavy-edge matching; returns false when the graph no longer shrinks.
bool coarsen(const WGraph &g, WGraph &cg, std::vector<idx> &cmap, Rng &rng) {
    const idx n = g.n;
    std::vector<idx> order(n);
    std::iota(order.begin(), order.end(), 0);
    for (idx i = n - 1; i > 0; --i) std::swap(order[i], order[rng.below(i + 1)]);
    std::vector<idx> match(n, -1);
    const idx maxvw = std::max<idx>(1, (g.totw + 49) / 50);   // keep coarse vertices light
    for (idx v : order) {
        if (match[v] != -1) continue;
        idx best = -1, bw = -1;
        for (idx e = g.xadj[v]; e < g.xadj[v + 1]; ++e) {
            idx u = g.adj[e];
            if (match[u] != -1 || u == v) continue;
            if (g.vw[u] + g.vw[v] > maxvw) continue;
            if (g.ew[e] > bw) { bw = g.ew[e]; best = u; }
        }
        if (best >= 0) { match[v] = best; match[best] = v; }
        else match[v] = v;
    }
    cmap.assign(n, -1);
    idx nc = 0;
    for (idx v = 0; v < n; ++v) {
        if (cmap[v] != -1) continue;
        cmap[v] = nc;
        if (match[v] != v) cmap[match[v]] = nc;
        ++nc;
    }
    if (nc > idx(0.95 * double(n))) return false;
    cg.n = nc;
    cg.vw.assign(nc, 0);
    cg.xadj.assign(nc + 1, 0);
    cg.adj.clear(); cg.ew.clear();
    cg.adj.reserve(g.adj.size()); cg.ew.reserve(g.adj.size());
    std::vector<idx> pos(nc, -1);
    std::vector<idx> first(nc, -1);
    for (idx v = 0; v < n; ++v) if (first[cmap[v]] == -1) first[cmap[v]] = v;
    for (idx c = 0; c < nc; ++c) {
        idx v0 = first[c];
        idx v1 = match[v0];
        idx start = idx(cg.adj.size());
        for (idx v : {v0, v1}) {
            cg.vw[c] += g.vw[v];
            for (idx e = g.xadj[v]; e < g.xadj[v + 1]; ++e) {
                idx cu = cmap[g.adj[e]];
                if (cu == c) continue;
                if (pos[cu] >= start) cg.ew[pos[cu]] += g.ew[e];
                else {
                    pos[cu] = idx(cg.adj.size());
                    cg.adj.push_back(cu);
                    cg.ew.push_back(g.ew[e]);
                }
            }
            if (v1 == v0) break;
        }
        cg.xadj[c + 1] = idx(cg.adj.size());
    }
    cg.totw = g.totw;
    return true;
}

// ------------------------------------------------------- FM refinement --
idx cut_of(const WGraph &g, const std::vector<int8_t> &where) {
    idx cut = 0;
    for (idx v = 0; v < g.n; ++v)
        for (idx e = g.xadj[v]; e < g.xadj[v + 1]; ++e)
            if (where[g.adj[e]] != where[v]) cut += g.ew[e];
    return cut / 2;
}

// Two-way Fiduccia-Mattheyses with lazy max-heaps. Balance: each side at most
// `maxside` weight.
void fm_refine(const WGraph &g, std::vector<int8_t> &where, int passes, double imbalance) {
    const idx n = g.n;
    const idx maxside = idx(double(g.totw) * (0.5 + imbalance)) + 1;
    std::vector<idx> gain(n);
    std::vector<idx> stamp(n, 0);
    std::vector<char> locked(n);
    idx pw[2] = {0, 0};
    for (idx v = 0; v < n; ++v) pw[where[v]] += g.vw[v];
    auto compute_gain = [&](idx v) {
        idx ext = 0, in = 0;
        for (idx e = g.xadj[v]; e < g.xadj[v + 1]; ++e) {
            if (where[g.adj[e]] != where[v]) ext += g.ew[e]; else in += g.ew[e];
        }
        return ext - in;
    };
    struct HE { idx gain, v, st; bool operator<(const HE &o) const { return gain < o.gain || (gain == o.gain && v > o.v); } };
    // max-heaps of (gain, lower vertex first) kept in vectors whose capacity survives
    // the passes (the same push / pop order as a std::priority_queue)
    std::vector<HE> heap[2];
    const std::less<HE> cmp;
    auto push = [&](int side, HE h) {
        heap[side].push_back(h);
        std::push_heap(heap[side].begin(), heap[side].end(), cmp);
    };
    std::vector<idx> moves;
    for (int pass = 0; pass < passes; ++pass) {
        heap[0].clear();
        heap[1].clear();
        std::fill(locked.begin(), locked.end(), 0);
        for (idx v = 0; v < n; ++v) {
            gain[v] = compute_gain(v);
            bool boundary = false;
            for (idx e = g.xadj[v]; e < g.xadj[v + 1]; ++e) if (where[g.adj[e]] != where[v]) { boundary = true; break; }
            if (boundary) push(where[v], {gain[v], v, ++stamp[v]});
        }
        idx cut = cut_of(g, where);
        idx best_cut = cut;
        idx best_bal = std::max(pw[0], pw[1]);
        moves.clear();
        idx best_len = 0;
        idx since_best = 0;
        const idx limit = std::max<idx>(25, n / 50);
        while (since_best < limit) {
            // Prefer moving from the heavier side; fall back to the other side.
            int from = pw[0] >= pw[1] ? 0 : 1;
            idx v = -1;
            for (int attempt = 0; attempt < 2 && v < 0; ++attempt) {
                int side = attempt == 0 ? from : 1 - from;
                auto &h = heap[side];
                auto pop = [&] {
                    std::pop_heap(h.begin(), h.end(), cmp);
                    h.pop_back();
                };
                while (!h.empty()) {
                    const HE top = h.front();
                    if (locked[top.v] || top.st != stamp[top.v] || where[top.v] != side) { pop(); continue; }
                    if (pw[1 - side] + g.vw[top.v] > maxside) break;
                    v = top.v; pop();
                    break;
                }
            }
            if (v < 0) break;
            int s = where[v];
            cut -= gain[v];
            where[v] = int8_t(1 - s);
            pw[s] -= g.vw[v]; pw[1 - s] += g.vw[v];
            locked[v] = 1;
            moves.push_back(v);
            // v left side s: for a neighbour on s the edge turns external (+2w), for one on
            // the other side internal (-2w); the exact gains of the unlocked neighbours
            for (idx e = g.xadj[v]; e < g.xadj[v + 1]; ++e) {
                idx u = g.adj[e];
                if (locked[u]) continue;
                gain[u] += where[u] == s ? 2 * g.ew[e] : -2 * g.ew[e];
                push(where[u], {gain[u], u, ++stamp[u]});
            }
            idx bal = std::max(pw[0], pw[1]);
            bool feasible = bal <= maxside;
            if (feasible && (cut < best_cut || (cut == best_cut && bal < best_bal))) {
                best_cut = cut; best_bal = bal; best_len = idx(moves.size()); since_best = 0;
            } else ++since_best;
        }
        // roll back past the best prefix
        for (idx k = idx(moves.size()) - 1; k >= best_len; --k) {
            idx v = moves[k];
            int s = where[v];
            where[v] = int8_t(1 - s);
            pw[s] -= g.vw[v]; pw[1 - s] += g.vw[v];
        }
        if (best_len == 0) break;
    }
}

// Region growing from a seed until half the weight is reached.
void grow_bisection(const WGraph &g, idx seed, std::vector<int8_t> &where) {
    where.assign(g.n, 1);
    idx half = g.totw / 2, w = 0;
    std::vector<idx> queue;
    std::vector<char> seen(g.n, 0);
    queue.push_back(seed); seen[seed] = 1;
    size_t head = 0;
    while (w < half) {
        if (head == queue.size()) {
            idx s = -1;
            for (idx v = 0; v < g.n; ++v) if (!seen[v]) { s = v; break; }
            if (s < 0) break;
            queue.push_back(s); seen[s] = 1;
        }
        idx v = queue[head++];
        where[v] = 0; w += g.vw[v];
        for (idx e = g.xadj[v]; e < g.xadj[v + 1]; ++e) {
            idx u = g.adj[e];
            if (!seen[u]) { seen[u] = 1; queue.push_back(u); }
        }
    }
}

std::vector<int8_t> multilevel_bisect(const WGraph &g0, const OrderingOptions &opt, Rng &rng) {
    std::vector<WGraph> graphs;
    std::vector<std::vector<idx>> cmaps;
    graphs.push_back(g0);
    while (graphs.back().n > 160) {
        WGraph cg; std::vector<idx> cmap;
        if (!coarsen(graphs.back(), cg, cmap, rng)) break;
        graphs.push_back(std::move(cg));
        cmaps.push_back(std::move(cmap));
    }
    const WGraph &gc = graphs.back();
    std::vector<int8_t> best;
    idx best_cut = -1;
    for (int t = 0; t < opt.init_tries; ++t) {
        std::vector<int8_t> where;
        grow_bisection(gc, rng.below(gc.n), where);
        fm_refine(gc, where, opt.refine_passes, 0.05);
        idx c = cut_of(gc, where);
        if (best_cut < 0 || c < best_cut) { best_cut = c; best = where; }
    }
    for (idx lvl = idx(graphs.size()) - 2; lvl >= 0; --lvl) {
        const WGraph &gf = graphs[lvl];
        const std::vector<idx> &cmap = cmaps[lvl];
        std::vector<int8_t> wf(gf.n);
        for (idx v = 0; v < gf.n; ++v) wf[v] = best[cmap[v]];
        fm_refine(gf, wf, opt.refine_passes, 0.05);
        best.swap(wf);
    }
    return best;
}

// Minimum vertex cover of the bipartite cut graph (Hopcroft-Karp + Koenig).
std::vector<char> cut_vertex_cover(const WGraph &g, const std::vector<int8_t> &where) {
    const idx n = g.n;
    std::vector<idx> L, R, lid(n, -1), rid(n, -1);
    for (idx v = 0; v < n; ++v) {
        bool b = false;
        for (idx e = g.xadj[v]; e < g.xadj[v + 1]; ++e) if (where[g.adj[e]] != where[v]) { b = true; break; }
        if (!b) continue;
        if (where[v] == 0) { lid[v] = idx(L.size()); L.push_back(v); }
        else { rid[v] = idx(R.size()); R.push_back(v); }
    }
    const idx nl = idx(L.size()), nr = idx(R.size());
    std::vector<idx> matchL(nl, -1), matchR(nr, -1), dist(nl);
    auto bfs = [&]() {
        std::queue<idx> q;
        bool found = false;
        for (idx l = 0; l < nl; ++l) {
            if (matchL[l] < 0) { dist[l] = 0; q.push(l); } else dist[l] = -1;
        }
        while (!q.empty()) {
            idx l = q.front(); q.pop();
            idx v = L[l];
            for (idx e = g.xadj[v]; e < g.xadj[v + 1]; ++e) {
                idx r = rid[g.adj[e]];
                if (r < 0) continue;
                idx l2 = matchR[r];
                if (l2 < 0) found = true;
                else if (dist[l2] < 0) { dist[l2] = dist[l] + 1; q.push(l2); }
            }
        }
        return found;
    };
    // iterative DFS for augmenting paths
    std::vector<idx> it(nl);
    auto dfs = [&](idx root) {
        std::vector<idx> stack{root};
        std::vector<idx> via;  // right vertex used to reach stack[k+1]
        it[root] = g.xadj[L[root]];
        while (!stack.empty()) {
            idx l = stack.back();
            idx v = L[l];
            bool advanced = false;
            for (; it[l] < g.xadj[v + 1]; ++it[l]) {
                idx r = rid[g.adj[it[l]]];
                if (r < 0) continue;
                idx l2 = matchR[r];
                if (l2 < 0) {
                    // augment along the stack
                    via.push_back(r);
                    for (size_t k = 0; k < stack.size(); ++k) {
                        matchL[stack[k]] = via[k];
                        matchR[via[k]] = stack[k];
                    }
                    return true;
                }
                if (dist[l2] == dist[l] + 1) {
                    via.push_back(r);
                    ++it[l];
                    it[l2] = g.xadj[L[l2]];
                    stack.push_back(l2);
                    advanced = true;
                    break;
                }
            }
            if (!advanced) {
                dist[l] = -1;
                stack.pop_back();
                if (!via.empty()) via.pop_back();
            }
        }
        return false;
    };
    while (bfs()) {
        for (idx l = 0; l < nl; ++l) if (matchL[l] < 0) { it[l] = g.xadj[L[l]]; dfs(l); }
    }
    // Koenig: Z = vertices reachable from unmatched left vertices by alternating paths.
    std::vector<char> zl(nl, 0), zr(nr, 0);
    std::queue<idx> q;
    for (idx l = 0; l < nl; ++l) if (matchL[l] < 0) { zl[l] = 1; q.push(l); }
    while (!q.empty()) {
        idx l = q.front(); q.pop();
        idx v = L[l];
        for (idx e = g.xadj[v]; e < g.xadj[v + 1]; ++e) {
            idx r = rid[g.adj[e]];
            if (r < 0 || zr[r] || matchL[l] == r) continue;
            zr[r] = 1;
            idx l2 = matchR[r];
            if (l2 >= 0 && !zl[l2]) { zl[l2] = 1; q.push(l2); }
        }
    }
    std::vector<char> sep(n, 0);
    for (idx l = 0; l < nl; ++l) if (!zl[l]) sep[L[l]] = 1;
    for (idx r = 0; r < nr; ++r) if (zr[r]) sep[R[r]] = 1;
    return sep;
}

// The same elimination on bit rows (graphs of up to kBitsetMdMax vertices, the
// nested-dissection leaves with their halos): a row's popcount is the vertex's
// degree and the neighbour update is a word-wise OR, so pivots and order are those
// of the list form below.
constexpr idx kBitsetMdMax = 4096;
std::vector<idx> md_local_bits(idx n, const std::vector<std::vector<idx>> &adj0, const std::vector<char> &elim) {
    const idx W = (n + 63) / 64;
    std::vector<uint64_t> rows(size_t(n * W), 0);
    auto row = [&](idx v) { return rows.data() + v * W; };
    for (idx v = 0; v < n; ++v)
        for (idx u : adj0[v])
            if (u != v) row(v)[u >> 6] |= uint64_t(1) << (u & 63);
    std::vector<idx> deg(n, 0);
    for (idx v = 0; v < n; ++v)
        for (idx w = 0; w < W; ++w) deg[v] += idx(__builtin_popcountll(row(v)[w]));
    std::vector<char> gone(n, 0);
    idx todo = 0;
    for (idx v = 0; v < n; ++v) todo += elim[v] ? 1 : 0;
    std::vector<idx> order;
    order.reserve(todo);
    std::vector<uint64_t> nb(static_cast<size_t>(W));
    while (idx(order.size()) < todo) {
        idx best = -1, bd = 0;
        for (idx v = 0; v < n; ++v) {
            if (!elim[v] || gone[v]) continue;
            if (best < 0 || deg[v] < bd) { best = v; bd = deg[v]; }
        }
        const idx p = best;
        order.push_back(p);
        gone[p] = 1;
        std::copy(row(p), row(p) + W, nb.begin());
        for (idx w = 0; w < W; ++w)
            for (uint64_t bits = nb[size_t(w)]; bits; bits &= bits - 1) {
                const idx u = w * 64 + idx(__builtin_ctzll(bits));
                uint64_t *ru = row(u);
                idx d = 0;
                for (idx x = 0; x < W; ++x) {
                    ru[x] |= nb[size_t(x)];
                    if (x == (u >> 6)) ru[x] &= ~(uint64_t(1) << (u & 63));
                    if (x == (p >> 6)) ru[x] &= ~(uint64_t(1) << (p & 63));
                    d += idx(__builtin_popcountll(ru[x]));
                }
                deg[u] = d;
            }
        std::fill(row(p), row(p) + W, 0);
        deg[p] = 0;
    }
    return order;
}

// Minimum degree on an explicit elimination graph. `elim` marks the vertices
// to order (the others are halo vertices that stay in the graph).
std::vector<idx> md_local(idx n, const std::vector<std::vector<idx>> &adj0, const std::vector<char> &elim) {
    if (n <= kBitsetMdMax) return md_local_bits(n, adj0, elim);
    std::vector<std::vector<idx>> adj = adj0;
    for (auto &a : adj) std::sort(a.begin(), a.end());
    std::vector<char> gone(n, 0);
    std::vector<idx> order;
    idx todo = 0;
    for (idx v = 0; v < n; ++v) todo += elim[v] ? 1 : 0;
    order.reserve(todo);
    std::vector<idx> tmp;
    while (idx(order.size()) < todo) {
        idx best = -1, bd = 0;
        for (idx v = 0; v < n; ++v) {
            if (!elim[v] || gone[v]) continue;
            idx dg = idx(adj[v].size());
            if (best < 0 || dg < bd) { best = v; bd = dg; }
        }
        idx p = best;
        order.push_back(p);
        gone[p] = 1;
        const std::vector<idx> nb = adj[p];
        for (idx u : nb) {
            // adj[u] = (adj[u] U nb) \ {u, p}
            tmp.clear();
            std::set_union(adj[u].begin(), adj[u].end(), nb.begin(), nb.end(), std::back_inserter(tmp));
            adj[u].clear();
            for (idx x : tmp) if (x != u && x != p) adj[u].push_back(x);
        }
        adj[p].clear();
    }
    return order;
}

struct NDState {
    const std::vector<idx> &xadj, &adj;
    const OrderingOptions &opt;
    Rng rng;
    std::vector<idx> iperm;
    std::vector<idx> node_parent;      // internal tree nodes
    std::vector<idx> node_post;        // completion index per node
    std::vector<idx> member_node;      // per vertex
    std::vector<char> placed;          // vertex already numbered
    std::vector<idx> local;            // scratch: global -> local id
    idx post_counter = 0;
    NDState(const std::vector<idx> &x, const std::vector<idx> &a, const OrderingOptions &o, idx n)
        : xadj(x), adj(a), opt(o), rng(o.seed), member_node(n, -1), placed(n, 0), local(n, -1) {}

    idx new_node(idx parent) {
        node_parent.push_back(parent);
        node_post.push_back(-1);
        return idx(node_parent.size()) - 1;
    }
    void finish(idx node) { node_post[node] = post_counter++; }

    // Split `verts` into connected components (within `verts`).
    std::vector<std::vector<idx>> components(const std::vector<idx> &verts) {
        for (size_t k = 0; k < verts.size(); ++k) local[verts[k]] = idx(k);
        std::vector<char> seen(verts.size(), 0);
        std::vector<std::vector<idx>> comps;
        for (size_t k = 0; k < verts.size(); ++k) {
            if (seen[k]) continue;
            std::vector<idx> comp{verts[k]};
            seen[k] = 1;
            for (size_t h = 0; h < comp.size(); ++h) {
                idx v = comp[h];
                for (idx e = xadj[v]; e < xadj[v + 1]; ++e) {
                    idx u = adj[e];
                    idx lu = local[u];
                    if (lu < 0 || lu >= idx(verts.size()) || verts[lu] != u || seen[lu]) continue;
                    seen[lu] = 1;
                    comp.push_back(u);
                }
            }
            std::sort(comp.begin(), comp.end());
            comps.push_back(std::move(comp));
        }
        for (idx v : verts) local[v] = -1;
        return comps;
    }

    void order_leaf(const std::vector<idx> &verts, idx parent) {
        idx node = new_node(parent);
        // local graph: leaf vertices first, then halo
        std::vector<idx> ids(verts);
        for (size_t k = 0; k < ids.size(); ++k) local[ids[k]] = idx(k);
        const idx nleaf = idx(ids.size());
        for (idx k = 0; k < nleaf; ++k) {
            idx v = ids[k];
            for (idx e = xadj[v]; e < xadj[v + 1]; ++e) {
                idx u = adj[e];
                if (local[u] < 0 && !placed[u]) { local[u] = idx(ids.size()); ids.push_back(u); }
            }
        }
        const idx nl = idx(ids.size());
        std::vector<std::vector<idx>> ladj(nl);
        std::vector<char> elim(nl, 0);
        for (idx k = 0; k < nleaf; ++k) elim[k] = 1;
        for (idx k = 0; k < nleaf; ++k) {
            idx v = ids[k];
            for (idx e = xadj[v]; e < xadj[v + 1]; ++e) {
                idx lu = local[adj[e]];
                if (lu < 0 || lu == k) continue;
                ladj[k].push_back(lu);
                if (lu >= nleaf) ladj[lu].push_back(k);
            }
        }
        for (idx v : ids) local[v] = -1;
        std::vector<idx> ord = md_local(nl, ladj, elim);
        for (idx k : ord) { iperm.push_back(ids[k]); member_node[ids[k]] = node; placed[ids[k]] = 1; }
        finish(node);
    }

    void recurse(const std::vector<idx> &verts, idx parent) {
        if (verts.empty()) return;
        auto comps = components(verts);
        if (comps.size() > 1) {
            for (auto &c : comps) recurse(c, parent);
            return;
        }
        const std::vector<idx> &vs = comps[0];
        const idx n = idx(vs.size());
        if (n <= opt.leaf_size) { order_leaf(vs, parent); return; }
        // build the induced unit-weight graph
        WGraph g;
        g.n = n;
        g.xadj.assign(n + 1, 0);
        for (idx k = 0; k < n; ++k) local[vs[k]] = k;
        for (idx k = 0; k < n; ++k) {
            idx v = vs[k];
            for (idx e = xadj[v]; e < xadj[v + 1]; ++e) {
                idx lu = local[adj[e]];
                if (lu >= 0 && lu != k && vs[lu] == adj[e]) { g.adj.push_back(lu); g.ew.push_back(1); }
            }
            g.xadj[k + 1] = idx(g.adj.size());
        }
        for (idx k = 0; k < n; ++k) local[vs[k]] = -1;
        g.vw.assign(n, 1);
        g.totw = n;
        std::vector<int8_t> where = multilevel_bisect(g, opt, rng);
        std::vector<char> sep = cut_vertex_cover(g, where);
        std::vector<idx> A, B, S;
        for (idx k = 0; k < n; ++k) {
            if (sep[k]) S.push_back(vs[k]);
            else if (where[k] == 0) A.push_back(vs[k]);
            else B.push_back(vs[k]);
        }
        if (A.empty() || B.empty()) { order_leaf(vs, parent); return; }
        idx snode = new_node(parent);
        recurse(A, snode);
        recurse(B, snode);
        for (idx v : S) { iperm.push_back(v); member_node[v] = snode; placed[v] = 1; }
        finish(snode);
    }

    // Temporal reuse: replay the previous separator tree, re-dissecting only the
    // subtrees whose components an edge of the new graph now joins. `first[c]` is
    // the first postorder index in c's subtree; `rebuild[c]` marks a subtree to
    // dissect afresh; `members[c]` are c's own vertices.
    void replay(idx c, idx parent, const std::vector<std::vector<idx>> &children,
                const std::vector<std::vector<idx>> &members, const std::vector<idx> &first,
                const std::vector<char> &rebuild, const std::vector<idx> &cmember, idx &rebuilt) {
        if (rebuild[c]) {
            std::vector<idx> verts;
            for (idx v = 0; v < idx(cmember.size()); ++v)
                if (cmember[v] >= first[c] && cmember[v] <= c) verts.push_back(v);
            rebuilt += idx(verts.size());
            recurse(verts, parent);
            return;
        }
        if (children[c].empty()) {
            order_leaf(members[c], parent);
            return;
        }
        idx node = new_node(parent);
        for (idx ch : children[c]) replay(ch, node, children, members, first, rebuild, cmember, rebuilt);
        for (idx v : members[c]) { iperm.push_back(v); member_node[v] = node; placed[v] = 1; }
        finish(node);
    }
};

NDResult finish_result(NDState &st, idx n) {
    if (idx(st.iperm.size()) != n) throw std::logic_error("nested dissection lost vertices");
    NDResult r;
    r.iperm = std::move(st.iperm);
    const idx nn = idx(st.node_parent.size());
    r.ncomp = nn;
    r.cparent.assign(nn, -1);
    for (idx k = 0; k < nn; ++k) {
        idx p = st.node_parent[k];
        r.cparent[st.node_post[k]] = p < 0 ? -1 : st.node_post[p];
    }
    r.cmember.resize(n);
    for (idx v = 0; v < n; ++v) r.cmember[v] = st.node_post[st.member_node[v]];
    return r;
}

}  // namespace

DirtySubtrees dirty_subtrees(idx n, const std::vector<idx> &xadj, const std::vector<idx> &adj,
                             const std::vector<idx> &cparent, const std::vector<idx> &cmember) {
    const idx nc = idx(cparent.size());
    DirtySubtrees out;
    std::vector<idx> depth(nc, 0);
    idx nroots = 0;
    for (idx c = nc - 1; c >= 0; --c) {              // parents follow children
        if (cparent[c] >= 0) depth[c] = depth[cparent[c]] + 1;
        else ++nroots;
    }
    auto lca = [&](idx a, idx b) {
        while (depth[a] > depth[b]) a = cparent[a];
        while (depth[b] > depth[a]) b = cparent[b];
        while (a != b && a >= 0 && b >= 0) { a = cparent[a]; b = cparent[b]; }
        return a == b ? a : idx(-1);
    };
    std::vector<char> dirty(nc, 0);
    for (idx v = 0; v < n; ++v)
        for (idx k = xadj[v]; k < xadj[v + 1]; ++k) {
            const idx u = adj[k];
            if (u >= v) continue;                        // each undirected edge once
            const idx a = cmember[v], b = cmember[u];
            const idx r = lca(a, b);
            if (r == a || r == b) continue;              // one component below the other
            if (r < 0 || (cparent[r] < 0 && nroots == 1)) {
                out.full = true;
                out.roots.clear();
                return out;
            }
            dirty[r] = 1;
        }
    for (idx c = 0; c < nc; ++c) {
        if (!dirty[c]) continue;
        idx p = cparent[c];
        while (p >= 0 && !dirty[p]) p = cparent[p];
        if (p < 0) out.roots.push_back(c);
    }
    return out;
}

NDResult nested_dissection_reuse(idx n, const std::vector<idx> &xadj, const std::vector<idx> &adj,
                                 const NDResult &prev, const OrderingOptions &opt, idx *rebuilt_vertices) {
    if (idx(prev.cmember.size()) != n || prev.ncomp <= 0) return nested_dissection(n, xadj, adj, opt);
    const DirtySubtrees dirty = dirty_subtrees(n, xadj, adj, prev.cparent, prev.cmember);
    if (dirty.full) {
        // no separator of the old forest is left to keep (an edge joins two trees, e.g.
        // new contact between bodies, or crosses the only root): dissect afresh, which
        // counts as a full dissection (-1)
        if (rebuilt_vertices) *rebuilt_vertices = -1;
        return nested_dissection(n, xadj, adj, opt);
    }
    const idx nc = prev.ncomp;
    std::vector<std::vector<idx>> children(nc), members(nc);
    std::vector<idx> first(nc);
    for (idx c = 0; c < nc; ++c) first[c] = c;
    for (idx c = 0; c < nc; ++c)               // postorder: children precede parents
        if (prev.cparent[c] >= 0) {
            children[prev.cparent[c]].push_back(c);
            first[prev.cparent[c]] = std::min(first[prev.cparent[c]], first[c]);
        }
    for (idx v = 0; v < n; ++v) members[prev.cmember[v]].push_back(v);
    std::vector<char> rebuild(nc, 0);
    for (idx c : dirty.roots) rebuild[c] = 1;
    NDState st(xadj, adj, opt, n);
    st.iperm.reserve(n);
    idx rebuilt = 0;
    for (idx c = 0; c < nc; ++c)
        if (prev.cparent[c] < 0) st.replay(c, -1, children, members, first, rebuild, prev.cmember, rebuilt);
    if (rebuilt_vertices) *rebuilt_vertices = rebuilt;
    return finish_result(st, n);
}

NDResult nested_dissection(idx n, const std::vector<idx> &xadj, const std::vector<idx> &adj,
                           const OrderingOptions &opt) {
    NDState st(xadj, adj, opt, n);
    st.iperm.reserve(n);
    std::vector<idx> all(n);
    std::iota(all.begin(), all.end(), 0);
    st.recurse(all, -1);
    return finish_result(st, n);
}

std::vector<idx> minimum_degree(idx n, const std::vector<idx> &xadj, const std::vector<idx> &adj) {
    // on a quotient graph: an explicit elimination graph (md_local, kept for the small
    // nested-dissection leaves) grows with the fill and is quadratic on whole meshes
    return quotient_minimum_degree(n, xadj, adj);
}

}  // namespace mfs
