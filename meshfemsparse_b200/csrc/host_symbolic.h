// Host-side symbolic analysis for the block-CSC Cholesky path.
//
// Everything here runs once per sparsity pattern on the CPU, exactly where the
// reference runs its symbolic stage (Solvers/CatamariFactorizer.cc:177-616):
// pin removal, ordering, elimination tree, relaxed supernodes, the factor
// storage layout, the child->parent relative index map of the assembly tree and
// the value-injection ("conversion") plan. The numeric stage on the GPU only
// consumes the flat arrays produced here.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace mfs {

using idx = int64_t;

// Upper-triangular compressed-sparse-column pattern: row indices sorted
// ascending inside every column, the diagonal (when present) is the last entry.
struct Pattern {
    idx n = 0;
    std::vector<idx> Ap, Ai;
    idx nnz() const { return Ap.empty() ? 0 : Ap.back(); }
};

// Block sparsity pattern from element stencils (SystemAssembler.hh:252-465):
// every element couples all of its `npe` block variables.
Pattern build_block_pattern(idx nvars, idx nelem, int npe, const idx *conn);

// ---------------------------------------------------------------- ordering --
struct OrderingOptions {
    idx leaf_size = 120;     // stop bisecting below this many vertices
    uint64_t seed = 12345;   // deterministic pseudo-random choices
    int refine_passes = 6;   // FM passes per level
    int init_tries = 8;      // region-growing seeds for the coarsest bisection
};

struct NDResult {
    std::vector<idx> iperm;     // new -> old
    std::vector<idx> cparent;   // separator-tree parent of every component (postordered, -1 root)
    std::vector<idx> cmember;   // component of every (old) vertex
    idx ncomp = 0;
};

// Nested dissection of an undirected graph given as a symmetric adjacency
// structure without self loops.
NDResult nested_dissection(idx n, const std::vector<idx> &xadj, const std::vector<idx> &adj,
                           const OrderingOptions &opt);

// Temporal reuse of a previous dissection of a graph on the same vertices (the
// PARTH idea): the previous separator tree is kept, and only the subtrees whose
// components an edge of the new graph joins (their lowest common ancestor) are
// dissected afresh; leaves are reordered by minimum degree as usual. Falls back to
// a full dissection when `prev` does not match or the new edges leave no subtree to
// keep (*rebuilt_vertices = -1 then), else *rebuilt_vertices = vertices re-dissected.
NDResult nested_dissection_reuse(idx n, const std::vector<idx> &xadj, const std::vector<idx> &adj,
                                 const NDResult &prev, const OrderingOptions &opt, idx *rebuilt_vertices);

// The subtrees of a previous separator forest (cparent postordered, cmember per
// vertex) that a graph on the same vertices violates (persistent_separator_tree.hh:
// 81-118): an edge whose two components are not ancestor and descendant marks their
// lowest common ancestor; `roots` are the marked components without a marked
// ancestor, ascending. An edge between two trees, or one whose ancestor is the root
// of a single-tree forest, asks for a full dissection (`full`, roots empty).
struct DirtySubtrees {
    bool full = false;
    std::vector<idx> roots;
};
DirtySubtrees dirty_subtrees(idx n, const std::vector<idx> &xadj, const std::vector<idx> &adj,
                             const std::vector<idx> &cparent, const std::vector<idx> &cmember);

// Final order of a dissection (hierarchical_camd.cc:165-333): constrained minimum
// degree with the separator forest's components as constraint sets (descendants
// first, each component contiguous), one independent problem per subtree rooted at
// `cut_depth` (clamped to the forest's depth) and one for the separators above,
// which receive every subtree's boundary clique as an initial element. Returns the
// new iperm (nd.iperm unchanged when cut_depth < 0 or the forest does not fit).
struct HierarchicalMDStats {
    bool applied = false;           // false: nd.iperm returned (cut < 0, or the forest does not fit the graph)
    int cut_depth = -1;
    idx tasks = 0, upper_vertices = 0, upper_elements = 0;
};
std::vector<idx> hierarchical_constrained_md(idx n, const std::vector<idx> &xadj, const std::vector<idx> &adj,
                                             const NDResult &nd, int cut_depth, HierarchicalMDStats *stats = nullptr);
// Cut depth of that final order: MFS_ND_CAMD_CUT_DEPTH from the environment (the
// reference reads CHOLMOD_NESDIS_CAMD_CUT_DEPTH), default 4; negative values keep
// the dissection's own order (separators in vertex order, leaves by halo minimum
// degree).
int camd_cut_depth_from_env();

// Minimum degree on a quotient graph (approximate external degrees, element
// absorption, simplicial mass elimination; ties to the lower vertex): the
// constrained engine above with a single constraint set.
std::vector<idx> quotient_minimum_degree(idx n, const std::vector<idx> &xadj, const std::vector<idx> &adj);

// Minimum-degree order of the whole graph (the AMD-style mode).
std::vector<idx> minimum_degree(idx n, const std::vector<idx> &xadj, const std::vector<idx> &adj);

// ---------------------------------------------------------------- symbolic --
enum OrderingMethod : int {
    ORDER_ND = 0,        // nested dissection (default, as CholmodNesdisParallel)
    ORDER_NATIVE = 1,    // input order, relaxation must not reorder (CatamariNative)
    ORDER_MD = 2,        // minimum degree (as CatamariAMD)
    ORDER_USER = 3,      // caller-supplied permutation
};

struct SymbolicOptions {
    int ordering = ORDER_ND;
    bool relax = true;               // relax_supernodes (CatamariFactorizer.cc:105)
    idx relax_zeros = 128;           // allowable explicit zeros per relaxed supernode
    double relax_ratio = 0.01;       // alternative allowance: zeros / stored entries
    OrderingOptions nd;
    const NDResult *nd_prev = nullptr;   // reuse this dissection's separator tree (same vertices)
    idx solve_subtrees = 0;          // subtree count the solve cut aims for (0: max(2368, 48 per tree))
};

// One conversion-plan entry: copy a vb x vb block of the user's value array
// into the factor storage. `src` addresses the upper-left value of the block in
// the caller's Ax array, `dst` the upper-left value in the factor, `ld` is the
// leading dimension of the destination panel. flags bit0: source must be
// transposed (block read from the lower triangle); bit1: destination is a
// diagonal block (only r >= c is written).
struct PlanEntry {
    idx dst;
    idx src;
    int32_t ld;
    int32_t flags;
};

struct Symbolic {
    int bs = 3;            // block size of the caller's matrix
    int vb = 3;            // block size the analysis runs at (bs, or 1 on the scalar fallback)
    idx n_full = 0;        // scalar rows of the caller's matrix
    idx n = 0;             // scalar rows after pin removal
    idx nv_full = 0, nv = 0;   // analysis variables (full / reduced)

    // Pins (CholeskyFactorizerBase.hh:402-426, CatamariFactorizer.cc:187-246)
    std::vector<idx> fixed_vars;            // sorted unique scalar pins
    std::vector<idx> reduced_row_for_row;   // scalar, size n_full, -1 when pinned
    std::vector<idx> permuted_reduced_row_for_row;  // scalar, size n_full, -1 when pinned

    // Reduced analysis pattern (upper CSC) and source offset of each entry in Ax.
    Pattern A;                              // over nv analysis variables
    std::vector<idx> src_off;               // per entry: Ax offset of the vb x vb block's upper-left
    int src_ld = 3;                         // column stride of a source block in Ax (bs for contiguous blocks)

    // Ordering at analysis-variable granularity.
    std::vector<idx> perm, iperm;           // perm[old] = new, iperm[new] = old
    std::vector<idx> scalar_perm, scalar_iperm;   // expanded to reduced scalar indices

    // ND separator tree snapshot (CholeskyFactorizerBase.hh:55-59).
    std::vector<idx> nd_cparent, nd_cmember;
    idx nd_ncomp = 0;
    idx nd_rebuilt = -1;                    // reused dissection: vertices re-dissected (-1: full dissection)

    // Supernodes (postordered; children precede parents).
    idx nsn = 0;
    std::vector<idx> sn_start;              // analysis-variable column start, size nsn+1
    std::vector<idx> sn_parent;             // -1 for roots
    std::vector<idx> child_ptr, child_list; // children of every supernode (ascending)
    std::vector<idx> struct_ptr, struct_rows;   // below-diagonal rows (analysis vars, permuted)

    // Scalar factor layout: panel s is (w+d) x w, column-major, ld = w+d.
    std::vector<idx> w, d, f;               // scalar width, degree, front size
    std::vector<idx> pan_off;               // offset of panel s in the factor value array
    idx factor_size = 0;                    // total stored values (sum f*w)
    idx factor_nnz = 0;                     // sum w(w+1)/2 + w*d (GetFactorNNZ)
    double flops = 0;                       // sum w^3/3 + w^2 d + w d^2 (EstimateTotalWork)

    // Assembly tree relative indices (child_rel_indices): one per struct entry,
    // scalar row inside the parent's front; and the count of those landing in
    // the parent's diagonal block (num_child_diag_indices, scalar).
    std::vector<int32_t> rel;
    std::vector<idx> num_child_diag;

    // Level schedule (height in the assembly tree; leaves are level 0).
    std::vector<int32_t> level;
    idx nlevels = 0;
    std::vector<idx> level_ptr, level_list;

    // Update-matrix arena: U_s (d x d, ld d) lives at upd_off[s] during the
    // levels [level(s), level(parent(s))].
    std::vector<idx> upd_off;
    idx upd_size = 0;
    // Forward-solve update vectors u_s (d x nrhs), unit size d: offsets here are
    // scaled by nrhs at solve time. Supernodes at levels <= solve_cut are solved
    // by whole subtrees (contiguous postorder ranges [sub_lo, sub_hi], largest
    // work first, fronts of at most sub_fmax rows), so their u_s live from the
    // start of the solve until their parent's level.
    std::vector<idx> sol_off;
    idx sol_size = 0;
    idx solve_cut = -1;
    std::vector<idx> sub_lo, sub_hi;
    idx sub_fmax = 0;

    // Conversion plan (CatamariConversionPlan.hh:402-541): entries grouped by
    // permuted analysis column, two buckets per column (transposed, copied).
    std::vector<idx> plan_ptr;              // size 2*nv+1
    std::vector<PlanEntry> plan;

    // Symmetric SpMV structure over permuted reduced block rows: for row i the
    // entries (source offset, permuted column, transpose flag).
    std::vector<idx> spmv_ptr;
    std::vector<idx> spmv_src;
    std::vector<int32_t> spmv_col;
    std::vector<int32_t> spmv_flag;         // bit0 transpose, bit1 diagonal (stored upper only)
};

// Full symbolic analysis. `Ap/Ai` is the caller's block (or scalar when bs==1)
// upper pattern over n_full/bs block variables; pins are scalar indices.
// Returns an empty string on success, else the error message.
// `user_sn_sizes` (optional, with ORDER_NATIVE / ORDER_USER): supernode sizes in
// analysis variables, replacing fundamental + relaxed supernode detection;
// every supernode must be a chain of the elimination tree.
std::string analyze(idx nblocks, const idx *Ap, const idx *Ai, int bs, const idx *pinned, idx npinned,
                    const SymbolicOptions &opt, const idx *user_perm, Symbolic &S,
                    const idx *user_sn_sizes = nullptr, idx n_user_sn = 0);

}  // namespace mfs
