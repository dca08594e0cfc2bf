// Internal host state shared by the C-ABI translation units: device buffers,
// the uploaded symbolic analysis, the factor states and the handle itself.
#pragma once
#include "../../include/mfs_b200.h"
#include "device.h"
#include "host_symbolic.h"

#include <cuda_runtime.h>

#include <atomic>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

namespace mfs {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct StatusError : std::runtime_error {
    mfs_status status;
    StatusError(mfs_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

#define MFS_CUDA(call)                                                                                   \
    do {                                                                                                 \
        cudaError_t _e = (call);                                                                         \
        if (_e != cudaSuccess)                                                                           \
            throw CudaError(std::string(#call) + ": " + cudaGetErrorString(_e));                         \
    } while (0)

#define MFS_LAUNCHED() MFS_CUDA(cudaGetLastError())

template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void ensure(size_t count) {
        if (count <= n && p) return;
        release();
        size_t c = std::max<size_t>(count, 1);
        cudaError_t e = cudaMalloc(&p, c * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            throw StatusError(MFS_OOM, std::string("cudaMalloc of ") + std::to_string(c * sizeof(T)) +
                                           " bytes failed: " + cudaGetErrorString(e));
        }
        n = c;
    }
    template <typename U>
    void upload(const std::vector<U> &v, cudaStream_t st) {
        ensure(v.size());
        if (v.empty()) return;
        std::vector<T> tmp(v.begin(), v.end());
        MFS_CUDA(cudaMemcpyAsync(p, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice, st));
        MFS_CUDA(cudaStreamSynchronize(st));
    }
    size_t bytes() const { return n * sizeof(T); }
};


struct LevelPlan {
    int small_off = 0, small_count = 0, small_max_front = 0;
    int all_off = 0, all_count = 0, all_max_front = 0;
    int large_count = 0;
    int asm_off = 0, asm_n = 0, asm_tiles = 0;
    struct Step {
        int left_off, left_n, left_tiles;   // the block's columns updated by the earlier blocks of its group
        int potrf_off, potrf_n, potrf_maxnb;
        int trsm_off, trsm_n, trsm_tiles;   // X := X inv(L)^T of the rows below the block
        int gemm_off, gemm_n, gemm_tiles;   // after a finished group: update of the next group's columns
        int rest_off, rest_n, rest_tiles;   // ... and of the columns after it (overlaps the next group)
    };
    std::vector<Step> steps;
    int syrk_off = 0, syrk_n = 0, syrk_tiles = 0;
    // solve task lists of this level
    int sasm_off = 0, sasm_n = 0, sasm_tiles = 0;
    int ftri_off = 0, ftri_n = 0;
    int btri_off = 0, btri_n = 0;
    int fsb_off = 0, fsb_n = 0, bsb_off = 0, bsb_n = 0;   // superblock diagonal solves (above the cut)
    int fstr_off = 0, fstr_n = 0, fred_off = 0, fred_n = 0;
    int bstr_off = 0, bstr_n = 0, bred_off = 0, bred_n = 0;
};

struct DevSym {
    // unique per upload (never reused, unlike the object's address once it is freed):
    // the key of the caches built from this symbolic data
    uint64_t id = next_id();
    static uint64_t next_id() {
        static std::atomic<uint64_t> counter{0};
        return ++counter;
    }
    std::shared_ptr<Symbolic> S;
    DBuf<int32_t> w, d, f, ld, col0, child_ptr, child_list, struct_rows, rel, small_list, all_list;
    DBuf<int64_t> pan_off, upd_off, sol_off, struct_ptr, diag_off;
    DBuf<int64_t> inv_off;               // 64 x 64 diagonal inverses of large fronts (-1: none)
    DBuf<PlanEntryDev> plan;
    DBuf<PlanEntryDev> plan_cat;         // the same plan in the catamari layout (built on the GPU)
    DBuf<int64_t> plan_ptr_dev;          // its bucket offsets
    DBuf<AssembleTask> asm_tasks;
    DBuf<PanelTask> potrf_tasks;
    DBuf<GemmTask> gemm_tasks;
    DBuf<SolveAsmTask> sasm_tasks;
    DBuf<SolveTask> ftri_tasks, btri_tasks;
    DBuf<StrTask> fstr_tasks, bstr_tasks;
    DBuf<StrReduce> fred, bred;
    DBuf<SbTask> fsb_tasks, bsb_tasks, isb_tasks;   // superblock solves (forward, backward) and inverses
    int nsb_inv = 0;
    std::vector<SbTask> isb_host;                   // the superblocks (their inverses' offsets)
    std::vector<int32_t> sb_fronts;                 // fronts with superblock solves
    int64_t max_str_entries = 0;       // structure partial sums of one level, per right-hand side
    DBuf<int2> subs;                     // subtree ranges solved one per CTA (levels <= solve_cut)
    int nsub = 0, sub_fmax = 0, solve_cut = -1;
    DBuf<int> flags;                     // one per 64-row diagonal block of every front
    DBuf<int64_t> spmv_ptr, spmv_src;
    DBuf<int32_t> spmv_col, spmv_flag;
    DBuf<int64_t> prrfr, sperm;
    std::vector<LevelPlan> levels;
    SnDev sd{};
    int64_t ax_len = 0;
    std::vector<int64_t> Ap_full, Ai_full;   // caller's pattern (for the element slot map)
    DBuf<int64_t> Ap_full_dev, Ai_full_dev;  // the same on the device
    int num_large = 0;
    int64_t inv_scratch = 0;             // elements of the block inverses of one column-block step
    int64_t factor_alloc = 0;            // panels followed by the diagonal inverses
    std::vector<int64_t> dpan;           // device panel offsets (leading dimension padded to 4)
    std::vector<int32_t> dld;            // device panel leading dimensions
    int64_t panel_alloc = 0;             // elements of the padded panels
    std::shared_ptr<void> lpc_graph;     // learned preconditioner: graph arrays (built on first use)
    std::vector<double> gemm_flops_prefix;   // prefix sums of the GEMM tasks' algorithmic flops
    std::vector<int32_t> large_fronts;       // fronts factored by the tiled (GEMM) path
    DBuf<int32_t> large_dev;                 // the same list on the device
    size_t bytes() const {
        return w.bytes() * 5 + col0.bytes() + child_ptr.bytes() + child_list.bytes() + struct_rows.bytes() +
               rel.bytes() + small_list.bytes() + all_list.bytes() + pan_off.bytes() + upd_off.bytes() +
               sol_off.bytes() + struct_ptr.bytes() + diag_off.bytes() + inv_off.bytes() + plan.bytes() + asm_tasks.bytes() +
               potrf_tasks.bytes() + gemm_tasks.bytes() + spmv_ptr.bytes() +
               spmv_src.bytes() + spmv_col.bytes() + spmv_flag.bytes() + prrfr.bytes() + sperm.bytes();
    }
};

struct State {
    std::shared_ptr<DevSym> sym;
    std::shared_ptr<DBuf<double>> f64;
    std::shared_ptr<DBuf<float>> f32;
    std::shared_ptr<DBuf<double>> ax, bx;   // values the numeric factor was computed from
    int type = 0;   // 0 none, 1 symbolic, 2 numeric
    double sigma = 0.0;
};

}  // namespace mfs

using namespace mfs;

struct mfs_handle {
    mfs_options opt{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    State cur, stash;
    bool has_stash = false;
    // FP32 factorizations under refinement use FP32-level (split FP16 / TF32 on tcgen05)
    // products from now on: a low-precision one perturbed a pivot or its refinement
    // stalled. Cleared by a new symbolic analysis and by a change of tensor_cores / refine.
    bool split_escalated = false;
    DBuf<double> upd64;            // update arena (multifrontal Schur complements)
    DBuf<float> upd32;
    DBuf<double> dscr64;           // inverses of the diagonal blocks of one column-block step
    DBuf<float> dscr32;
    DBuf<double> sol;
    DBuf<double> sb_scratch;       // accumulated right-hand sides of the superblock solves (n x pass)
    // tensor maps of the superblock solves, built for the factor array `smaps_base`
    // (element size smaps_es) of the symbolic data `smaps_sym`
    DBuf<TensorMapBlob> smaps;
    const void *smaps_base = nullptr;
    uint64_t smaps_sym = 0;
    int smaps_es = 0;
    std::shared_ptr<DBuf<double>> asm_ax;   // output of the last mfs_assemble (device resident)
    std::shared_ptr<DBuf<double>> asm_spare;   // an earlier assembly buffer, reused once nothing holds it
    DBuf<double> rhs, work_r, work_z, work_p, work_ap, work_x, work_s, io;
    DBuf<double> partials, dots;
    DBuf<int> active;
    DBuf<int> fail;
    DBuf<int> perturbed;          // pivots perturbed in the last numeric factorization
    DBuf<int> refactored;         // FP32 diagonal blocks factored again in FP64 (last numeric)
    DBuf<double> dorig;           // injected diagonal (perturbation reference)
    DBuf<int> solve_err;          // set by a solve kernel whose dependency wait timed out
    DBuf<int> gemm_err;           // set by a tensor-core GEMM whose pipeline wait timed out
    DBuf<double> str_partials;    // chunk partial sums of the solve structure phases (scratch)
    int *fail_host = nullptr;
    double *dots_host = nullptr;
    // assembly
    DBuf<int64_t> slot_ptr, contrib;
    int64_t nslots = 0, nelem = 0;
    DBuf<double> ke;
    std::string err;
    mfs_stats stats{};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::shared_ptr<void> lpc_work;      // learned preconditioner: work buffers (built on first use)
    cudaStream_t side = nullptr;         // high-priority stream of the factorization's column-block chain
    cudaEvent_t ev_ready = nullptr, ev_rest = nullptr, ev_join = nullptr;
    // use_graphs: instantiated graphs of the factorization's launch sequence, keyed by
    // everything the launches bake in (symbolic data, buffers, values, shift)
    struct FactorGraph {
        uint64_t ds;                       // DevSym::id
        const void *factor, *upd, *dscr, *ax, *bx, *dorig, *h16, *h16lo, *tmaps;
        double sigma;
        int split;
        cudaGraphExec_t exec;
    };
    std::vector<FactorGraph> factor_graphs;
    std::shared_ptr<NDResult> nd_prev;       // last nested dissection (temporal reuse)
    std::vector<int64_t> nd_prev_key;        // its block size, block count and sorted pins: reuse needs the same
    int nd_reuse_count = 0;                  // analyses since the last full dissection
    // TMA-fed GEMM: one tensor map per large front's panel (indexed by supernode),
    // built for the array `tmaps_base` (the FP32 factor or its FP16 copy) of the
    // symbolic data `tmaps_sym`
    DBuf<TensorMapBlob> tmaps;
    const void *tmaps_base = nullptr;
    uint64_t tmaps_sym = 0;
    const void *tmaps_lo = nullptr;          // the lo copy the maps after the first nsn cover (split FP16)
    DBuf<uint16_t> h16;                      // FP16 operand copy of the panels (tensor_cores 5, 6)
    DBuf<uint16_t> h16lo;                    // split FP16 (tensor_cores 6): 2^11 x the remainder of h16
    DBuf<int32_t> sexp;                      // per front: power-of-two scale exponent of that copy
    std::vector<cudaEvent_t> gemm_events;    // time_kernels: (start, end) per GEMM launch
    size_t gemm_events_used = 0;
    double gemm_flops_timed = 0.0;
    // time_kernels: per timed GEMM launch {flops, tiles, tasks, kind} (kind: 0 left-looking
    // group update, 1 row solve, 2 next-group update, 3 trailing update, 4 level SYRK)
    std::vector<double> gemm_launch_info;
    std::vector<float> gemm_launch_ms;
};

namespace mfs {
// GPU construction of the pattern-dependent structures (kernels_pattern.cu).
// Block pattern from element stencils (device connectivity, npe <= 32): fills Ap
// (device, nvars + 1) and, when Ai is non-null, Ai (device); returns nnz.
int64_t gpu_build_pattern(int64_t nvars, int64_t nelem, int npe, const int64_t *conn, int64_t *Ap, int64_t *Ai,
                          cudaStream_t st);
// Element -> slot map of the assembly (device connectivity of 4-node elements and
// device full pattern): slot_ptr (nslots + 1) and contrib, as the host map.
void gpu_build_slot_map(int64_t nelem, const int64_t *conn, int64_t nb, const int64_t *Ap, const int64_t *Ai,
                        int64_t nslots, DBuf<int64_t> &slot_ptr, DBuf<int64_t> &contrib, cudaStream_t st);
// Block conversion plan of the analysis, in the device panel layout (plan_dev) and
// in the catamari layout (plan_cat), with its bucket offsets (2 nv + 1).
void gpu_build_plan(const Symbolic &S, const std::vector<int64_t> &dpan, const std::vector<int32_t> &dld,
                    DBuf<PlanEntryDev> &plan_dev, DBuf<PlanEntryDev> &plan_cat, DBuf<int64_t> &plan_ptr,
                    cudaStream_t st);
}  // namespace mfs

inline void set_device(mfs_handle *h) {
    if (h->opt.device < 0) throw StatusError(MFS_INVALID_ARG, "analysis-only handle (device -1) has no GPU state");
    MFS_CUDA(cudaSetDevice(h->opt.device));
}

template <typename F>
mfs_status guarded(mfs_handle *h, F &&fn) {
    try {
        fn();
        if (h) h->err.clear();
        return MFS_OK;
    } catch (const StatusError &e) {
        if (h) h->err = e.what();
        return e.status;
    } catch (const CudaError &e) {
        if (h) h->err = e.what();
        return MFS_CUDA_ERROR;
    } catch (const std::bad_alloc &e) {
        if (h) h->err = "host allocation failed";
        return MFS_OOM;
    } catch (const std::exception &e) {
        if (h) h->err = e.what();
        return MFS_INTERNAL;
    }
}
