// C ABI (include/mfs_b200.h): handle lifetime, symbolic upload, the level
// schedule of the numeric factorization, solves, FP64 refinement, element
// assembly and the factor stash. Host logic only; kernels live in
// kernels_factor.cu / kernels_solve.cu.
#include "../../include/mfs_b200.h"
#include "../../include/mfs_b200_testing.h"
#include "device.h"
#include "handle.h"
#include "host_symbolic.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <type_traits>
#include <stdexcept>
#include <string>
#include <vector>

namespace mfs {
long long g_kernel_launches = 0;

int current_device() {
    int d = 0;
    if (cudaGetDevice(&d) != cudaSuccess) return 0;
    return d;
}

int device_sm_count() {
    static int sms[kMaxDevices] = {};
    static PerDeviceOnce once;
    const int d = current_device();
    if (d < 0 || d >= kMaxDevices) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
        return v;
    }
    once([&] { cudaDeviceGetAttribute(&sms[d], cudaDevAttrMultiProcessorCount, d); });
    return sms[d];
}
}  // namespace mfs

using namespace mfs;

namespace {

// Fronts up to this size are factored whole in one CTA's shared memory (f x f entries).
int small_front_limit(const mfs_handle *h) {
    const int el = h->opt.precision == MFS_PREC_FP32 ? 4 : 8;
    const int cap = int(std::sqrt(double(kMaxSmemOptin) / el));
    if (h->opt.small_front_max > cap)
        throw StatusError(MFS_INVALID_ARG, "small_front_max above " + std::to_string(cap) +
                                               " (a front must fit one CTA's shared memory)");
    if (h->opt.small_front_max > 0) return h->opt.small_front_max;
    return h->opt.precision == MFS_PREC_FP32 ? 160 : 128;
}

std::shared_ptr<DevSym> upload_symbolic(mfs_handle *h, std::shared_ptr<Symbolic> Sp) {
    const Symbolic &S = *Sp;
    cudaStream_t st = h->stream;
    auto ds = std::make_shared<DevSym>();
    ds->S = Sp;
    const idx nsn = S.nsn;
    std::vector<int32_t> col0(nsn), w32(nsn), d32(nsn), f32v(nsn);
    for (idx s = 0; s < nsn; ++s) {
        col0[s] = int32_t(S.vb * S.sn_start[s]);
        w32[s] = int32_t(S.w[s]);
        d32[s] = int32_t(S.d[s]);
        f32v[s] = int32_t(S.f[s]);
    }
    // Device panel layout: the catamari panel with its leading dimension rounded up
    // to a multiple of 8, so every column starts 16-byte aligned, in the factor and in
    // the half-precision operand copy of an FP32 factor alike.
    ds->dpan.assign(nsn + 1, 0);
    ds->dld.assign(nsn, 0);
    for (idx s = 0; s < nsn; ++s) {
        ds->dld[s] = int32_t((S.f[s] + 7) & ~idx(7));
        ds->dpan[s + 1] = ds->dpan[s] + int64_t(ds->dld[s]) * S.w[s];
    }
    ds->panel_alloc = ds->dpan[nsn];
    const std::vector<int64_t> &dpan = ds->dpan;
    const std::vector<int32_t> &dld = ds->dld;
    ds->w.upload(w32, st);
    ds->d.upload(d32, st);
    ds->f.upload(f32v, st);
    ds->ld.upload(dld, st);
    ds->col0.upload(col0, st);
    ds->child_ptr.upload(S.child_ptr, st);
    ds->child_list.upload(S.child_list, st);
    ds->struct_rows.upload(S.struct_rows, st);
    ds->rel.upload(S.rel, st);
    ds->pan_off.upload(dpan, st);
    ds->upd_off.upload(S.upd_off, st);
    ds->sol_off.upload(S.sol_off, st);
    ds->struct_ptr.upload(S.struct_ptr, st);
    std::vector<int64_t> diag(S.n);
    for (idx s = 0; s < nsn; ++s)
        for (idx k = 0; k < S.w[s]; ++k) diag[S.vb * S.sn_start[s] + k] = dpan[s] + k * dld[s] + k;
    ds->diag_off.upload(diag, st);
    {
        // the block conversion plan, built on the GPU from the reduced pattern, the
        // ordering and the supernodes, in the padded device layout (and the catamari
        // layout, exported by mfs_conversion_plan_device)
        gpu_build_plan(S, dpan, dld, ds->plan, ds->plan_cat, ds->plan_ptr_dev, st);
    }
    ds->spmv_ptr.upload(S.spmv_ptr, st);
    ds->spmv_src.upload(S.spmv_src, st);
    ds->spmv_col.upload(S.spmv_col, st);
    ds->spmv_flag.upload(S.spmv_flag, st);
    ds->prrfr.upload(S.permuted_reduced_row_for_row, st);
    ds->sperm.upload(S.scalar_perm, st);

    // level schedule and tiled task lists
    const int small_max = small_front_limit(h);
    std::vector<int32_t> small_list, all_list;
    std::vector<AssembleTask> asm_tasks;
    std::vector<PanelTask> potrf_tasks;
    std::vector<GemmTask> gemm_tasks;
    ds->levels.resize(S.nlevels);
    ds->num_large = 0;
    std::vector<int64_t> inv_off(nsn, -1);
    int64_t inv_end = ds->panel_alloc;
    for (idx l = 0; l < S.nlevels; ++l) {
        LevelPlan &L = ds->levels[l];
        std::vector<idx> large;
        L.small_off = int(small_list.size());
        L.all_off = int(all_list.size());
        for (idx k = S.level_ptr[l]; k < S.level_ptr[l + 1]; ++k) {
            idx s = S.level_list[k];
            all_list.push_back(int32_t(s));
            L.all_max_front = std::max<int>(L.all_max_front, int(S.f[s]));
            if (S.f[s] <= small_max) {
                small_list.push_back(int32_t(s));
                L.small_max_front = std::max<int>(L.small_max_front, int(S.f[s]));
            } else large.push_back(s);
        }
        L.small_count = int(small_list.size()) - L.small_off;
        L.all_count = int(all_list.size()) - L.all_off;
        L.large_count = int(large.size());
        ds->num_large += L.large_count;
        if (large.empty()) continue;
        L.asm_off = int(asm_tasks.size());
        int base = 0;
        idx maxw = 0;
        for (idx s : large) {
            ds->large_fronts.push_back(int32_t(s));
            inv_off[s] = inv_end;
            inv_end += ((S.w[s] + 63) / 64) * 4096;
            asm_tasks.push_back({int32_t(s), base});
            base += int((S.f[s] + kAsmCols - 1) / kAsmCols);
            maxw = std::max(maxw, S.w[s]);
        }
        L.asm_n = int(large.size());
        L.asm_tiles = base;
        const bool f64 = h->opt.precision != MFS_PREC_FP32;
        const int NB = f64 ? 64 : 128;                  // column block of the large-front factorization
        const int TM = gemm_tile_m(f64), TN = gemm_tile_n(f64);
        // The in-place row solve needs every CTA tile to span the block's columns
        // (with the FP32 tiles' alignment shift of up to 3 columns).
        if (NB + (f64 ? 0 : 7) > TN) throw StatusError(MFS_INTERNAL, "column block wider than the GEMM tile");
        // sn: the front of the task; for a mode-0 task its panel holds A and B, which the
        // TMA-fed kernel reads through the panel's tensor map
        auto gemm = [&](int64_t a_off, int64_t b_off, int64_t c_off, int lda, int ldb, int ldc, idx m, idx n, idx k,
                        int lower, int mode, int &base, idx sn) {
            GemmTask g{};
            g.a_off = a_off; g.b_off = b_off; g.c_off = c_off;
            g.lda = lda; g.ldb = ldb; g.ldc = ldc;
            g.m = int32_t(m); g.n = int32_t(n); g.k = int32_t(k);
            // FP32 operands (and their FP16 copies) are staged in 16-byte chunks: a
            // tile starts at the 8-element aligned element at or before the operand
            // (panel leading dimensions are multiples of 8, so the shift is the same
            // for every column).
            int da = 0, db = 0;
            if (!f64) {
                if ((lda & 3) || (ldb & 3)) throw StatusError(MFS_INTERNAL, "unaligned GEMM operand");
                da = int(a_off & 7);
                db = int(b_off & 7);
            }
            g.shift = da | (db << 8);
            g.tiles_m = int32_t((m + da + TM - 1) / TM);
            g.tiles_n = int32_t((n + db + TN - 1) / TN);
            g.tile_base = base;
            g.lower = lower;
            g.mode = mode;
            g.amap = g.bmap = -1;
            g.sn = int32_t(sn);
            if (!f64 && mode == 0 && sn >= 0) {
                const int64_t ra = a_off - dpan[sn], rb = b_off - dpan[sn];
                g.amap = g.bmap = int32_t(sn);
                g.ax = int32_t(ra % dld[sn]) - da;
                g.ay = int32_t(ra / dld[sn]);
                g.bx = int32_t(rb % dld[sn]) - db;
                g.by = int32_t(rb / dld[sn]);
            }
            base += g.tiles_m * g.tiles_n;
            gemm_tasks.push_back(g);
        };
        // Column blocks of NB are grouped by GB = factor_group NB (default 4): inside a group the block
        // columns are brought up to date left-looking (one GEMM with k = kb - group
        // start), after a group the rest of the front gets one rank-GB update. The
        // Schur updates so run with k up to GB instead of NB, reading and writing
        // the trailing columns GB / NB times less often.
        const idx GB = idx(h->opt.factor_group > 0 ? h->opt.factor_group : 4) * NB;
        for (idx kb = 0; kb < maxw; kb += NB) {
            LevelPlan::Step sp{};
            const idx ko = kb - kb % GB;                // start of the block's group
            sp.left_off = int(gemm_tasks.size());
            int lb = 0;
            if (kb > ko)
                for (idx s : large) {
                    const idx w = S.w[s], f = S.f[s], ld = dld[s], pan = dpan[s];
                    if (w <= kb) continue;
                    const int nb = int(std::min<idx>(NB, w - kb));
                    const int64_t a = pan + ko * ld + kb;
                    gemm(a, a, pan + kb * ld + kb, int(ld), int(ld), int(ld), f - kb, nb, kb - ko, 1, 0, lb, s);
                }
            sp.left_n = int(gemm_tasks.size()) - sp.left_off;
            sp.left_tiles = lb;
            sp.potrf_off = int(potrf_tasks.size());
            int64_t dslot = 0;
            for (idx s : large) {
                const idx w = S.w[s], ld = dld[s], pan = dpan[s];
                if (w <= kb) continue;
                const int nb = int(std::min<idx>(NB, w - kb));
                PanelTask pt{};
                pt.off = pan + kb * ld + kb;
                pt.ldi = (nb + 3) & ~3;
                pt.inv_full = dslot;
                dslot += int64_t(pt.ldi) * nb;
                pt.inv_out = inv_off[s] + (kb / 64) * 4096;
                pt.ld = int32_t(ld);
                pt.nb = nb;
                pt.col = int32_t(col0[s] + kb);
                potrf_tasks.push_back(pt);
                sp.potrf_maxnb = std::max(sp.potrf_maxnb, nb);
            }
            sp.potrf_n = int(potrf_tasks.size()) - sp.potrf_off;
            ds->inv_scratch = std::max<int64_t>(ds->inv_scratch, dslot);
            // rows below the diagonal block: X := X inv(L)^T (in place; one CTA tile spans all nb columns)
            sp.trsm_off = int(gemm_tasks.size());
            int tb = 0;
            {
                int q = sp.potrf_off;
                for (idx s : large) {
                    if (S.w[s] <= kb) continue;
                    const PanelTask &pt = potrf_tasks[q++];
                    const idx m = S.f[s] - (kb + pt.nb);   // rows of the front below the block
                    if (m > 0)
                        gemm(pt.off + pt.nb, pt.inv_full, pt.off + pt.nb, pt.ld, pt.ldi, pt.ld, m, pt.nb, pt.nb, 0, 1,
                             tb, s);
                }
            }
            sp.trsm_n = int(gemm_tasks.size()) - sp.trsm_off;
            sp.trsm_tiles = tb;
            // after the last block of a group: update the columns after the group, the next
            // group's GB columns apart from the rest, so that the next group's panels can
            // start while the rest is updated (one-group look-ahead)
            sp.gemm_off = int(gemm_tasks.size());
            int gb = 0;
            std::vector<idx> rest_fronts;
            for (idx s : large) {
                const idx w = S.w[s], f = S.f[s], ld = dld[s], pan = dpan[s];
                if (w <= kb) continue;
                const idx ke = std::min<idx>(kb + NB, w);          // end of this block
                if (ke != std::min<idx>(ko + GB, w) || ke >= w) continue;
                const int64_t a = pan + ko * ld + ke;
                gemm(a, a, pan + ke * ld + ke, int(ld), int(ld), int(ld), f - ke, std::min<idx>(GB, w - ke), ke - ko,
                     1, 0, gb, s);
                if (ke + GB < w) rest_fronts.push_back(s);
            }
            sp.gemm_n = int(gemm_tasks.size()) - sp.gemm_off;
            sp.gemm_tiles = gb;
            sp.rest_off = int(gemm_tasks.size());
            int rb = 0;
            for (idx s : rest_fronts) {
                const idx w = S.w[s], f = S.f[s], ld = dld[s], pan = dpan[s];
                const idx ke = std::min<idx>(kb + NB, w), kr = ke + GB;
                const int64_t a = pan + ko * ld + kr;
                gemm(a, a, pan + kr * ld + kr, int(ld), int(ld), int(ld), f - kr, w - kr, ke - ko, 1, 0, rb, s);
            }
            sp.rest_n = int(gemm_tasks.size()) - sp.rest_off;
            sp.rest_tiles = rb;
            L.steps.push_back(sp);
        }
        L.syrk_off = int(gemm_tasks.size());
        int sb = 0;
        for (idx s : large) {
            if (S.d[s] == 0 || S.upd_off[s] < 0) continue;
            const int64_t a = dpan[s] + S.w[s];
            gemm(a, a, S.upd_off[s], dld[s], dld[s], int(S.d[s]), S.d[s], S.d[s], S.w[s], 1, 0, sb, s);
        }
        L.syrk_n = int(gemm_tasks.size()) - L.syrk_off;
        L.syrk_tiles = sb;
    }
    // ---- solve tasks (all supernodes, level by level)
    const int RB = solve_rows_per_task();
    const int DG = diag_blocks_per_task();
    std::vector<int32_t> flag_base(nsn);
    int nflags = 0;
    for (idx s = 0; s < nsn; ++s) {
        flag_base[s] = nflags;
        nflags += int((S.w[s] + RB - 1) / RB);
    }
    // Superblock diagonal solves of the levels above the solve cut: one flag and one
    // stored inverse (nrp x nrp, after the 64 x 64 diagonal inverses) per superblock.
    std::vector<SbTask> fsb, bsb, isb;
    std::vector<int32_t> sb_flag(nsn, -1);
    std::vector<int64_t> sb_inv(nsn, -1);
    std::vector<int32_t> sb_first(nsn, -1);
    ds->sb_fronts.clear();
    int nsbflags = 0;
    const idx SBk = kSuperBlock;
    for (idx l = S.solve_cut + 1; l < S.nlevels; ++l)
        for (idx k = S.level_ptr[l]; k < S.level_ptr[l + 1]; ++k) {
            const idx s = S.level_list[k];
            const idx nsb = (S.w[s] + SBk - 1) / SBk;
            sb_flag[s] = nsbflags;
            nsbflags += 2 * int(nsb);
            sb_inv[s] = inv_end;
            sb_first[s] = int32_t(isb.size());
            ds->sb_fronts.push_back(int32_t(s));
            for (idx K = 0; K < nsb; ++K) {
                const idx nr = std::min(SBk, S.w[s] - K * SBk), nrp = (nr + 63) & ~idx(63);
                isb.push_back({int32_t(s), int32_t(K), sb_flag[s], 0, inv_end, -1, -1});
                inv_end += nrp * nrp;
            }
        }
    // tensor maps of the solves: two per superblock inverse, then two per front
    const int32_t nsbm = int32_t(isb.size());
    std::vector<int32_t> sb_fidx(nsn, -1);
    for (size_t i = 0; i < ds->sb_fronts.size(); ++i) sb_fidx[ds->sb_fronts[i]] = int32_t(i);
    // every superblock before a front's last is full (SB x SB)
    auto sb_task = [&](idx s, idx K, idx part) {
        return SbTask{int32_t(s),         int32_t(K), sb_flag[s], int32_t(part), sb_inv[s] + K * SBk * SBk,
                      2 * (nsbm + sb_fidx[s]), 2 * (sb_first[s] + int32_t(K))};
    };
    auto sb_parts = [&](idx s, idx K) { return (std::min(SBk, S.w[s] - K * SBk) + 63) / 64; };
    std::vector<SolveAsmTask> sasm;
    std::vector<SolveTask> ftri, btri;
    std::vector<StrTask> fstr, bstr;
    std::vector<StrReduce> fred, bred;
    int64_t max_str = 0;                          // partial-sum entries of one level and one right-hand side
    for (idx l = 0; l < S.nlevels; ++l) {
        LevelPlan &L = ds->levels[l];
        L.sasm_off = int(sasm.size());
        L.ftri_off = int(ftri.size());
        L.btri_off = int(btri.size());
        int base = 0, maxblk = 0, maxnbw = 0;
        for (idx k = S.level_ptr[l]; k < S.level_ptr[l + 1]; ++k) {
            const idx s = S.level_list[k];
            if (S.child_ptr[s + 1] > S.child_ptr[s] || S.d[s] > 0) {
                sasm.push_back({int32_t(s), base});
                base += int((S.f[s] + kSolveAsmRows - 1) / kSolveAsmRows);
            }
            const int nbw = int((S.w[s] + RB - 1) / RB), nbd = int((S.d[s] + RB - 1) / RB);
            maxblk = std::max(maxblk, nbw + nbd);
            maxnbw = std::max(maxnbw, (nbw + DG - 1) / DG);
        }
        L.sasm_n = int(sasm.size()) - L.sasm_off;
        L.sasm_tiles = base;
        // ascending task (block pair) index across the level's fronts: every dependency
        // precedes its task
        for (int b = 0; b < maxnbw; ++b)
            for (idx k = S.level_ptr[l]; k < S.level_ptr[l + 1]; ++k) {
                const idx s = S.level_list[k];
                const int nlk = int((S.w[s] + RB * DG - 1) / (RB * DG));
                if (b < nlk) ftri.push_back({int32_t(s), b, flag_base[s], 0});
            }
        // structure slabs (rows from w rounded down to a multiple of 4): forward kStrRows-row
        // slabs x kStrCols-column chunks, backward kStrBCols-column slabs x row chunks
        L.fstr_off = int(fstr.size());
        L.fred_off = int(fred.size());
        L.bstr_off = int(bstr.size());
        L.bred_off = int(bred.size());
        const idx brows = str_bwd_rows(h->opt.precision != MFS_PREC_FP32);
        for (idx k = S.level_ptr[l]; k < S.level_ptr[l + 1]; ++k) {
            const idx s = S.level_list[k];
            if (S.d[s] == 0) continue;
            const idx span = S.f[s] - (S.w[s] & ~idx(3));
            const int nrs = int((span + kStrRows - 1) / kStrRows), ncs = int((S.w[s] + kStrCols - 1) / kStrCols);
            for (int a = 0; a < nrs; ++a) {
                fred.push_back({int32_t(s), a, int32_t(fstr.size()) - L.fstr_off, ncs});
                for (int c = 0; c < ncs; ++c) fstr.push_back({int32_t(s), a, c, 0});
            }
            const int nws = int((S.w[s] + kStrBCols - 1) / kStrBCols), nds = int((span + brows - 1) / brows);
            for (int a = 0; a < nws; ++a) {
                bred.push_back({int32_t(s), a, int32_t(bstr.size()) - L.bstr_off, nds});
                for (int c = 0; c < nds; ++c) bstr.push_back({int32_t(s), a, c, 0});
            }
        }
        L.fstr_n = int(fstr.size()) - L.fstr_off;
        L.fred_n = int(fred.size()) - L.fred_off;
        L.bstr_n = int(bstr.size()) - L.bstr_off;
        L.bred_n = int(bred.size()) - L.bred_off;
        max_str = std::max<int64_t>(max_str, std::max(int64_t(L.fstr_n) * kStrRows, int64_t(L.bstr_n) * kStrBCols));
        for (int p = 0; p < maxnbw; ++p)
            for (idx k = S.level_ptr[l]; k < S.level_ptr[l + 1]; ++k) {
                const idx s = S.level_list[k];
                const int nlk = int((S.w[s] + RB * DG - 1) / (RB * DG));
                if (p < nlk) btri.push_back({int32_t(s), nlk - 1 - p, flag_base[s], 0});
            }
        L.ftri_n = int(ftri.size()) - L.ftri_off;
        L.btri_n = int(btri.size()) - L.btri_off;
        // superblock tasks, one per 64-row part: ascending superblock index across the
        // level's fronts (forward), descending (backward); every dependency precedes
        // its task and the parts of a superblock are adjacent
        L.fsb_off = int(fsb.size());
        L.bsb_off = int(bsb.size());
        if (l > S.solve_cut) {
            idx maxnsb = 0;
            for (idx k = S.level_ptr[l]; k < S.level_ptr[l + 1]; ++k)
                maxnsb = std::max<idx>(maxnsb, (S.w[S.level_list[k]] + SBk - 1) / SBk);
            for (idx K = 0; K < maxnsb; ++K)
                for (idx k = S.level_ptr[l]; k < S.level_ptr[l + 1]; ++k) {
                    const idx s = S.level_list[k];
                    if (K < (S.w[s] + SBk - 1) / SBk)
                        for (idx part = 0; part < sb_parts(s, K); ++part) fsb.push_back(sb_task(s, K, part));
                }
            for (idx p = 0; p < maxnsb; ++p)
                for (idx k = S.level_ptr[l]; k < S.level_ptr[l + 1]; ++k) {
                    const idx s = S.level_list[k];
                    const idx nsb = (S.w[s] + SBk - 1) / SBk;
                    if (p < nsb)
                        for (idx part = 0; part < sb_parts(s, nsb - 1 - p); ++part)
                            bsb.push_back(sb_task(s, nsb - 1 - p, part));
                }
        }
        L.fsb_n = int(fsb.size()) - L.fsb_off;
        L.bsb_n = int(bsb.size()) - L.bsb_off;
    }
    ds->small_list.upload(small_list, st);
    ds->large_dev.upload(ds->large_fronts, st);
    ds->all_list.upload(all_list, st);
    ds->inv_off.upload(inv_off, st);
    // (+64: the solves' 16-byte loads of a panel column may reach 3 elements past its end)
    ds->factor_alloc = inv_end + 64;
    auto up = [&](auto &buf, const auto &vec) {
        buf.ensure(vec.size());
        if (!vec.empty())
            MFS_CUDA(cudaMemcpyAsync(buf.p, vec.data(), vec.size() * sizeof(vec[0]), cudaMemcpyHostToDevice, st));
    };
    up(ds->asm_tasks, asm_tasks);
    up(ds->potrf_tasks, potrf_tasks);
    up(ds->gemm_tasks, gemm_tasks);
    // algorithmic flops per task: 2 m n k for an update (the lower triangle only for
    // lower tasks, whose block starts on the diagonal), m n k for a row solve by inv(L)
    ds->gemm_flops_prefix.assign(gemm_tasks.size() + 1, 0.0);
    for (size_t t = 0; t < gemm_tasks.size(); ++t) {
        const GemmTask &g = gemm_tasks[t];
        const double m = g.m, n = g.n, k = g.k;
        double fl = g.mode == 1 ? m * n * k : 2.0 * m * n * k;
        if (g.lower && g.mode == 0) fl = 2.0 * k * (m * n - std::min(m, n) * (std::min(m, n) - 1.0) / 2.0);
        ds->gemm_flops_prefix[t + 1] = ds->gemm_flops_prefix[t] + fl;
    }
    up(ds->sasm_tasks, sasm);
    up(ds->ftri_tasks, ftri);
    up(ds->btri_tasks, btri);
    up(ds->fstr_tasks, fstr);
    up(ds->bstr_tasks, bstr);
    up(ds->fred, fred);
    up(ds->bred, bred);
    up(ds->fsb_tasks, fsb);
    up(ds->bsb_tasks, bsb);
    up(ds->isb_tasks, isb);
    ds->nsb_inv = int(isb.size());
    ds->isb_host = isb;
    ds->max_str_entries = max_str;
    {
        std::vector<int2> sv(S.sub_lo.size());
        for (size_t k = 0; k < sv.size(); ++k) sv[k] = make_int2(int(S.sub_lo[k]), int(S.sub_hi[k]));
        up(ds->subs, sv);
        ds->nsub = int(sv.size());
        ds->sub_fmax = int(S.sub_fmax);
        ds->solve_cut = int(S.solve_cut);
    }
    ds->flags.ensure(size_t(std::max(std::max(nflags, nsbflags), 1)));
    MFS_CUDA(cudaMemsetAsync(ds->flags.p, 0, ds->flags.bytes(), st));
    MFS_CUDA(cudaStreamSynchronize(st));

    SnDev &sd = ds->sd;
    sd.w = ds->w.p;
    sd.d = ds->d.p;
    sd.f = ds->f.p;
    sd.col0 = ds->col0.p;
    sd.pan_off = ds->pan_off.p;
    sd.upd_off = ds->upd_off.p;
    sd.sol_off = ds->sol_off.p;
    sd.ld = ds->ld.p;
    sd.inv_off = ds->inv_off.p;
    sd.child_ptr = ds->child_ptr.p;
    sd.child_list = ds->child_list.p;
    sd.struct_ptr = ds->struct_ptr.p;
    sd.struct_rows = ds->struct_rows.p;
    sd.rel = ds->rel.p;
    sd.vb = S.vb;
    return ds;
}

void ensure_side_stream(mfs_handle *h) {
    if (h->side) return;
    int least = 0, greatest = 0;
    MFS_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    MFS_CUDA(cudaStreamCreateWithPriority(&h->side, cudaStreamNonBlocking, greatest));
    MFS_CUDA(cudaEventCreateWithFlags(&h->ev_ready, cudaEventDisableTiming));
    MFS_CUDA(cudaEventCreateWithFlags(&h->ev_rest, cudaEventDisableTiming));
    MFS_CUDA(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
}

void clear_factor_graphs(mfs_handle *h) {
    for (auto &g : h->factor_graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    h->factor_graphs.clear();
}

// FP32 Schur updates: 1 = single-pass TF32 on tcgen05 (cp.async operands), 4 = the same
// with TMA-fed operands for the updates (mode 0) and cp.async for the row solves,
// 5 = FP16 operands (a per-front power-of-two scaled half copy of the panels, written
// by the row solves) on tcgen05 kind::f16 with TMA for the updates, 6 = split FP16
// (hi and 2^11-scaled lo half copies, three MMAs per k slice; row solves in split
// TF32 on tcgen05): FP32-level products, 3 = split 3xTF32 (mma.sync), 0 = single-pass
// TF32 on mma.sync. Option values: tensor_cores 0 (auto: 6 with refinement, else 3),
// 1, 2 (-> 3), 3 (-> 0), 4, 5 and 6 (with refinement, else 3). The automatic choice
// is split FP16: its FP32-level factor needs 3-4 refinement iterations where the
// single-pass modes need 6-7, which outweighs its dearer Schur updates as soon as the
// solves carry several right-hand sides, and it never needs escalating.
// FP16 operands are safe under refinement: |L(i, j)| <= sqrt(A(j, j)) for an SPD
// matrix, so the per-front scale keeps every operand below 2^12 (no overflow), and
// the refinement needs the same iteration count as with TF32 operands.
int fp32_split(const mfs_handle *h) {
    if (h->split_escalated) return 6;
    const int tc = h->opt.tensor_cores;
    if (tc == 6 || tc == 0) return h->opt.refine ? 6 : 3;
    if (tc == 5) return h->opt.refine ? 5 : 3;
    return tc == 1 ? 1 : tc == 2 ? 3 : tc == 3 ? 0 : 4;
}

// Tensor maps of the large fronts' panels in `base` (the FP32 factor, or its FP16
// copy) for the TMA-fed GEMM (built on the host once per symbolic analysis and
// array; not during graph capture).
void ensure_panel_maps(mfs_handle *h, DevSym &ds, const void *base, bool half, const void *lo = nullptr) {
    if (h->tmaps_base == base && h->tmaps_sym == ds.id && h->tmaps_lo == lo) return;
    const Symbolic &S = *ds.S;
    const size_t es = half ? 2 : 4;
    const size_t nsn = size_t(std::max<idx>(S.nsn, 1));
    // [0, nsn): the copy at base; [nsn, 2 nsn): the lo copy (split FP16)
    std::vector<TensorMapBlob> maps(lo ? 2 * nsn : nsn);
    std::memset(maps.data(), 0, maps.size() * sizeof(TensorMapBlob));
    for (int c = 0; c < (lo ? 2 : 1); ++c) {
        const char *b = static_cast<const char *>(c ? lo : base);
        for (int32_t s : ds.large_fronts)
            if (!encode_operand_map(&maps[c * nsn + size_t(s)], b + size_t(ds.dpan[s]) * es, lo ? 2 : half ? 1 : 0,
                                    uint64_t(S.f[s]),
                                    uint64_t(S.w[s]), uint64_t(ds.dld[s])))
                throw StatusError(MFS_INTERNAL, "cuTensorMapEncodeTiled refused a panel tensor map");
    }
    h->tmaps.ensure(maps.size());
    MFS_CUDA(cudaMemcpyAsync(h->tmaps.p, maps.data(), maps.size() * sizeof(TensorMapBlob), cudaMemcpyHostToDevice,
                             h->stream));
    MFS_CUDA(cudaStreamSynchronize(h->stream));
    h->tmaps_base = base;
    h->tmaps_sym = ds.id;
    h->tmaps_lo = lo;
}

// Tensor maps of the superblock solves for the factor array `base` (elements of es
// bytes): per superblock inverse (nrp x nrp) and per front's L11 (w x w, leading
// dimension ld), a forward box (64 rows x FC columns) and a backward box (FC rows x
// 64 columns), FC = 32 KB / (64 es).
void ensure_solve_maps(mfs_handle *h, DevSym &ds, const void *base, int es) {
    if (h->smaps_base == base && h->smaps_sym == ds.id && h->smaps_es == es) return;
    const Symbolic &S = *ds.S;
    const uint32_t FC = uint32_t(32768 / (64 * es));
    const size_t nb = ds.isb_host.size(), nf = ds.sb_fronts.size();
    std::vector<TensorMapBlob> maps(std::max<size_t>(2 * (nb + nf), 1));
    std::memset(maps.data(), 0, maps.size() * sizeof(TensorMapBlob));
    const char *b = static_cast<const char *>(base);
    bool ok = true;
    for (size_t i = 0; i < nb && ok; ++i) {
        const SbTask &t = ds.isb_host[i];
        const idx nr = std::min<idx>(kSuperBlock, S.w[t.sn] - idx(t.K) * kSuperBlock);
        const uint64_t nrp = uint64_t((nr + 63) & ~idx(63));
        const void *p = b + size_t(t.inv) * es;
        ok = encode_plain_map(&maps[2 * i], p, es, nrp, nrp, nrp, 64, FC) &&
             encode_plain_map(&maps[2 * i + 1], p, es, nrp, nrp, nrp, FC, 64);
    }
    for (size_t i = 0; i < nf && ok; ++i) {
        const int32_t s = ds.sb_fronts[i];
        const void *p = b + size_t(ds.dpan[s]) * es;
        const uint64_t w = uint64_t(S.w[s]), ld = uint64_t(ds.dld[s]);
        ok = encode_plain_map(&maps[2 * (nb + i)], p, es, w, w, ld, 64, FC) &&
             encode_plain_map(&maps[2 * (nb + i) + 1], p, es, w, w, ld, FC, 64);
    }
    if (!ok) throw StatusError(MFS_INTERNAL, "cuTensorMapEncodeTiled refused a solve tensor map");
    h->smaps.ensure(maps.size());
    MFS_CUDA(cudaMemcpyAsync(h->smaps.p, maps.data(), maps.size() * sizeof(TensorMapBlob), cudaMemcpyHostToDevice,
                             h->stream));
    MFS_CUDA(cudaStreamSynchronize(h->stream));
    h->smaps_base = base;
    h->smaps_sym = ds.id;
    h->smaps_es = es;
}

template <typename T>
void run_factor(mfs_handle *h, DevSym &ds, T *factor, T *upd, T *dscr, const double *Ax, const double *Bx,
                double sigma) {
    const Symbolic &S = *ds.S;
    cudaStream_t st = h->stream;
    // FP32 factors: single-pass TF32 when FP64 refinement recovers the accuracy,
    // split 3xTF32 (FP32-level products) otherwise or when asked for.
    // 1: single-pass TF32 on tcgen05, 3: split 3xTF32 (mma.sync), 0: single-pass TF32 on mma.sync
    const int split = fp32_split(h);
    // GEMM launch, bracketed by CUDA events on its stream when kernel timing is on
    const bool timing = h->opt.time_kernels != 0;
    h->gemm_events_used = 0;
    h->gemm_flops_timed = 0.0;
    h->gemm_launch_info.clear();
    auto launch = [&](const GemmTask *tasks, int ntasks, int ntiles, const T *A, const T *B, T *C, int sp, int *err,
                      cudaStream_t s, bool mode0) {
        if constexpr (std::is_same<T, float>::value) {
            if ((sp == 4 || sp == 5 || sp == 6) && mode0) {
                launch_gemm_tma(sp == 6 ? 2 : sp == 5 ? 1 : 0, tasks, ntasks, ntiles, h->tmaps.p, C,
                                sp >= 5 ? h->sexp.p : nullptr, err, s, int(std::max<idx>(ds.S->nsn, 1)));
                return;
            }
            if (sp == 5 || sp == 6) {
                launch_gemm_tc(tasks, ntasks, ntiles, A, B, C, err, s, h->h16.p, h->sexp.p,
                               sp == 6 ? h->h16lo.p : nullptr);
                return;
            }
        }
        launch_gemm<T>(tasks, ntasks, ntiles, A, B, C, sp >= 4 ? 1 : sp, err, s);
    };
    auto tgemm = [&](const GemmTask *tasks, int ntasks, int ntiles, const T *A, const T *B, T *C, int sp, int *err,
                     cudaStream_t s, int kind, bool mode0 = true) {
        if (ntasks <= 0) return;
        if (!timing) {
            launch(tasks, ntasks, ntiles, A, B, C, sp, err, s, mode0);
            return;
        }
        if (h->gemm_events_used + 2 > h->gemm_events.size()) {
            cudaEvent_t e0, e1;
            MFS_CUDA(cudaEventCreate(&e0));
            MFS_CUDA(cudaEventCreate(&e1));
            h->gemm_events.push_back(e0);
            h->gemm_events.push_back(e1);
        }
        const size_t t0 = size_t(tasks - ds.gemm_tasks.p);
        const double fl = ds.gemm_flops_prefix[t0 + ntasks] - ds.gemm_flops_prefix[t0];
        h->gemm_flops_timed += fl;
        h->gemm_launch_info.insert(h->gemm_launch_info.end(), {fl, double(ntiles), double(ntasks), double(kind)});
        MFS_CUDA(cudaEventRecord(h->gemm_events[h->gemm_events_used], s));
        launch(tasks, ntasks, ntiles, A, B, C, sp, err, s, mode0);
        MFS_CUDA(cudaEventRecord(h->gemm_events[h->gemm_events_used + 1], s));
        h->gemm_events_used += 2;
    };
    launch_zero<T>(factor, ds.panel_alloc, st);
    launch_zero<T>(factor + (ds.factor_alloc - 64), 64, st);   // the tail the solves' vector loads may reach
    MFS_LAUNCHED();
    launch_inject<T>(ds.plan.p, int64_t(S.plan.size()), S.vb, S.src_ld, Ax, Bx, Bx ? sigma : 0.0, factor, st);
    MFS_LAUNCHED();
    if (!Bx && sigma != 0.0) {
        launch_diag_shift<T>(ds.diag_off.p, S.n, sigma, factor, st);
        MFS_LAUNCHED();
    }
    // The FP32 factor preconditions FP64 refinement: a large front's diagonal block
    // whose FP32 factorization meets a non-positive or tiny pivot is factored again
    // in FP64 (mfs_stats.refactored_blocks); pivots that stay non-positive there, and
    // non-positive pivots of fronts factored whole in shared memory, are perturbed
    // (relative to the injected diagonal) instead of failing.
    PivotCtl pv{h->fail.p, h->perturbed.p, nullptr, nullptr};
    if (h->opt.precision == MFS_PREC_FP32 && h->opt.refine) {
        h->dorig.ensure(size_t(std::max<idx>(S.n, 1)));
        pv.refactored = h->refactored.p;
        launch_extract_diag<T>(ds.diag_off.p, S.n, factor, h->dorig.p, st);
        if (split == 5 || split == 6)
            launch_front_scale(ds.large_dev.p, int(ds.large_fronts.size()), ds.sd, h->dorig.p, h->sexp.p, st);
        MFS_LAUNCHED();
        pv.dorig = h->dorig.p;
    }
    for (const LevelPlan &L : ds.levels) {
        if (L.small_count > 0) {
            launch_small_factor<T>(ds.small_list.p + L.small_off, L.small_count, L.small_max_front, ds.sd, factor,
                                   upd, pv, st);
            MFS_LAUNCHED();
        }
        if (L.large_count == 0) continue;
        launch_assemble_large<T>(ds.asm_tasks.p + L.asm_off, L.asm_n, L.asm_tiles, ds.sd, factor, upd, st);
        MFS_LAUNCHED();
        // One-group look-ahead: the column-block chain (left-looking update, panel, row
        // solve) and the update of the next group's columns run on a high-priority
        // stream, so their CTAs take the next free SMs; the update of the columns after
        // the next group runs meanwhile on the handle's stream. The next such update
        // overlaps that region and waits for it; the level's SYRK waits for both.
        cudaStream_t hs = h->side;
        MFS_CUDA(cudaEventRecord(h->ev_join, st));
        MFS_CUDA(cudaStreamWaitEvent(hs, h->ev_join, 0));
        bool rest_pending = false;
        for (const auto &sp : L.steps) {
            tgemm(ds.gemm_tasks.p + sp.left_off, sp.left_n, sp.left_tiles, factor, factor, factor, split,
                           h->gemm_err.p, hs, 0);
            MFS_LAUNCHED();
            launch_panel<T>(ds.potrf_tasks.p + sp.potrf_off, sp.potrf_n, sp.potrf_maxnb, factor, dscr, pv, split == 1 || split == 4 || split == 5,
                            hs);
            MFS_LAUNCHED();
            tgemm(ds.gemm_tasks.p + sp.trsm_off, sp.trsm_n, sp.trsm_tiles, factor, dscr, factor, split,
                           h->gemm_err.p, hs, 1, false);
            MFS_LAUNCHED();
            if (sp.gemm_n == 0) continue;
            if (sp.rest_n > 0) MFS_CUDA(cudaEventRecord(h->ev_ready, hs));
            if (rest_pending) {
                MFS_CUDA(cudaStreamWaitEvent(hs, h->ev_rest, 0));
                rest_pending = false;
            }
            tgemm(ds.gemm_tasks.p + sp.gemm_off, sp.gemm_n, sp.gemm_tiles, factor, factor, factor, split,
                           h->gemm_err.p, hs, 2);
            MFS_LAUNCHED();
            if (sp.rest_n > 0) {
                MFS_CUDA(cudaStreamWaitEvent(st, h->ev_ready, 0));
                tgemm(ds.gemm_tasks.p + sp.rest_off, sp.rest_n, sp.rest_tiles, factor, factor, factor, split,
                               h->gemm_err.p, st, 3);
                MFS_LAUNCHED();
                MFS_CUDA(cudaEventRecord(h->ev_rest, st));
                rest_pending = true;
            }
        }
        MFS_CUDA(cudaEventRecord(h->ev_join, hs));
        MFS_CUDA(cudaStreamWaitEvent(st, h->ev_join, 0));
        if (L.syrk_n > 0) {
            tgemm(ds.gemm_tasks.p + L.syrk_off, L.syrk_n, L.syrk_tiles, factor, factor, upd, split, h->gemm_err.p, st,
                  4);
            MFS_LAUNCHED();
        }
    }
    // inverses of the superblocks of L11 that the diagonal solves apply
    launch_sb_inverse<T>(ds.isb_tasks.p, ds.nsb_inv, ds.sd, factor, st);
    MFS_LAUNCHED();
}

// The factorization's launch sequence, replayed from an instantiated CUDA graph when
// use_graphs is on: the first call with a new key runs directly (it also makes the
// one-time allocations and kernel attribute settings), the second captures the
// sequence from the handle's stream (the look-ahead stream joins the capture through
// its events) and later calls launch the graph. Kernel timing runs directly.
template <typename T>
void factor_sequence(mfs_handle *h, DevSym &ds, T *factor, T *upd, T *dscr, const double *Ax, const double *Bx,
                     double sigma) {
    ensure_side_stream(h);
    const int split = fp32_split(h);
    if constexpr (std::is_same<T, float>::value) {
        if (split == 4) ensure_panel_maps(h, ds, factor, false);
        if (split == 5 || split == 6) {
            h->h16.ensure(size_t(std::max<int64_t>(ds.panel_alloc, 1)));
            h->sexp.ensure(size_t(std::max<idx>(ds.S->nsn, 1)));
            if (split == 6) h->h16lo.ensure(size_t(std::max<int64_t>(ds.panel_alloc, 1)));
            ensure_panel_maps(h, ds, h->h16.p, true, split == 6 ? h->h16lo.p : nullptr);
        }
    }
    // (the legacy default stream cannot be captured: graphs need a handle or caller stream)
    if (!h->opt.use_graphs || h->opt.time_kernels || h->stream == nullptr) {
        run_factor<T>(h, ds, factor, upd, dscr, Ax, Bx, sigma);
        return;
    }
    const void *dorig = h->dorig.p;
    mfs_handle::FactorGraph key{ds.id,    factor,      upd,         dscr,  Ax,    Bx,     dorig,
                                h->h16.p, h->h16lo.p, h->tmaps.p, sigma, split, nullptr};
    auto same = [&](const mfs_handle::FactorGraph &g) {
        return g.ds == key.ds && g.factor == key.factor && g.upd == key.upd && g.dscr == key.dscr &&
               g.ax == key.ax && g.bx == key.bx && g.dorig == key.dorig && g.h16 == key.h16 && g.h16lo == key.h16lo &&
               g.tmaps == key.tmaps && g.sigma == key.sigma &&
               g.split == key.split;
    };
    auto it = std::find_if(h->factor_graphs.begin(), h->factor_graphs.end(), same);
    if (it != h->factor_graphs.end() && it->exec) {
        MFS_CUDA(cudaGraphLaunch(it->exec, h->stream));
        return;
    }
    if (it == h->factor_graphs.end()) {
        run_factor<T>(h, ds, factor, upd, dscr, Ax, Bx, sigma);
        if (h->factor_graphs.size() >= 4) {
            if (h->factor_graphs.front().exec) cudaGraphExecDestroy(h->factor_graphs.front().exec);
            h->factor_graphs.erase(h->factor_graphs.begin());
        }
        h->factor_graphs.push_back(key);
        return;
    }
    cudaStream_t st = h->stream;
    MFS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaGraph_t graph = nullptr;
    try {
        run_factor<T>(h, ds, factor, upd, dscr, Ax, Bx, sigma);
    } catch (...) {
        cudaStreamEndCapture(st, &graph);
        if (graph) cudaGraphDestroy(graph);
        throw;
    }
    MFS_CUDA(cudaStreamEndCapture(st, &graph));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    MFS_CUDA(e);
    it->exec = exec;
    MFS_CUDA(cudaGraphLaunch(exec, st));
}

template <typename T>
void run_solve(mfs_handle *h, DevSym &ds, const T *factor, double *X, int nrhs) {
    const Symbolic &S = *ds.S;
    cudaStream_t st = h->stream;
    const bool sb = h->opt.solve_chain != 1;
    const int pass = sb ? kSbMaxRhs : kMaxSolveRhs;
    const int chunk = std::min(nrhs, pass);
    h->sol.ensure(size_t(std::max<idx>(S.sol_size, 1)) * chunk);
    h->str_partials.ensure(size_t(std::max<int64_t>(ds.max_str_entries, 1)) * chunk);
    if (sb) {
        h->sb_scratch.ensure(size_t(std::max<idx>(S.n, 1)) * chunk);
        ensure_solve_maps(h, ds, factor, int(sizeof(T)));
    }
    for (int r0 = 0; r0 < nrhs; r0 += pass) {
        const int nr = std::min(pass, nrhs - r0);
        double *Xc = X + int64_t(r0) * S.n;
        MFS_CUDA(cudaMemsetAsync(ds.flags.p, 0, ds.flags.bytes(), st));
        // levels <= solve_cut: whole subtrees, one per CTA
        launch_subtree_solve<T>(true, ds.subs.p, ds.nsub, ds.sub_fmax, ds.sd, factor, Xc, S.n, nr, h->sol.p, st);
        MFS_LAUNCHED();
        for (size_t l = size_t(ds.solve_cut + 1); l < ds.levels.size(); ++l) {
            const LevelPlan &L = ds.levels[l];
            launch_fwd_asm(ds.sasm_tasks.p + L.sasm_off, L.sasm_n, L.sasm_tiles, ds.sd, Xc, S.n, nr, h->sol.p, st);
            MFS_LAUNCHED();
            if (!sb)
                MFS_CUDA(launch_diag<T>(true, ds.ftri_tasks.p + L.ftri_off, L.ftri_n, ds.sd, factor, Xc, S.n, nr,
                                        ds.flags.p, h->solve_err.p, st));
            else
                MFS_CUDA(launch_sb_solve<T>(true, ds.fsb_tasks.p + L.fsb_off, L.fsb_n, ds.sd, factor, h->smaps.p, Xc, S.n, nr,
                                            h->sb_scratch.p, ds.flags.p, h->solve_err.p, st));
            launch_str<T>(true, ds.fstr_tasks.p + L.fstr_off, L.fstr_n, ds.fred.p + L.fred_off, L.fred_n, ds.sd,
                          factor, Xc, S.n, nr, h->sol.p, h->str_partials.p, st);
            MFS_LAUNCHED();
        }
        for (size_t l = ds.levels.size(); l-- > size_t(ds.solve_cut + 1);) {
            const LevelPlan &L = ds.levels[l];
            launch_str<T>(false, ds.bstr_tasks.p + L.bstr_off, L.bstr_n, ds.bred.p + L.bred_off, L.bred_n, ds.sd,
                          factor, Xc, S.n, nr, h->sol.p, h->str_partials.p, st);
            MFS_LAUNCHED();
            if (!sb)
                MFS_CUDA(launch_diag<T>(false, ds.btri_tasks.p + L.btri_off, L.btri_n, ds.sd, factor, Xc, S.n, nr,
                                        ds.flags.p, h->solve_err.p, st));
            else
                MFS_CUDA(launch_sb_solve<T>(false, ds.bsb_tasks.p + L.bsb_off, L.bsb_n, ds.sd, factor, h->smaps.p, Xc, S.n, nr,
                                            h->sb_scratch.p, ds.flags.p, h->solve_err.p, st));
        }
        launch_subtree_solve<T>(false, ds.subs.p, ds.nsub, ds.sub_fmax, ds.sd, factor, Xc, S.n, nr, h->sol.p, st);
        MFS_LAUNCHED();
    }
}

// After a stream synchronisation: a solve wait that timed out is an error.
void check_solve_error(mfs_handle *h) {
    int e = 0;
    MFS_CUDA(cudaMemcpy(&e, h->solve_err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) {
        MFS_CUDA(cudaMemset(h->solve_err.p, 0, sizeof(int)));
        throw StatusError(MFS_TIMEOUT, "triangular solve: a dependency wait timed out");
    }
}

void solve_current(mfs_handle *h, double *X, int nrhs) {
    DevSym &ds = *h->cur.sym;
    if (h->opt.precision == MFS_PREC_FP32) run_solve<float>(h, ds, h->cur.f32->p, X, nrhs);
    else run_solve<double>(h, ds, h->cur.f64->p, X, nrhs);
}

// Y = (A + sigma I | A + sigma B) X on the permuted reduced system.
void apply_current(mfs_handle *h, const double *Ax, const double *Bx, double sigma, const double *X, double *Y,
                   int nrhs) {
    DevSym &ds = *h->cur.sym;
    const Symbolic &S = *ds.S;
    launch_spmv(ds.spmv_ptr.p, ds.spmv_src.p, ds.spmv_col.p, ds.spmv_flag.p, S.nv, S.vb, S.src_ld, Ax, X, Y, S.n,
                nrhs, h->stream);
    MFS_LAUNCHED();
    if (sigma == 0.0) return;
    const int64_t cnt = int64_t(S.n) * nrhs;
    if (Bx) {
        h->work_s.ensure(size_t(cnt));
        launch_spmv(ds.spmv_ptr.p, ds.spmv_src.p, ds.spmv_col.p, ds.spmv_flag.p, S.nv, S.vb, S.src_ld, Bx, X,
                    h->work_s.p, S.n, nrhs, h->stream);
        launch_axpy(Y, h->work_s.p, sigma, cnt, h->stream);
    } else {
        launch_axpy(Y, X, sigma, cnt, h->stream);
    }
    MFS_LAUNCHED();
}

// Preconditioned CG on the permuted reduced system, preconditioned by the
// current (FP32) factor, everything else FP64. B and X are n x nrhs (ld n).
void refine_solve(mfs_handle *h, const double *B, double *X, int nrhs) {
    DevSym &ds = *h->cur.sym;
    const Symbolic &S = *ds.S;
    const int64_t n = S.n;
    const size_t sz = size_t(n) * nrhs;
    cudaStream_t st = h->stream;
    if (nrhs > 64) throw StatusError(MFS_INVALID_ARG, "refined solves support at most 64 right-hand sides");
    h->work_r.ensure(sz);
    h->work_z.ensure(sz);
    h->work_p.ensure(sz);
    h->work_ap.ensure(sz);
    const int np = reduce_partials_count();
    h->partials.ensure(size_t(np) * 64);
    h->dots.ensure(4 * 64);
    h->active.ensure(64);
    double *bb = h->dots.p, *rz = h->dots.p + 64, *rz2 = h->dots.p + 128, *pap = h->dots.p + 192;
    if (!h->cur.ax) throw StatusError(MFS_NO_FACTOR, "matrix values of the current factor are not available");
    const double *Ax = h->cur.ax->p;
    const double *Bx = h->cur.bx ? h->cur.bx->p : nullptr;
    const double sigma = h->cur.sigma;
    std::vector<int> act(nrhs, 1);
    MFS_CUDA(cudaMemcpyAsync(h->active.p, act.data(), nrhs * sizeof(int), cudaMemcpyHostToDevice, st));
    launch_colnorm2(B, n, nrhs, h->partials.p, bb, st);
    MFS_CUDA(cudaMemsetAsync(X, 0, sz * sizeof(double), st));
    launch_copy(h->work_r.p, B, int64_t(sz), st);
    launch_copy(h->work_z.p, B, int64_t(sz), st);
    MFS_LAUNCHED();
    solve_current(h, h->work_z.p, nrhs);
    launch_copy(h->work_p.p, h->work_z.p, int64_t(sz), st);
    launch_coldot(h->work_r.p, h->work_z.p, n, nrhs, h->partials.p, rz, st);
    MFS_LAUNCHED();
    std::vector<double> hb(nrhs), hr(nrhs);
    MFS_CUDA(cudaMemcpyAsync(hb.data(), bb, nrhs * sizeof(double), cudaMemcpyDeviceToHost, st));
    MFS_CUDA(cudaStreamSynchronize(st));
    const double tol = h->opt.refine_tol > 0 ? h->opt.refine_tol : 1e-10;
    const int maxit = h->opt.refine_maxit > 0 ? h->opt.refine_maxit : 50;
    int it = 0;
    double worst = 0.0;
    bool all_done = false;
    for (int r = 0; r < nrhs; ++r) if (hb[r] == 0.0) act[r] = 0;
    while (it < maxit) {
        ++it;
        apply_current(h, Ax, Bx, sigma, h->work_p.p, h->work_ap.p, nrhs);
        launch_coldot(h->work_p.p, h->work_ap.p, n, nrhs, h->partials.p, pap, st);
        launch_pcg_update_x_r(X, h->work_r.p, h->work_p.p, h->work_ap.p, rz, pap, h->active.p, n, nrhs, st);
        launch_colnorm2(h->work_r.p, n, nrhs, h->partials.p, rz2, st);
        MFS_LAUNCHED();
        MFS_CUDA(cudaMemcpyAsync(hr.data(), rz2, nrhs * sizeof(double), cudaMemcpyDeviceToHost, st));
        MFS_CUDA(cudaStreamSynchronize(st));
        check_solve_error(h);
        worst = 0.0;
        all_done = true;
        for (int r = 0; r < nrhs; ++r) {
            double rel = hb[r] > 0 ? std::sqrt(hr[r] / hb[r]) : 0.0;
            if (act[r] && rel <= tol) act[r] = 0;
            if (act[r]) all_done = false;
            worst = std::max(worst, rel);
        }
        if (all_done) break;
        MFS_CUDA(cudaMemcpyAsync(h->active.p, act.data(), nrhs * sizeof(int), cudaMemcpyHostToDevice, st));
        launch_copy(h->work_z.p, h->work_r.p, int64_t(sz), st);
        MFS_LAUNCHED();
        solve_current(h, h->work_z.p, nrhs);
        launch_coldot(h->work_r.p, h->work_z.p, n, nrhs, h->partials.p, rz2, st);
        launch_pcg_update_p(h->work_p.p, h->work_z.p, rz2, rz, h->active.p, n, nrhs, st);
        MFS_LAUNCHED();
        MFS_CUDA(cudaMemcpyAsync(rz, rz2, nrhs * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    h->stats.refine_iterations = it;
    h->stats.residual = worst;
    if (!all_done) {
        char buf[160];
        std::snprintf(buf, sizeof(buf),
                      "refinement did not reach the residual target within %d iterations (worst %.3e)", it, worst);
        throw StatusError(MFS_NOT_POSDEF, buf);
    }
}

void require_symbolic(mfs_handle *h) {
    if (!h->cur.sym || h->cur.type < 1) throw StatusError(MFS_NO_FACTOR, "Symbolic factorization does not exist");
}
void require_numeric(mfs_handle *h) {
    if (!h->cur.sym || h->cur.type < 2) throw StatusError(MFS_NO_FACTOR, "Numeric factorization does not exist");
}

const double *stage_input(mfs_handle *h, DBuf<double> &buf, const double *src, size_t count, bool on_device) {
    if (on_device) return src;
    buf.ensure(count);
    if (count) MFS_CUDA(cudaMemcpyAsync(buf.p, src, count * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    return buf.p;
}

}  // namespace

// Scratch of mfs_apply_noalloc: the permuted reduced copies of x and of y,
// kNoAllocApplyEntries doubles each (16 MiB on every GPU that loads this
// library, held until the process exits). In host code the name only stands in
// for the array; its device address comes from cudaGetSymbolAddress.
constexpr int64_t kNoAllocApplyEntries = int64_t(1) << 20;
static __device__ __align__(256) double g_noalloc_apply_scratch[2 * kNoAllocApplyEntries];

namespace {

// Device address of the scratch on device `dev` (which must be current),
// looked up on the first call for that device and cached.
double *noalloc_apply_scratch(int dev) {
    static std::mutex mu;
    static double *addr[256] = {};
    if (dev < 0 || dev >= 256) throw StatusError(MFS_INVALID_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void *p = nullptr;
        MFS_CUDA(cudaGetSymbolAddress(&p, g_noalloc_apply_scratch));
        addr[dev] = static_cast<double *>(p);
    }
    return addr[dev];
}

}  // namespace

extern "C" {

mfs_status mfs_default_options(mfs_options *opt) {
    if (!opt) return MFS_INVALID_ARG;
    std::memset(opt, 0, sizeof(*opt));
    opt->precision = MFS_PREC_FP64;
    opt->ordering = MFS_ORDER_ND;
    opt->relax = 1;
    opt->device = 0;
    opt->relax_zeros = 128;
    opt->relax_ratio = 0.01;
    opt->nd_leaf_size = 120;
    opt->seed = 12345;
    opt->stream = nullptr;
    opt->small_front_max = 0;
    opt->refine = 0;
    opt->refine_tol = 1e-10;
    opt->refine_maxit = 50;
    opt->use_graphs = 0;
    opt->tensor_cores = 0;
    opt->time_kernels = 0;
    return MFS_OK;
}

mfs_status mfs_create(mfs_handle **out, const mfs_options *opt) {
    if (!out) return MFS_INVALID_ARG;
    *out = nullptr;
    auto h = std::make_unique<mfs_handle>();
    if (opt) h->opt = *opt;
    else mfs_default_options(&h->opt);
    mfs_status s = guarded(h.get(), [&] {
        if (h->opt.precision != MFS_PREC_FP64 && h->opt.precision != MFS_PREC_FP32)
            throw StatusError(MFS_INVALID_ARG, "unknown precision");
        h->stats.failed_column = -1;
        if (h->opt.device == -1) return;   // analysis-only handle: no CUDA context is touched
        int ndev = 0;
        MFS_CUDA(cudaGetDeviceCount(&ndev));
        if (h->opt.device < 0 || h->opt.device >= ndev) throw StatusError(MFS_INVALID_ARG, "invalid CUDA device");
        set_device(h.get());
        if (h->opt.stream) h->stream = static_cast<cudaStream_t>(h->opt.stream);
        else {
            MFS_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
            h->own_stream = true;
        }
        MFS_CUDA(cudaEventCreate(&h->ev0));
        MFS_CUDA(cudaEventCreate(&h->ev1));
        MFS_CUDA(cudaMallocHost(&h->fail_host, 4 * sizeof(int)));
        MFS_CUDA(cudaMallocHost(&h->dots_host, 64 * sizeof(double)));
        h->fail.ensure(1);
        h->perturbed.ensure(1);
        h->refactored.ensure(1);
        h->solve_err.ensure(1);
        MFS_CUDA(cudaMemset(h->solve_err.p, 0, sizeof(int)));
        h->gemm_err.ensure(1);
        MFS_CUDA(cudaMemset(h->gemm_err.p, 0, sizeof(int)));
    });
    if (s != MFS_OK) {
        // keep the message reachable for callers that only get a status
        return s;
    }
    *out = h.release();
    return MFS_OK;
}

mfs_status mfs_set_options(mfs_handle *h, const mfs_options *opt) {
    if (!h || !opt) return MFS_INVALID_ARG;
    if (opt->precision != h->opt.precision || opt->device != h->opt.device)
        return MFS_INVALID_ARG;   // fixed for the lifetime of a handle
    void *stream = h->opt.stream;
    if (opt->tensor_cores != h->opt.tensor_cores || opt->refine != h->opt.refine) h->split_escalated = false;
    h->opt = *opt;
    h->opt.stream = stream;
    return MFS_OK;
}

mfs_status mfs_destroy(mfs_handle *h) {
    if (!h) return MFS_OK;
    if (h->opt.device == -1) {
        delete h;
        return MFS_OK;
    }
    cudaSetDevice(h->opt.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->side) {
        cudaStreamSynchronize(h->side);
        cudaStreamDestroy(h->side);
    }
    if (h->ev_ready) cudaEventDestroy(h->ev_ready);
    if (h->ev_rest) cudaEventDestroy(h->ev_rest);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    for (cudaEvent_t e : h->gemm_events) cudaEventDestroy(e);
    clear_factor_graphs(h);
    if (h->fail_host) cudaFreeHost(h->fail_host);
    if (h->dots_host) cudaFreeHost(h->dots_host);
    delete h;
    return MFS_OK;
}

mfs_status mfs_last_error(const mfs_handle *h, char *buf, size_t len) {
    if (!h || !buf || len == 0) return MFS_INVALID_ARG;
    std::strncpy(buf, h->err.c_str(), len - 1);
    buf[len - 1] = 0;
    return MFS_OK;
}

mfs_status mfs_build_pattern(int64_t nvars, int64_t nelem, int32_t npe, const int64_t *conn, int64_t *Ap,
                             int64_t *Ai, int64_t *nnz) {
    if (nvars < 0 || nelem < 0 || npe <= 0 || !Ap || !nnz || (nelem > 0 && !conn)) return MFS_INVALID_ARG;
    try {
        Pattern P = build_block_pattern(nvars, nelem, npe, conn);
        std::copy(P.Ap.begin(), P.Ap.end(), Ap);
        *nnz = P.nnz();
        if (Ai) std::copy(P.Ai.begin(), P.Ai.end(), Ai);
        return MFS_OK;
    } catch (const std::invalid_argument &) {
        return MFS_INVALID_ARG;
    } catch (...) {
        return MFS_INTERNAL;
    }
}

mfs_status mfs_build_pattern_device(int32_t device, int64_t nvars, int64_t nelem, int32_t npe,
                                    const int64_t *conn, int64_t *Ap, int64_t *Ai, int64_t *nnz, void *stream) {
    if (nvars < 0 || nelem < 0 || npe <= 0 || !Ap || !nnz || (nelem > 0 && !conn)) return MFS_INVALID_ARG;
    return guarded(nullptr, [&] {
        MFS_CUDA(cudaSetDevice(device));
        *nnz = gpu_build_pattern(nvars, nelem, npe, conn, Ap, Ai, static_cast<cudaStream_t>(stream));
    });
}

mfs_status mfs_symbolic(mfs_handle *h, int64_t n_blocks, const int64_t *Ap, const int64_t *Ai, int32_t block_size,
                        const int64_t *pinned, int64_t n_pinned, const int64_t *user_perm,
                        const int64_t *supernode_sizes, int64_t num_supernodes) {
    if (!h) return MFS_INVALID_ARG;
    return guarded(h, [&] {
        if (!Ap || (n_pinned > 0 && !pinned) || n_blocks < 0) throw StatusError(MFS_INVALID_ARG, "null pattern");
        if (Ap[n_blocks] > 0 && !Ai) throw StatusError(MFS_INVALID_ARG, "null Ai");
        const bool host_only = h->opt.device == -1;
        if (!host_only) set_device(h);
        // A new analysis replaces the current factorization (the stash is kept).
        h->cur = State();
        h->asm_ax.reset();
        h->asm_spare.reset();
        h->nslots = 0;
        h->nelem = 0;
        auto Sp = std::make_shared<Symbolic>();
        SymbolicOptions so;
        so.ordering = h->opt.ordering;
        so.relax = h->opt.relax != 0;
        so.relax_zeros = h->opt.relax_zeros;
        so.relax_ratio = h->opt.relax_ratio;
        so.nd.leaf_size = h->opt.nd_leaf_size > 0 ? h->opt.nd_leaf_size : 120;
        so.nd.seed = h->opt.seed;
        so.solve_subtrees = h->opt.solve_subtrees;
        // the history belongs to one variable set: the same block size, block count and
        // pins (a pin change or the scalar fallback starts afresh, as the reference's
        // temporal reuse state does)
        std::vector<int64_t> key{int64_t(block_size), n_blocks};
        {
            std::vector<int64_t> pins(pinned, pinned + std::max<int64_t>(n_pinned, 0));
            std::sort(pins.begin(), pins.end());
            pins.erase(std::unique(pins.begin(), pins.end()), pins.end());
            key.insert(key.end(), pins.begin(), pins.end());
        }
        const bool reuse = h->opt.nd_reuse_period > 0 && h->nd_prev && h->nd_prev_key == key &&
                           h->nd_reuse_count < h->opt.nd_reuse_period;
        if (reuse) so.nd_prev = h->nd_prev.get();
        std::string e = analyze(n_blocks, Ap, Ai, block_size, pinned, n_pinned, so, user_perm, *Sp, supernode_sizes,
                                supernode_sizes ? num_supernodes : 0);
        if (!e.empty())
            throw StatusError(e.rfind("Fixed variable index out of range", 0) == 0 ? MFS_SIZE_MISMATCH : MFS_INVALID_ARG,
                              e);
        // keep this dissection's separator tree for the next analysis
        h->stats.nd_reused = Sp->nd_rebuilt >= 0 ? 1 : 0;
        h->stats.nd_rebuilt_vertices = Sp->nd_rebuilt >= 0 ? Sp->nd_rebuilt : Sp->nv;
        if (!Sp->nd_cmember.empty()) {
            auto nd = std::make_shared<NDResult>();
            nd->cparent = Sp->nd_cparent;
            nd->cmember = Sp->nd_cmember;
            nd->ncomp = Sp->nd_ncomp;
            h->nd_prev = nd;
            h->nd_prev_key = key;
            h->nd_reuse_count = Sp->nd_rebuilt >= 0 ? h->nd_reuse_count + 1 : 0;
        }
        if (host_only) {
            auto ds = std::make_shared<DevSym>();
            ds->S = Sp;
            ds->ax_len = Ap[n_blocks] * int64_t(block_size) * block_size;
            h->cur.sym = ds;
            h->split_escalated = false;
            h->cur.type = 1;
            h->stats.num_levels = int(Sp->nlevels);
            return;
        }
        clear_factor_graphs(h);
        auto ds = upload_symbolic(h, Sp);
        ds->ax_len = Ap[n_blocks] * int64_t(block_size) * block_size;
        ds->Ap_full.assign(Ap, Ap + n_blocks + 1);
        ds->Ai_full.assign(Ai, Ai + Ap[n_blocks]);
        const Symbolic &S = *Sp;
        if (h->opt.precision == MFS_PREC_FP32) h->upd32.ensure(size_t(std::max<idx>(S.upd_size, 1)));
        else h->upd64.ensure(size_t(std::max<idx>(S.upd_size, 1)));
        h->cur.sym = ds;
        h->split_escalated = false;
        h->cur.type = 1;
        h->stats.num_levels = int(S.nlevels);
        h->stats.num_large = ds->num_large;
    });
}

// The numeric factorization of the current values (h->cur.ax / bx, h->cur.sigma);
// counters to mfs_stats, errors thrown. An FP32 factorization under refinement with
// single-pass TF32 / FP16 products that had to perturb a pivot is redone once with
// split FP16 (FP32-level) products, which the handle then keeps: on high-contrast
// inputs the low-precision Schur updates lose definiteness and refinement stalls.
void numeric_core(mfs_handle *h) {
    DevSym &ds = *h->cur.sym;
    const Symbolic &S = *ds.S;
    cudaStream_t st = h->stream;
    const double *dBx = h->cur.bx ? h->cur.bx->p : nullptr;
    const double sigma = h->cur.sigma;
    const int big = INT_MAX;
    MFS_CUDA(cudaMemcpyAsync(h->fail.p, &big, sizeof(int), cudaMemcpyHostToDevice, st));
    MFS_CUDA(cudaMemsetAsync(h->perturbed.p, 0, sizeof(int), st));
    MFS_CUDA(cudaMemsetAsync(h->refactored.p, 0, sizeof(int), st));
    MFS_CUDA(cudaEventRecord(h->ev0, st));
    if (h->opt.precision == MFS_PREC_FP32) {
        if (!h->cur.f32 || h->cur.f32.use_count() > 1) h->cur.f32 = std::make_shared<DBuf<float>>();
        h->cur.f32->ensure(size_t(ds.factor_alloc));
        h->upd32.ensure(size_t(std::max<idx>(S.upd_size, 1)));
        h->dscr32.ensure(size_t(std::max<int64_t>(ds.inv_scratch, 1)));
        factor_sequence<float>(h, ds, h->cur.f32->p, h->upd32.p, h->dscr32.p, h->cur.ax->p, dBx, sigma);
    } else {
        if (!h->cur.f64 || h->cur.f64.use_count() > 1) h->cur.f64 = std::make_shared<DBuf<double>>();
        h->cur.f64->ensure(size_t(ds.factor_alloc));
        h->upd64.ensure(size_t(std::max<idx>(S.upd_size, 1)));
        h->dscr64.ensure(size_t(std::max<int64_t>(ds.inv_scratch, 1)));
        factor_sequence<double>(h, ds, h->cur.f64->p, h->upd64.p, h->dscr64.p, h->cur.ax->p, dBx, sigma);
    }
    MFS_CUDA(cudaEventRecord(h->ev1, st));
    MFS_CUDA(cudaMemcpyAsync(h->fail_host, h->fail.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MFS_CUDA(cudaMemcpyAsync(h->fail_host + 1, h->perturbed.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MFS_CUDA(cudaMemcpyAsync(h->fail_host + 2, h->gemm_err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MFS_CUDA(cudaMemcpyAsync(h->fail_host + 3, h->refactored.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    MFS_CUDA(cudaStreamSynchronize(st));
    float ms = 0;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->stats.factor_ms = ms;
    h->stats.perturbed_pivots = h->fail_host[1];
    h->stats.refactored_blocks = h->fail_host[3];
    h->stats.gemm_ms = 0.0;
    h->stats.gemm_flops = h->gemm_flops_timed;
    h->stats.gemm_launches = int64_t(h->gemm_events_used / 2);
    h->gemm_launch_ms.clear();
    for (size_t e = 0; e + 1 < h->gemm_events_used; e += 2) {
        float g = 0;
        MFS_CUDA(cudaEventElapsedTime(&g, h->gemm_events[e], h->gemm_events[e + 1]));
        h->stats.gemm_ms += g;
        h->gemm_launch_ms.push_back(g);
    }
    if (h->fail_host[2]) {
        MFS_CUDA(cudaMemset(h->gemm_err.p, 0, sizeof(int)));
        throw StatusError(MFS_TIMEOUT, "Schur update: a tensor-core pipeline wait timed out");
    }
    if (*h->fail_host != INT_MAX) {
        h->stats.failed_column = *h->fail_host;
        throw StatusError(MFS_NOT_POSDEF, std::to_string(*h->fail_host) + "/" + std::to_string(S.n) +
                                              "  pivots successful in numeric factorization (non-positive definite?)");
    }
    const int sp = h->opt.precision == MFS_PREC_FP32 ? fp32_split(h) : 3;
    if (h->opt.precision == MFS_PREC_FP32 && h->opt.refine && sp != 3 && sp != 6 && h->stats.perturbed_pivots > 0 &&
        !h->split_escalated) {
        h->split_escalated = true;
        ++h->stats.split_escalations;
        numeric_core(h);
    }
}

mfs_status mfs_numeric(mfs_handle *h, const double *Ax, const double *Bx, double sigma, int32_t flags) {
    if (!h) return MFS_INVALID_ARG;
    return guarded(h, [&] {
        require_symbolic(h);
        set_device(h);
        DevSym &ds = *h->cur.sym;
        const bool dev = (flags & MFS_DEVICE_POINTERS) != 0;
        cudaStream_t st = h->stream;
        // The numeric factor becomes invalid from here until success.
        h->cur.type = 1;
        const size_t axn = size_t(ds.ax_len);
        auto take_values = [&](std::shared_ptr<DBuf<double>> &dst, const double *src) {
            if (!dst || dst.use_count() > 1) dst = std::make_shared<DBuf<double>>();
            dst->ensure(axn);
            if (axn)
                MFS_CUDA(cudaMemcpyAsync(dst->p, src, axn * sizeof(double),
                                         dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
        };
        if (Ax) {
            take_values(h->cur.ax, Ax);
        } else {
            if (!h->asm_ax) throw StatusError(MFS_INVALID_ARG, "no values: pass Ax or assemble first");
            h->cur.ax = h->asm_ax;
        }
        if (Bx) take_values(h->cur.bx, Bx);
        else h->cur.bx.reset();
        h->cur.sigma = sigma;
        numeric_core(h);
        h->stats.failed_column = -1;
        h->cur.type = 2;
    });
}

mfs_status mfs_solve(mfs_handle *h, const double *B, double *X, int64_t nrhs, int64_t ldb, int32_t flags) {
    if (!h) return MFS_INVALID_ARG;
    return guarded(h, [&] {
        require_numeric(h);
        set_device(h);
        DevSym &ds = *h->cur.sym;
        const Symbolic &S = *ds.S;
        const int mode = flags & 3;
        const bool dev = (flags & MFS_DEVICE_POINTERS) != 0;
        if (nrhs < 1) throw StatusError(MFS_INVALID_ARG, "Must specify at least one rhs.");
        const int64_t rows = mode == MFS_SOLVE_FULL ? S.n_full : S.n;
        if (ldb < rows) throw StatusError(MFS_SIZE_MISMATCH, "Incorrect RHS size");
        if (!B || !X) throw StatusError(MFS_INVALID_ARG, "null vector");
        cudaStream_t st = h->stream;
        const size_t sz = size_t(S.n) * nrhs;
        h->rhs.ensure(sz);
        const double *Bd = B;
        double *Xd = X;
        const size_t io_sz = size_t(ldb) * nrhs;
        if (!dev) {
            h->io.ensure(io_sz);
            MFS_CUDA(cudaMemcpyAsync(h->io.p, B, io_sz * sizeof(double), cudaMemcpyHostToDevice, st));
            Bd = h->io.p;
            Xd = h->io.p;
        }
        MFS_CUDA(cudaEventRecord(h->ev0, st));
        const int64_t *map = mode == MFS_SOLVE_FULL ? ds.prrfr.p : (mode == MFS_SOLVE_REDUCED ? ds.sperm.p : nullptr);
        launch_gather_rows(map, rows, Bd, ldb, h->rhs.p, S.n, int(nrhs), st);
        MFS_LAUNCHED();
        double *result = h->rhs.p;
        const bool refine = h->opt.refine && h->opt.precision == MFS_PREC_FP32;
        if (refine) {
            h->work_x.ensure(sz);
            try {
                refine_solve(h, h->rhs.p, h->work_x.p, int(nrhs));
            } catch (const StatusError &e) {
                // refinement stalled on a low-precision factor: factor the same values again
                // with FP32-level products (kept for the handle) and solve once more
                if (e.status != MFS_NOT_POSDEF || fp32_split(h) == 3 || fp32_split(h) == 6) throw;
                h->split_escalated = true;
                ++h->stats.split_escalations;
                numeric_core(h);
                refine_solve(h, h->rhs.p, h->work_x.p, int(nrhs));
            }
            result = h->work_x.p;
        } else {
            solve_current(h, h->rhs.p, int(nrhs));
        }
        launch_scatter_rows(map, rows, result, S.n, Xd, ldb, int(nrhs), st);
        MFS_LAUNCHED();
        MFS_CUDA(cudaEventRecord(h->ev1, st));
        if (!dev) MFS_CUDA(cudaMemcpyAsync(X, h->io.p, io_sz * sizeof(double), cudaMemcpyDeviceToHost, st));
        MFS_CUDA(cudaStreamSynchronize(st));
        check_solve_error(h);
        float ms = 0;
        cudaEventElapsedTime(&ms, h->ev0, h->ev1);
        h->stats.solve_ms = ms;
    });
}

mfs_status mfs_apply(mfs_handle *h, const double *x, double *y, int64_t nrhs, int64_t ld, int32_t flags) {
    if (!h) return MFS_INVALID_ARG;
    return guarded(h, [&] {
        require_symbolic(h);
        std::shared_ptr<DBuf<double>> vals = h->cur.ax ? h->cur.ax : h->asm_ax;
        if (!vals) throw StatusError(MFS_NO_FACTOR, "no matrix values on the device");
        set_device(h);
        DevSym &ds = *h->cur.sym;
        const Symbolic &S = *ds.S;
        const int mode = flags & 3;
        const bool dev = (flags & MFS_DEVICE_POINTERS) != 0;
        const int64_t rows = mode == MFS_SOLVE_FULL ? S.n_full : S.n;
        if (ld < rows || nrhs < 1) throw StatusError(MFS_SIZE_MISMATCH, "Incorrect vector size");
        cudaStream_t st = h->stream;
        const size_t sz = size_t(S.n) * nrhs;
        const size_t io_sz = size_t(ld) * nrhs;
        h->rhs.ensure(sz);
        h->work_x.ensure(sz);
        const double *xd = x;
        double *yd = y;
        if (!dev) {
            h->io.ensure(io_sz);
            MFS_CUDA(cudaMemcpyAsync(h->io.p, x, io_sz * sizeof(double), cudaMemcpyHostToDevice, st));
            xd = h->io.p;
            yd = h->io.p;
        }
        const int64_t *map = mode == MFS_SOLVE_FULL ? ds.prrfr.p : (mode == MFS_SOLVE_REDUCED ? ds.sperm.p : nullptr);
        launch_gather_rows(map, rows, xd, ld, h->rhs.p, S.n, int(nrhs), st);
        apply_current(h, vals->p, nullptr, 0.0, h->rhs.p, h->work_x.p, int(nrhs));
        launch_scatter_rows(map, rows, h->work_x.p, S.n, yd, ld, int(nrhs), st);
        MFS_LAUNCHED();
        if (!dev) MFS_CUDA(cudaMemcpyAsync(y, h->io.p, io_sz * sizeof(double), cudaMemcpyDeviceToHost, st));
        MFS_CUDA(cudaStreamSynchronize(st));
    });
}

mfs_status mfs_assembly_setup(mfs_handle *h, int64_t nelem, const int64_t *conn) {
    if (!h) return MFS_INVALID_ARG;
    return guarded(h, [&] {
        require_symbolic(h);
        set_device(h);
        DevSym &ds = *h->cur.sym;
        if (ds.S->bs != 3) throw StatusError(MFS_INVALID_ARG, "element assembly expects 3x3 blocks");
        if (nelem < 0 || (nelem > 0 && !conn)) throw StatusError(MFS_INVALID_ARG, "bad connectivity");
        const int64_t nb = int64_t(ds.Ap_full.size()) - 1;
        const int64_t nslots = ds.Ap_full[nb];
        {
            // the element -> slot map, built on the GPU. Per element, in the reference's
            // order (SystemAssembler.hh:60-98): columns by sorted global index; an upper
            // block (bi, bj) takes He(i_loc, j_loc) when the local order agrees with the
            // global one, else the transpose of He(j_loc, i_loc); the diagonal block adds
            // its upper triangle only; each slot sums its contributions in element order.
            cudaStream_t st = h->stream;
            if (!ds.Ap_full_dev.p || ds.Ap_full_dev.n < ds.Ap_full.size()) {
                ds.Ap_full_dev.upload(ds.Ap_full, st);
                ds.Ai_full_dev.upload(ds.Ai_full, st);
            }
            DBuf<int64_t> cd;
            if (nelem > 0) {
                cd.ensure(size_t(nelem) * 4);
                MFS_CUDA(cudaMemcpyAsync(cd.p, conn, size_t(nelem) * 4 * sizeof(int64_t), cudaMemcpyHostToDevice, st));
            }
            gpu_build_slot_map(nelem, cd.p, nb, ds.Ap_full_dev.p, ds.Ai_full_dev.p, nslots, h->slot_ptr, h->contrib,
                               st);
            h->nslots = nslots;
            h->nelem = nelem;
        }
    });
}

mfs_status mfs_assemble(mfs_handle *h, const double *Ke, double *Ax_out, int32_t flags) {
    if (!h) return MFS_INVALID_ARG;
    return guarded(h, [&] {
        require_symbolic(h);
        if (h->nslots == 0 && h->nelem == 0) throw StatusError(MFS_INVALID_ARG, "call mfs_assembly_setup first");
        set_device(h);
        DevSym &ds = *h->cur.sym;
        cudaStream_t st = h->stream;
        const bool dev = (flags & MFS_DEVICE_POINTERS) != 0;
        const size_t ke_n = size_t(h->nelem) * 144;
        const double *Ked = dev ? Ke : stage_input(h, h->ke, Ke, ke_n, false);
        // The current factor may still hold the previous assembly (its values drive
        // refinement): assemble into another buffer then, alternating between two.
        if (!h->asm_ax || h->asm_ax.use_count() > 1) {
            if (h->asm_spare && h->asm_spare.use_count() == 1) std::swap(h->asm_ax, h->asm_spare);
            else {
                h->asm_spare = h->asm_ax;
                h->asm_ax = std::make_shared<DBuf<double>>();
            }
            if (h->asm_ax.use_count() > 1) h->asm_ax = std::make_shared<DBuf<double>>();
        }
        h->asm_ax->ensure(size_t(ds.ax_len));
        MFS_CUDA(cudaEventRecord(h->ev0, st));
        launch_assemble_elements(h->slot_ptr.p, h->contrib.p, h->nslots, Ked, h->asm_ax->p, st);
        MFS_LAUNCHED();
        MFS_CUDA(cudaEventRecord(h->ev1, st));
        if (Ax_out) {
            MFS_CUDA(cudaMemcpyAsync(Ax_out, h->asm_ax->p, size_t(ds.ax_len) * sizeof(double),
                                     dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
        }
        MFS_CUDA(cudaStreamSynchronize(st));
        float ms = 0;
        cudaEventElapsedTime(&ms, h->ev0, h->ev1);
        h->stats.assemble_ms = ms;
    });
}

mfs_status mfs_info(const mfs_handle *h, int64_t *n_full, int64_t *n_reduced, int64_t *factor_nnz, double *flops,
                    int64_t *num_supernodes, int32_t *factorization_type) {
    if (!h) return MFS_INVALID_ARG;
    const bool has = h->cur.sym && h->cur.type >= 1;
    if (factorization_type) *factorization_type = h->cur.type;
    if (!has) return MFS_NO_FACTOR;
    const Symbolic &S = *h->cur.sym->S;
    if (n_full) *n_full = S.n_full;
    if (n_reduced) *n_reduced = S.n;
    if (factor_nnz) *factor_nnz = S.factor_nnz;
    if (flops) *flops = S.flops;
    if (num_supernodes) *num_supernodes = S.nsn;
    return MFS_OK;
}

mfs_status mfs_inverse_permutation(const mfs_handle *h, int64_t *iperm_out) {
    if (!h || !iperm_out) return MFS_INVALID_ARG;
    if (!h->cur.sym || h->cur.type < 1) return MFS_NO_FACTOR;
    const Symbolic &S = *h->cur.sym->S;
    std::copy(S.scalar_iperm.begin(), S.scalar_iperm.end(), iperm_out);
    return MFS_OK;
}

mfs_status mfs_nd_ordering(const mfs_handle *h, int64_t *ncomp, int64_t *nmember, int64_t *cparent,
                           int64_t *cmember) {
    if (!h || !ncomp || !nmember) return MFS_INVALID_ARG;
    if (!h->cur.sym || h->cur.type < 1) return MFS_NO_FACTOR;
    const Symbolic &S = *h->cur.sym->S;
    *ncomp = int64_t(S.nd_cparent.size());
    *nmember = int64_t(S.nd_cmember.size());
    if (cparent) std::copy(S.nd_cparent.begin(), S.nd_cparent.end(), cparent);
    if (cmember) std::copy(S.nd_cmember.begin(), S.nd_cmember.end(), cmember);
    return MFS_OK;
}

mfs_status mfs_supernodes(const mfs_handle *h, int64_t *nsn, int64_t *nstruct, int32_t *vb, int64_t *sn_start,
                          int64_t *parent, int64_t *struct_ptr, int64_t *struct_rows, int64_t *rel) {
    if (!h || !nsn || !nstruct) return MFS_INVALID_ARG;
    if (!h->cur.sym || h->cur.type < 1) return MFS_NO_FACTOR;
    const Symbolic &S = *h->cur.sym->S;
    *nsn = S.nsn;
    *nstruct = int64_t(S.struct_rows.size());
    if (vb) *vb = S.vb;
    if (sn_start) std::copy(S.sn_start.begin(), S.sn_start.end(), sn_start);
    if (parent) std::copy(S.sn_parent.begin(), S.sn_parent.end(), parent);
    if (struct_ptr) std::copy(S.struct_ptr.begin(), S.struct_ptr.end(), struct_ptr);
    if (struct_rows) std::copy(S.struct_rows.begin(), S.struct_rows.end(), struct_rows);
    if (rel) std::copy(S.rel.begin(), S.rel.end(), rel);
    return MFS_OK;
}

mfs_status mfs_conversion_plan(const mfs_handle *h, int64_t *nv, int64_t *nentries, int64_t *column_offsets,
                               int64_t *entries) {
    if (!h || !nv || !nentries) return MFS_INVALID_ARG;
    if (!h->cur.sym || h->cur.type < 1) return MFS_NO_FACTOR;
    const Symbolic &S = *h->cur.sym->S;
    *nv = S.nv;
    *nentries = int64_t(S.plan.size());
    if (column_offsets) std::copy(S.plan_ptr.begin(), S.plan_ptr.end(), column_offsets);
    if (entries)
        for (size_t k = 0; k < S.plan.size(); ++k) {
            entries[4 * k] = S.plan[k].dst;
            entries[4 * k + 1] = S.plan[k].src;
            entries[4 * k + 2] = S.plan[k].ld;
            entries[4 * k + 3] = S.plan[k].flags;
        }
    return MFS_OK;
}

mfs_status mfs_conversion_plan_device(const mfs_handle *h, int64_t *nv, int64_t *nentries, int64_t *column_offsets,
                                      int64_t *entries) {
    if (!h || !nv || !nentries) return MFS_INVALID_ARG;
    if (!h->cur.sym || h->cur.type < 1) return MFS_NO_FACTOR;
    if (h->opt.device < 0) return MFS_INVALID_ARG;
    const DevSym &ds = *h->cur.sym;
    const Symbolic &S = *ds.S;
    *nv = S.nv;
    *nentries = int64_t(S.plan.size());
    if (cudaSetDevice(h->opt.device) != cudaSuccess) return MFS_CUDA_ERROR;
    if (column_offsets && cudaMemcpy(column_offsets, ds.plan_ptr_dev.p, size_t(2 * S.nv + 1) * sizeof(int64_t),
                                     cudaMemcpyDeviceToHost) != cudaSuccess)
        return MFS_CUDA_ERROR;
    if (entries && !S.plan.empty()) {
        std::vector<PlanEntryDev> pe(S.plan.size());
        if (cudaMemcpy(pe.data(), ds.plan_cat.p, pe.size() * sizeof(PlanEntryDev), cudaMemcpyDeviceToHost) !=
            cudaSuccess)
            return MFS_CUDA_ERROR;
        for (size_t k = 0; k < pe.size(); ++k) {
            entries[4 * k] = pe[k].dst;
            entries[4 * k + 1] = pe[k].src;
            entries[4 * k + 2] = pe[k].ld;
            entries[4 * k + 3] = pe[k].flags;
        }
    }
    return MFS_OK;
}

mfs_status mfs_factor_values(const mfs_handle *h, int64_t *factor_size, double *out) {
    if (!h || !factor_size) return MFS_INVALID_ARG;
    if (!h->cur.sym || h->cur.type < 2) return MFS_NO_FACTOR;
    const Symbolic &S = *h->cur.sym->S;
    *factor_size = S.factor_size;
    if (!out) return MFS_OK;
    mfs_handle *hm = const_cast<mfs_handle *>(h);
    return guarded(hm, [&] {
        set_device(hm);
        // the device panels carry padded leading dimensions: repack into the catamari layout
        const DevSym &ds = *h->cur.sym;
        auto repack = [&](const auto *dev) {
            using T = std::remove_const_t<std::remove_pointer_t<decltype(dev)>>;
            std::vector<T> tmp(size_t(ds.panel_alloc));
            MFS_CUDA(cudaMemcpy(tmp.data(), dev, tmp.size() * sizeof(T), cudaMemcpyDeviceToHost));
            for (size_t s = 0; s + 1 < ds.dpan.size(); ++s)
                for (idx j = 0; j < S.w[s]; ++j)
                    for (idx i = 0; i < S.f[s]; ++i)
                        out[S.pan_off[s] + j * S.f[s] + i] = double(tmp[ds.dpan[s] + j * ds.dld[s] + i]);
        };
        if (h->opt.precision == MFS_PREC_FP32) repack(static_cast<const float *>(h->cur.f32->p));
        else repack(static_cast<const double *>(h->cur.f64->p));
    });
}

mfs_status mfs_stash(mfs_handle *h) {
    if (!h) return MFS_INVALID_ARG;
    return guarded(h, [&] {
        require_symbolic(h);
        set_device(h);
        State s;
        s.sym = h->cur.sym;
        s.type = h->cur.type;
        s.sigma = h->cur.sigma;
        s.ax = h->cur.ax;
        s.bx = h->cur.bx;
        const size_t fs = size_t(h->cur.sym->factor_alloc);
        if (h->cur.type >= 2) {
            if (h->cur.f64) {
                s.f64 = std::make_shared<DBuf<double>>();
                s.f64->ensure(fs);
                MFS_CUDA(cudaMemcpyAsync(s.f64->p, h->cur.f64->p, fs * sizeof(double), cudaMemcpyDeviceToDevice,
                                         h->stream));
            }
            if (h->cur.f32) {
                s.f32 = std::make_shared<DBuf<float>>();
                s.f32->ensure(fs);
                MFS_CUDA(cudaMemcpyAsync(s.f32->p, h->cur.f32->p, fs * sizeof(float), cudaMemcpyDeviceToDevice,
                                         h->stream));
            }
        }
        MFS_CUDA(cudaStreamSynchronize(h->stream));
        h->stash = s;
        h->has_stash = true;
    });
}

mfs_status mfs_swap_stash(mfs_handle *h) {
    if (!h) return MFS_INVALID_ARG;
    return guarded(h, [&] {
        if (!h->has_stash) throw StatusError(MFS_NO_FACTOR, "No stashed factorization");
        clear_factor_graphs(h);
        std::swap(h->cur, h->stash);
        if (h->cur.sym) {
            const Symbolic &S = *h->cur.sym->S;
            if (h->opt.precision == MFS_PREC_FP32) h->upd32.ensure(size_t(std::max<idx>(S.upd_size, 1)));
            else h->upd64.ensure(size_t(std::max<idx>(S.upd_size, 1)));
        }
    });
}

mfs_status mfs_clear_stash(mfs_handle *h) {
    if (!h) return MFS_INVALID_ARG;
    clear_factor_graphs(h);
    h->stash = State();
    h->has_stash = false;
    return MFS_OK;
}

mfs_status mfs_has_stash(const mfs_handle *h, int32_t *has) {
    if (!h || !has) return MFS_INVALID_ARG;
    *has = h->has_stash ? 1 : 0;
    return MFS_OK;
}

mfs_status mfs_clear_factors(mfs_handle *h) {
    if (!h) return MFS_INVALID_ARG;
    clear_factor_graphs(h);
    h->cur = State();
    h->asm_ax.reset();
    h->asm_spare.reset();
    h->nslots = 0;
    h->nelem = 0;
    return MFS_OK;
}

// y = H x like mfs_apply, with device vectors only and every temporary in the
// fixed array above: nothing is allocated, on the device or pinned, during the
// call. Every entry of the scratch that is read was written earlier in the same
// call (gather, then the SpMV overwrites y), so nothing needs clearing between
// calls.
mfs_status mfs_apply_noalloc(mfs_handle *h, const double *x, double *y, int64_t nrhs, int64_t ld, int32_t flags) {
    if (!h) return MFS_INVALID_ARG;
    return guarded(h, [&] {
        require_symbolic(h);
        const double *vals = h->cur.ax ? h->cur.ax->p : (h->asm_ax ? h->asm_ax->p : nullptr);
        if (!vals) throw StatusError(MFS_NO_FACTOR, "no matrix values on the device");
        if (!(flags & MFS_DEVICE_POINTERS))
            throw StatusError(MFS_INVALID_ARG, "mfs_apply_noalloc takes device vectors only (MFS_DEVICE_POINTERS)");
        if (!x || !y) throw StatusError(MFS_INVALID_ARG, "null vector");
        set_device(h);
        DevSym &ds = *h->cur.sym;
        const Symbolic &S = *ds.S;
        const int mode = flags & 3;
        const int64_t rows = mode == MFS_SOLVE_FULL ? S.n_full : S.n;
        if (ld < rows || nrhs < 1) throw StatusError(MFS_SIZE_MISMATCH, "Incorrect vector size");
        if (int64_t(S.n) * nrhs > kNoAllocApplyEntries)
            throw StatusError(MFS_SIZE_MISMATCH,
                              "mfs_apply_noalloc: free variables x right-hand sides = " +
                                  std::to_string(int64_t(S.n) * nrhs) + " exceeds its fixed scratch of " +
                                  std::to_string(kNoAllocApplyEntries) + " entries");
        double *xs = noalloc_apply_scratch(h->opt.device);
        double *ys = xs + kNoAllocApplyEntries;
        cudaStream_t st = h->stream;
        const int64_t *map = mode == MFS_SOLVE_FULL ? ds.prrfr.p : (mode == MFS_SOLVE_REDUCED ? ds.sperm.p : nullptr);
        launch_gather_rows(map, rows, x, ld, xs, S.n, int(nrhs), st);
        apply_current(h, vals, nullptr, 0.0, xs, ys, int(nrhs));
        launch_scatter_rows(map, rows, ys, S.n, y, ld, int(nrhs), st);
        MFS_LAUNCHED();
        MFS_CUDA(cudaStreamSynchronize(st));
    });
}

mfs_status mfs_debug_gemm_launches(const mfs_handle *h, int64_t max_launches, double *out, int64_t *count) {
    if (!h || !count || (max_launches > 0 && !out)) return MFS_INVALID_ARG;
    const size_t n = std::min(h->gemm_launch_ms.size(), h->gemm_launch_info.size() / 4);
    *count = int64_t(n);
    for (size_t i = 0; i < n && int64_t(i) < max_launches; ++i) {
        out[5 * i] = double(h->gemm_launch_ms[i]);
        for (int c = 0; c < 4; ++c) out[5 * i + 1 + c] = h->gemm_launch_info[4 * i + c];
    }
    return MFS_OK;
}

mfs_status mfs_get_stats(const mfs_handle *h, mfs_stats *st) {
    if (!h || !st) return MFS_INVALID_ARG;
    *st = h->stats;
    int64_t bytes = 0;
    if (h->cur.sym) bytes += int64_t(h->cur.sym->bytes());
    if (h->cur.f64) bytes += int64_t(h->cur.f64->bytes());
    if (h->cur.f32) bytes += int64_t(h->cur.f32->bytes());
    if (h->cur.ax) bytes += int64_t(h->cur.ax->bytes());
    bytes += int64_t(h->upd64.bytes() + h->upd32.bytes() + h->sol.bytes() + h->rhs.bytes());
    st->device_bytes = bytes;
    st->kernel_launches = g_kernel_launches;
    return MFS_OK;
}

}  // extern "C"
