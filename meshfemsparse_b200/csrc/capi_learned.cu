// C ABI of the learned preconditioner (include/mfs_b200.h, "learned PCG"):
// network lifetime and weights, the training step (loss, gradient, Adam) and
// PCG with M^{-1} = D^{-1/2} G^T G D^{-1/2}, falling back to the Cholesky
// factor when PCG misses the tolerance within the iteration cap. Host logic
// only; the kernels are in kernels_learned.cu.
#include "handle.h"
#include "learned.h"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <random>
#include <vector>

struct mfs_lpc {
    int device = 0;
    int n = 0;                           // parameters
    int step = 0;                        // Adam steps taken
    mfs::DBuf<float> w, m, v, grad;      // FP32 master weights, Adam moments, last gradient
    mfs::DBuf<__nv_bfloat16> wb;         // BF16 weights read by the kernels
};

namespace {

using namespace mfs;

// Graph arrays that the SpMV structure lacks (diagonal position, transposed entry).
struct LGraphDev {
    DBuf<int64_t> diag, mirror;
    DBuf<float> ea;
    int64_t nnz = 0;
    LGraph g{};
};

struct LWorkDev {
    int64_t nv = -1, nnz = -1;
    int nrhs = 0;
    DBuf<double> dinv;
    DBuf<float> eh, esum, h[kLLayers + 1], s[kLLayers], pre[kLLayers], q, G, dG, dq, dod, dh0, dh1, ds, part;
    DBuf<double> ax, bp, xp, bs, xs, z, y, e, t, gy, gz, r, pz, p, ap;
    DBuf<double> partials, dots;
    DBuf<int> active;
    LWork w{};
};

LGraphDev &graph_of(mfs_handle *h) {
    DevSym &ds = *h->cur.sym;
    const Symbolic &S = *ds.S;
    if (S.vb != 3 || S.src_ld != 3)
        throw StatusError(MFS_INVALID_ARG, "the learned preconditioner needs a 3 x 3 block analysis (whole-block pins)");
    if (ds.lpc_graph) return *static_cast<LGraphDev *>(ds.lpc_graph.get());
    auto gd = std::make_shared<LGraphDev>();
    const int64_t nv = S.nv;
    const int64_t nnz = S.spmv_ptr[nv];
    std::vector<int64_t> diag(nv), mirror(nnz);
    for (int64_t i = 0; i < nv; ++i) {
        const int32_t *b = S.spmv_col.data() + S.spmv_ptr[i], *e = S.spmv_col.data() + S.spmv_ptr[i + 1];
        const int32_t *it = std::lower_bound(b, e, int32_t(i));
        if (it == e || *it != i) throw StatusError(MFS_INTERNAL, "block row without a diagonal entry");
        diag[i] = S.spmv_ptr[i] + (it - b);
    }
    for (int64_t i = 0; i < nv; ++i)
        for (int64_t k = S.spmv_ptr[i]; k < S.spmv_ptr[i + 1]; ++k) {
            const int64_t j = S.spmv_col[k];
            const int32_t *b = S.spmv_col.data() + S.spmv_ptr[j], *e = S.spmv_col.data() + S.spmv_ptr[j + 1];
            const int32_t *it = std::lower_bound(b, e, int32_t(i));
            if (it == e || *it != i) throw StatusError(MFS_INTERNAL, "block pattern is not symmetric");
            mirror[k] = S.spmv_ptr[j] + (it - b);
        }
    gd->diag.upload(diag, h->stream);
    gd->mirror.upload(mirror, h->stream);
    gd->ea.ensure(size_t(nnz));
    gd->nnz = nnz;
    gd->g = LGraph{nv, ds.spmv_ptr.p, ds.spmv_src.p, gd->diag.p, gd->mirror.p, ds.spmv_col.p, ds.spmv_flag.p, gd->ea.p};
    ds.lpc_graph = gd;
    return *gd;
}

LWorkDev &work_of(mfs_handle *h, const LGraphDev &gd, int nrhs) {
    if (!h->lpc_work) h->lpc_work = std::make_shared<LWorkDev>();
    LWorkDev &W = *static_cast<LWorkDev *>(h->lpc_work.get());
    const int64_t nv = gd.g.nv, nnz = gd.nnz;
    if (W.nv != nv || W.nnz != nnz) {
        W.dinv.ensure(size_t(3 * nv));
        W.eh.ensure(size_t(9 * nnz));
        W.esum.ensure(size_t(9 * nv));
        W.h[0].ensure(size_t(kLIn * nv));
        for (int l = 1; l <= kLLayers; ++l) W.h[l].ensure(size_t(kLHid * nv));
        for (int l = 0; l < kLLayers; ++l) {
            W.s[l].ensure(size_t(lpc_layer_in(l) * nv));
            W.pre[l].ensure(size_t(kLHid * nv));
        }
        W.q.ensure(size_t(kLHead * nv));
        W.G.ensure(size_t(9 * nnz));
        W.dG.ensure(size_t(9 * nnz));
        W.dq.ensure(size_t(kLHead * nv));
        W.dod.ensure(size_t(6 * nv));
        W.dh0.ensure(size_t(kLHid * nv));
        W.dh1.ensure(size_t(kLHid * nv));
        W.ds.ensure(size_t(kLHid * nv));
        const LParamLayout L = lpc_layout();
        const int maxp = std::max(kLHid * (2 * kLHid + 10), 150);
        W.part.ensure(size_t(std::max(lpc_dense_parts(), lpc_head_parts())) * maxp);
        (void)L;
        W.nv = nv;
        W.nnz = nnz;
        W.nrhs = 0;
    }
    if (nrhs > W.nrhs) {
        const size_t sz = size_t(3 * nv) * nrhs;
        for (DBuf<double> *b : {&W.bp, &W.xp, &W.bs, &W.xs, &W.z, &W.y, &W.e, &W.t, &W.gy, &W.gz, &W.r, &W.pz, &W.p,
                                &W.ap})
            b->ensure(sz);
        W.partials.ensure(size_t(reduce_partials_count()) * nrhs);
        W.dots.ensure(size_t(4) * nrhs);
        W.active.ensure(size_t(nrhs));
        W.nrhs = nrhs;
    }
    W.w.dinv = W.dinv.p;
    W.w.eh = W.eh.p;
    W.w.esum = W.esum.p;
    for (int l = 0; l <= kLLayers; ++l) W.w.h[l] = W.h[l].p;
    for (int l = 0; l < kLLayers; ++l) {
        W.w.s[l] = W.s[l].p;
        W.w.pre[l] = W.pre[l].p;
    }
    W.w.q = W.q.p;
    W.w.G = W.G.p;
    W.w.dG = W.dG.p;
    W.w.dq = W.dq.p;
    W.w.dod = W.dod.p;
    W.w.dh[0] = W.dh0.p;
    W.w.dh[1] = W.dh1.p;
    W.w.ds = W.ds.p;
    W.w.part = W.part.p;
    return W;
}

// Matrix values on the device: the caller's (host or device) or the last assembly.
const double *values_of(mfs_handle *h, LWorkDev &W, const double *Ax, bool dev) {
    DevSym &ds = *h->cur.sym;
    if (!Ax) {
        if (!h->asm_ax) throw StatusError(MFS_INVALID_ARG, "no values: pass Ax or assemble first");
        return h->asm_ax->p;
    }
    if (dev) return Ax;
    W.ax.ensure(size_t(ds.ax_len));
    MFS_CUDA(cudaMemcpyAsync(W.ax.p, Ax, size_t(ds.ax_len) * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    return W.ax.p;
}

// Caller-order vectors (host or device) -> permuted reduced n x nrhs.
void gather_in(mfs_handle *h, const double *src, bool dev, int mode, int64_t ld, int nrhs, double *dst) {
    DevSym &ds = *h->cur.sym;
    const Symbolic &S = *ds.S;
    const int64_t rows = mode == MFS_SOLVE_FULL ? S.n_full : S.n;
    const int64_t *map = mode == MFS_SOLVE_FULL ? ds.prrfr.p : (mode == MFS_SOLVE_REDUCED ? ds.sperm.p : nullptr);
    const double *in = src;
    if (!dev) {
        h->io.ensure(size_t(ld) * nrhs);
        MFS_CUDA(cudaMemcpyAsync(h->io.p, src, size_t(ld) * nrhs * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        in = h->io.p;
    }
    launch_gather_rows(map, rows, in, ld, dst, S.n, nrhs, h->stream);
    MFS_LAUNCHED();
}

void scatter_out(mfs_handle *h, const double *src, double *out, bool dev, int mode, int64_t ld, int nrhs) {
    DevSym &ds = *h->cur.sym;
    const Symbolic &S = *ds.S;
    const int64_t rows = mode == MFS_SOLVE_FULL ? S.n_full : S.n;
    const int64_t *map = mode == MFS_SOLVE_FULL ? ds.prrfr.p : (mode == MFS_SOLVE_REDUCED ? ds.sperm.p : nullptr);
    double *dst = out;
    if (!dev) {
        h->io.ensure(size_t(ld) * nrhs);
        dst = h->io.p;
    }
    launch_scatter_rows(map, rows, src, S.n, dst, ld, nrhs, h->stream);
    MFS_LAUNCHED();
    if (!dev)
        MFS_CUDA(cudaMemcpyAsync(out, h->io.p, size_t(ld) * nrhs * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
}

void spmv(mfs_handle *h, const double *Ax, const double *X, double *Y, int nrhs) {
    DevSym &ds = *h->cur.sym;
    const Symbolic &S = *ds.S;
    launch_spmv(ds.spmv_ptr.p, ds.spmv_src.p, ds.spmv_col.p, ds.spmv_flag.p, S.nv, S.vb, S.src_ld, Ax, X, Y, S.n,
                nrhs, h->stream);
    MFS_LAUNCHED();
}

void check_net(const mfs_handle *h, const mfs_lpc *net) {
    if (net && net->device != h->opt.device)
        throw StatusError(MFS_INVALID_ARG, "the network lives on another device than the handle");
}

void check_common(mfs_handle *h, int64_t nrhs, int64_t ld, int mode) {
    if (!h->cur.sym || h->cur.type < 1) throw StatusError(MFS_NO_FACTOR, "Symbolic factorization does not exist");
    const Symbolic &S = *h->cur.sym->S;
    if (nrhs < 1 || nrhs > 64) throw StatusError(MFS_INVALID_ARG, "between 1 and 64 right-hand sides");
    const int64_t rows = mode == MFS_SOLVE_FULL ? S.n_full : S.n;
    if (ld < rows) throw StatusError(MFS_SIZE_MISMATCH, "Incorrect RHS size");
}

// loss and gradient (device) for pairs already gathered into W.bp / W.xp
double loss_grad(mfs_handle *h, mfs_lpc *net, const LGraphDev &gd, LWorkDev &W, const double *Ax, int nrhs) {
    cudaStream_t st = h->stream;
    const LGraph &g = gd.g;
    const int64_t n = 3 * g.nv;
    lpc_features(g, Ax, W.w, st);
    lpc_forward(g, net->wb.p, W.w, st);
    MFS_LAUNCHED();
    // scaled pair, M^{-1} applied, error and its energy
    lpc_scale_rows(W.bp.p, W.dinv.p, false, W.bs.p, n, nrhs, n, st);
    lpc_scale_rows(W.xp.p, W.dinv.p, true, W.xs.p, n, nrhs, n, st);
    lpc_gmv(g, W.G.p, false, W.bs.p, W.z.p, n, nrhs, nullptr, nullptr, st);
    lpc_gmv(g, W.G.p, true, W.z.p, W.y.p, n, nrhs, nullptr, nullptr, st);
    launch_copy(W.e.p, W.y.p, n * nrhs, st);
    launch_axpy(W.e.p, W.xs.p, -1.0, n * nrhs, st);
    lpc_scale_rows(W.e.p, W.dinv.p, false, W.t.p, n, nrhs, n, st);
    spmv(h, Ax, W.t.p, W.ap.p, nrhs);
    lpc_scale_rows(W.ap.p, W.dinv.p, false, W.gy.p, n, nrhs, n, st);   // gy = Hs e (scaled below)
    double *nrm = W.dots.p, *en = W.dots.p + nrhs;
    launch_coldot(W.xp.p, W.bp.p, n, nrhs, W.partials.p, nrm, st);
    launch_coldot(W.e.p, W.gy.p, n, nrhs, W.partials.p, en, st);
    MFS_LAUNCHED();
    std::vector<double> hd(2 * size_t(nrhs));
    MFS_CUDA(cudaMemcpyAsync(hd.data(), W.dots.p, hd.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    MFS_CUDA(cudaStreamSynchronize(st));
    double loss = 0.0;
    for (int r = 0; r < nrhs; ++r) {
        const double nr = hd[r] > 0 ? hd[r] : 1.0;
        loss += hd[nrhs + r] / nr / nrhs;
        // dL/dy_r = 2 Hs e_r / (nrhs x_r^T b_r), in place on gy
        if (n) launch_axpy(W.gy.p + r * n, W.gy.p + r * n, 2.0 / (nr * nrhs) - 1.0, n, st);
    }
    lpc_gmv(g, W.G.p, false, W.gy.p, W.gz.p, n, nrhs, nullptr, nullptr, st);
    lpc_dg(g, W.z.p, W.gy.p, W.gz.p, W.bs.p, n, nrhs, W.dG.p, st);
    lpc_backward(g, net->wb.p, W.w, net->grad.p, st);
    MFS_LAUNCHED();
    return loss;
}

void init_weights(mfs_lpc *net, uint64_t seed, cudaStream_t st) {
    const LParamLayout L = lpc_layout();
    std::vector<float> w(size_t(L.total), 0.f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < kLLayers; ++l) {
        const int din = lpc_layer_in(l), dtot = 2 * din + 10;
        const float bound = std::sqrt(6.f / float(dtot)) * 0.5f;
        std::uniform_real_distribution<float> U(-bound, bound);
        for (int k = 0; k < kLHid; ++k)
            for (int m = 0; m < dtot; ++m) w[size_t(L.w[l] + k * dtot + m)] = (m == dtot - 1) ? 0.f : U(rng);
    }
    // head weights start at zero: G = I, i.e. Jacobi-preconditioned CG
    MFS_CUDA(cudaMemcpyAsync(net->w.p, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice, st));
    MFS_CUDA(cudaMemsetAsync(net->m.p, 0, w.size() * sizeof(float), st));
    MFS_CUDA(cudaMemsetAsync(net->v.p, 0, w.size() * sizeof(float), st));
    lpc_to_bf16(net->w.p, net->wb.p, L.total, st);
    MFS_LAUNCHED();
    MFS_CUDA(cudaStreamSynchronize(st));
    net->step = 0;
}

}  // namespace

extern "C" {

mfs_status mfs_lpc_param_count(int64_t *count) {
    if (!count) return MFS_INVALID_ARG;
    *count = lpc_layout().total;
    return MFS_OK;
}

mfs_status mfs_lpc_create(mfs_lpc **out, int32_t device, uint64_t seed) {
    if (!out || device < 0) return MFS_INVALID_ARG;
    *out = nullptr;
    auto net = std::make_unique<mfs_lpc>();
    const mfs_status s = guarded(nullptr, [&] {
        MFS_CUDA(cudaSetDevice(device));
        net->device = device;
        net->n = lpc_layout().total;
        net->w.ensure(size_t(net->n));
        net->m.ensure(size_t(net->n));
        net->v.ensure(size_t(net->n));
        net->grad.ensure(size_t(net->n));
        net->wb.ensure(size_t(net->n));
        init_weights(net.get(), seed, nullptr);
    });
    if (s == MFS_OK) *out = net.release();
    return s;
}

mfs_status mfs_lpc_destroy(mfs_lpc *net) {
    if (!net) return MFS_INVALID_ARG;
    cudaSetDevice(net->device);
    delete net;
    return MFS_OK;
}

mfs_status mfs_lpc_get_weights(const mfs_lpc *net, float *w, int64_t count) {
    if (!net || !w) return MFS_INVALID_ARG;
    if (count != net->n) return MFS_SIZE_MISMATCH;
    return guarded(nullptr, [&] {
        MFS_CUDA(cudaSetDevice(net->device));
        MFS_CUDA(cudaMemcpy(w, net->w.p, size_t(count) * sizeof(float), cudaMemcpyDeviceToHost));
    });
}

mfs_status mfs_lpc_set_weights(mfs_lpc *net, const float *w, int64_t count) {
    if (!net || !w) return MFS_INVALID_ARG;
    if (count != net->n) return MFS_SIZE_MISMATCH;
    return guarded(nullptr, [&] {
        MFS_CUDA(cudaSetDevice(net->device));
        MFS_CUDA(cudaMemcpy(net->w.p, w, size_t(count) * sizeof(float), cudaMemcpyHostToDevice));
        MFS_CUDA(cudaMemset(net->m.p, 0, size_t(count) * sizeof(float)));
        MFS_CUDA(cudaMemset(net->v.p, 0, size_t(count) * sizeof(float)));
        lpc_to_bf16(net->w.p, net->wb.p, net->n, nullptr);
        MFS_LAUNCHED();
        MFS_CUDA(cudaDeviceSynchronize());
        net->step = 0;
    });
}

mfs_status mfs_lpc_loss_grad(mfs_handle *h, mfs_lpc *net, const double *Ax, const double *B, const double *X,
                             int64_t nrhs, int64_t ld, int32_t flags, double *loss, float *grad) {
    if (!h || !net || !B || !X) return MFS_INVALID_ARG;
    return guarded(h, [&] {
        const int mode = flags & 3;
        const bool dev = (flags & MFS_DEVICE_POINTERS) != 0;
        check_common(h, nrhs, ld, mode);
        check_net(h, net);
        set_device(h);
        LGraphDev &gd = graph_of(h);
        LWorkDev &W = work_of(h, gd, int(nrhs));
        const double *ax = values_of(h, W, Ax, dev);
        gather_in(h, B, dev, mode, ld, int(nrhs), W.bp.p);
        gather_in(h, X, dev, mode, ld, int(nrhs), W.xp.p);
        const double l = loss_grad(h, net, gd, W, ax, int(nrhs));
        if (grad)
            MFS_CUDA(cudaMemcpyAsync(grad, net->grad.p, size_t(net->n) * sizeof(float), cudaMemcpyDeviceToHost,
                                     h->stream));
        MFS_CUDA(cudaStreamSynchronize(h->stream));
        if (loss) *loss = l;
    });
}

mfs_status mfs_lpc_train_step(mfs_handle *h, mfs_lpc *net, const double *Ax, const double *B, const double *X,
                              int64_t nrhs, int64_t ld, int32_t flags, float lr, double *loss) {
    if (!h || !net || !B || !X || !(lr > 0.f)) return MFS_INVALID_ARG;
    return guarded(h, [&] {
        const int mode = flags & 3;
        const bool dev = (flags & MFS_DEVICE_POINTERS) != 0;
        check_common(h, nrhs, ld, mode);
        check_net(h, net);
        set_device(h);
        LGraphDev &gd = graph_of(h);
        LWorkDev &W = work_of(h, gd, int(nrhs));
        const double *ax = values_of(h, W, Ax, dev);
        gather_in(h, B, dev, mode, ld, int(nrhs), W.bp.p);
        gather_in(h, X, dev, mode, ld, int(nrhs), W.xp.p);
        const double l = loss_grad(h, net, gd, W, ax, int(nrhs));
        if (!std::isfinite(l)) throw StatusError(MFS_INVALID_ARG, "training loss is not finite");
        net->step += 1;
        lpc_adam(net->w.p, net->wb.p, net->m.p, net->v.p, net->grad.p, net->n, lr, net->step, h->stream);
        MFS_LAUNCHED();
        MFS_CUDA(cudaStreamSynchronize(h->stream));
        if (loss) *loss = l;
    });
}

mfs_status mfs_pcg_solve(mfs_handle *h, mfs_lpc *net, const double *Ax, const double *B, double *X, int64_t nrhs,
                         int64_t ld, int32_t flags, int32_t maxit, double tol, int32_t *iterations) {
    if (!h || !B || !X) return MFS_INVALID_ARG;
    int fallback = 0;
    const mfs_status s = guarded(h, [&] {
        const int mode = flags & 3;
        const bool dev = (flags & MFS_DEVICE_POINTERS) != 0;
        check_common(h, nrhs, ld, mode);
        check_net(h, net);
        set_device(h);
        cudaStream_t st = h->stream;
        LGraphDev &gd = graph_of(h);
        LWorkDev &W = work_of(h, gd, int(nrhs));
        const LGraph &g = gd.g;
        const int nr = int(nrhs);
        const int64_t n = 3 * g.nv;
        const size_t sz = size_t(n) * nr;
        if (maxit <= 0) maxit = 200;
        if (!(tol > 0)) tol = 1e-10;
        MFS_CUDA(cudaEventRecord(h->ev0, st));
        const double *ax = values_of(h, W, Ax, dev);
        gather_in(h, B, dev, mode, ld, nr, W.bp.p);
        lpc_features(g, ax, W.w, st);
        if (net) lpc_forward(g, net->wb.p, W.w, st);
        MFS_LAUNCHED();
        // z = M^{-1} r: D^{-1/2} G^T G D^{-1/2} r, or D^{-1} r without a network
        auto precond = [&](const double *r, double *z) {
            if (net) {
                lpc_gmv(g, W.G.p, false, r, W.t.p, n, nr, W.dinv.p, nullptr, st);
                lpc_gmv(g, W.G.p, true, W.t.p, z, n, nr, nullptr, W.dinv.p, st);
            } else {
                lpc_scale_rows(r, W.dinv.p, false, W.t.p, n, nr, n, st);
                lpc_scale_rows(W.t.p, W.dinv.p, false, z, n, nr, n, st);
            }
        };
        double *bb = W.dots.p, *rz = W.dots.p + nr, *rz2 = W.dots.p + 2 * nr, *pap = W.dots.p + 3 * nr;
        std::vector<int> act(static_cast<size_t>(nr), 1);
        launch_colnorm2(W.bp.p, n, nr, W.partials.p, bb, st);
        MFS_CUDA(cudaMemsetAsync(W.xp.p, 0, sz * sizeof(double), st));
        launch_copy(W.r.p, W.bp.p, int64_t(sz), st);
        precond(W.r.p, W.pz.p);
        launch_copy(W.p.p, W.pz.p, int64_t(sz), st);
        launch_coldot(W.r.p, W.pz.p, n, nr, W.partials.p, rz, st);
        MFS_LAUNCHED();
        std::vector<double> hb(static_cast<size_t>(nr)), hr(static_cast<size_t>(nr));
        MFS_CUDA(cudaMemcpyAsync(hb.data(), bb, nr * sizeof(double), cudaMemcpyDeviceToHost, st));
        MFS_CUDA(cudaStreamSynchronize(st));
        for (int r = 0; r < nr; ++r)
            if (hb[r] == 0.0) act[r] = 0;
        MFS_CUDA(cudaMemcpyAsync(W.active.p, act.data(), nr * sizeof(int), cudaMemcpyHostToDevice, st));
        int it = 0;
        bool done = std::none_of(act.begin(), act.end(), [](int a) { return a != 0; });
        double worst = 0.0;
        while (!done && it < maxit) {
            ++it;
            spmv(h, ax, W.p.p, W.ap.p, nr);
            launch_coldot(W.p.p, W.ap.p, n, nr, W.partials.p, pap, st);
            launch_pcg_update_x_r(W.xp.p, W.r.p, W.p.p, W.ap.p, rz, pap, W.active.p, n, nr, st);
            launch_colnorm2(W.r.p, n, nr, W.partials.p, rz2, st);
            MFS_LAUNCHED();
            MFS_CUDA(cudaMemcpyAsync(hr.data(), rz2, nr * sizeof(double), cudaMemcpyDeviceToHost, st));
            MFS_CUDA(cudaStreamSynchronize(st));
            worst = 0.0;
            done = true;
            for (int r = 0; r < nr; ++r) {
                const double rel = hb[r] > 0 ? std::sqrt(hr[r] / hb[r]) : 0.0;
                if (act[r] && rel <= tol) act[r] = 0;
                if (act[r]) done = false;
                worst = std::max(worst, rel);
            }
            if (done) break;
            MFS_CUDA(cudaMemcpyAsync(W.active.p, act.data(), nr * sizeof(int), cudaMemcpyHostToDevice, st));
            precond(W.r.p, W.pz.p);
            launch_coldot(W.r.p, W.pz.p, n, nr, W.partials.p, rz2, st);
            launch_pcg_update_p(W.p.p, W.pz.p, rz2, rz, W.active.p, n, nr, st);
            MFS_LAUNCHED();
            MFS_CUDA(cudaMemcpyAsync(rz, rz2, nr * sizeof(double), cudaMemcpyDeviceToDevice, st));
        }
        h->stats.pcg_iterations = it;
        h->stats.residual = worst;
        if (done) {
            MFS_CUDA(cudaEventRecord(h->ev1, st));
            scatter_out(h, W.xp.p, X, dev, mode, ld, nr);
            MFS_CUDA(cudaStreamSynchronize(st));
            float ms = 0;
            cudaEventElapsedTime(&ms, h->ev0, h->ev1);
            h->stats.pcg_ms = ms;
            if (iterations) *iterations = it;
            return;
        }
        fallback = 1;
        if (iterations) *iterations = it;
    });
    if (s != MFS_OK) return s;
    h->stats.pcg_fallback = fallback;
    if (!fallback) return MFS_OK;
    // PCG missed the tolerance within the cap: factor the same values and solve.
    mfs_status f = mfs_numeric(h, Ax, nullptr, 0.0, flags & MFS_DEVICE_POINTERS);
    if (f != MFS_OK) return f;
    f = mfs_solve(h, B, X, nrhs, ld, flags);
    h->stats.pcg_fallback = 1;
    return f;
}

}  // extern "C"
