#!/usr/bin/env python
"""Benchmark: Newton-step solves/s (assemble -> factor -> solve to ||b-Hx||/||b|| <= 1e-10).

One "step" = one Newton solve of the configured workload: on-device element
assembly (K1), numeric factorization (K2-K5) and the multi-RHS solve (K6) with
FP64 refinement (K7 residuals) for the FP32 form. `value` times that with the
element Hessians and right-hand sides already resident in HBM; `e2e` times the
same step through the C ABI with host (pinned) buffers, copies included.

Multi-GPU: the path does not shard (one sparse factorization per step), so
`--gpus N` runs N independent replicas (one per rank, no collective on the data
path); value = solves of all ranks / max-over-ranks device time.

`--impl reference` times the CPU restatement of the reference path (the oracle
port: FP64 supernodal multifrontal factor + solve with OpenBLAS dense kernels,
all host threads) on complete steps of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Newton solves/s at 1e-10 residual: FP32+refine & learned PCG vs FP64 plain"
UNIT = "solves/s"
# DRAM bytes (read + write) of the split-FP16 GEMM launches over one config-2
# factorization: ncu capture of `bench.py --profile`, gemm_tma 72.73 + 29.0 GB,
# gemm_tc 6.78 + 3.5 GB (captured with one 256-column CTA per split tile; the two
# 128-column CTAs that now share a tile read its A operand twice, the second time
# mostly from L2)
GEMM_TRAFFIC_SPLIT16_CONFIG2 = 112.0e9


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--config", type=int, default=2)
    p.add_argument("--k", type=int, default=None, help="override the cube side (smaller runs)")
    p.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison arm")
    p.add_argument("--no-config4", action="store_true",
                   help="default workload: skip the short learned-PCG Newton-sequence arm (config 4) whose summary "
                        "the line carries under \"config4\"")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    p.add_argument("--tc", type=int, default=0,
                   help="FP32 Schur updates: 0 auto (6 under refinement), 1 TF32, 2 split 3xTF32, 4 TF32 with TMA, "
                        "5 FP16 operands with TMA, 6 split FP16 (hi/lo) operands with TMA")
    p.add_argument("--profile", action="store_true",
                   help="build the workload, run one untimed assemble + factorization + refined solve, exit "
                        "(the command profilers capture)")
    p.add_argument("--maxit", type=int, default=50, help="refinement iteration cap")
    p.add_argument("--gemm-table", default=None,
                   help="write the per-launch GEMM record (ms, flops, tiles, tasks, kind) of the kernel-timed "
                        "factorization to this file")
    p.add_argument("--group", type=int, default=0, help="column blocks per factorization group (0: default)")
    p.add_argument("--subtrees", type=int, default=0,
                   help="subtree count the solve cut aims for (0: default)")
    p.add_argument("--chain", type=int, default=0, help="diagonal solves: 0 superblock inverses, 1 block-pair chains")
    p.add_argument("--cpu-seconds", type=float, default=150.0,
                   help="reference arm: stop timing complete CPU steps once this much is spent")
    p.add_argument("--train-hessians", type=int, default=10, help="config 4: Hessians of the training set")
    p.add_argument("--train-steps", type=int, default=300, help="config 4: Adam steps before timing")
    return p.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "b200" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        pg = dist
    return rank, world, local, pg


def max_over_ranks(value: float, dist, device) -> float:
    """The largest of every rank's value (a timed region's device time): replicas report
    the slowest rank. Every rank must call it at the same point."""
    if not dist:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return json.load(fh), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "500", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------- GPU arm
def run_b200(args, rank, world, local, dist):
    import torch
    from meshfemsparse_b200 import B200Factorizer, _lib, workloads

    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    t0 = time.time()
    wl = workloads.build(args.config, k=args.k, device=dev)
    t_gen = time.time() - t0
    stream = torch.cuda.current_stream()
    lib = _lib.load()
    n_full = wl.n_full
    nrhs = wl.nrhs

    def make(single):
        f = B200Factorizer(single, refine=single, stream=stream.cuda_stream, device=local, tensor_cores=args.tc,
                           refine_maxit=args.maxit, solve_chain=args.chain, factor_group=args.group,
                           solve_subtrees=args.subtrees)
        t = time.time()
        f.factorizeSymbolic(wl.H, wl.pins)
        f.setElements(wl.tets)
        return f, time.time() - t

    f32, t_sym = make(True)
    Ke_dev = torch.from_numpy(wl.Ke.reshape(-1)).to(dev)
    B_dev = torch.from_numpy(np.ascontiguousarray(wl.rhs.T)).to(dev)        # column-major n_full x nrhs
    X_dev = torch.empty_like(B_dev)
    D = _lib.MFS_DEVICE_POINTERS

    def step(f, Ke_ptr, B_ptr, X_ptr, flags):
        _lib.check(lib.mfs_assemble(f._h, Ke_ptr, None, flags), f._h, "assemble")
        _lib.check(lib.mfs_numeric(f._h, None, None, 0.0, 0), f._h, "numeric")
        _lib.check(lib.mfs_solve(f._h, B_ptr, X_ptr, nrhs, n_full, _lib.MFS_SOLVE_FULL | flags), f._h, "solve")

    def timed(f, K, W, Ke_ptr, B_ptr, X_ptr, flags, sample_clocks=False):
        for _ in range(W):
            step(f, Ke_ptr, B_ptr, X_ptr, flags)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        l0 = f.stats()["kernel_launches"]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            step(f, Ke_ptr, B_ptr, X_ptr, flags)
        e1.record(stream)
        torch.cuda.synchronize()
        launches = f.stats()["kernel_launches"] - l0
        clocks = sampler.stop() if sampler else None
        total = e0.elapsed_time(e1)
        total = max_over_ranks(total, dist, dev)
        if dist:
            dist.barrier()
        return total, launches, clocks

    pK, pB, pX = C.c_void_p(Ke_dev.data_ptr()), C.c_void_p(B_dev.data_ptr()), C.c_void_p(X_dev.data_ptr())
    if args.profile:
        step(f32, pK, pB, pX, D)
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"profile_step": f32.stats()}), flush=True)
        return
    tot32, launches, clocks = timed(f32, args.steps, args.warmup, pK, pB, pX, D, sample_clocks=True)
    st32 = f32.stats()
    ms32 = tot32 / args.steps

    # residual of the timed FP32+refine result, checked in FP64 on the device
    def residual(f, X):
        Y = torch.empty_like(X)
        _lib.check(lib.mfs_apply(f._h, C.c_void_p(X.data_ptr()), C.c_void_p(Y.data_ptr()), nrhs, n_full,
                                 _lib.MFS_SOLVE_FULL | D), f._h, "apply")
        keep = torch.ones(n_full, dtype=torch.bool, device=dev)
        keep[torch.from_numpy(wl.pins).to(dev)] = False
        R = (B_dev - Y)[:, keep]
        return float((R.norm(dim=1) / B_dev[:, keep].norm(dim=1)).max().item())

    res32 = residual(f32, X_dev)

    # e2e through host (pinned) buffers
    Ke_h = torch.from_numpy(wl.Ke.reshape(-1)).pin_memory()
    B_h = torch.from_numpy(np.ascontiguousarray(wl.rhs.T)).pin_memory()
    X_h = torch.empty_like(B_h).pin_memory()
    K_e2e = max(1, min(args.steps, 3))
    tot_e2e, _, _ = timed(f32, K_e2e, 1, C.c_void_p(Ke_h.data_ptr()), C.c_void_p(B_h.data_ptr()),
                          C.c_void_p(X_h.data_ptr()), 0)
    e2e_ms = tot_e2e / K_e2e

    peaks, peak_kind = measured_peaks()
    flops = f32.getFlopEstimate()
    achieved_seq = flops / (st32["factor_ms"] * 1e-3) / 1e12
    # Dominant kernel (tcgen05 TF32 GEMM: Schur updates, row solves, SYRK), timed live:
    # one extra untimed factorization with a CUDA-event pair around every GEMM launch
    # on its own stream; achieved = the launches' algorithmic flops / their summed time.
    f32._opts.time_kernels = 1
    _lib.check(lib.mfs_set_options(f32._h, C.byref(f32._opts)), f32._h, "options")
    step(f32, pK, pB, pX, D)
    torch.cuda.synchronize()
    stk = f32.stats()
    if args.gemm_table:
        np.savetxt(args.gemm_table, _lib.debug_gemm_launches(f32._h), fmt="%.6g",
                   header="ms flops tiles tasks kind(0 left,1 rowsolve,2 next-group,3 trailing,4 syrk)")
    f32._opts.time_kernels = 0
    _lib.check(lib.mfs_set_options(f32._h, C.byref(f32._opts)), f32._h, "options")
    gemm_tf = stk["gemm_flops"] / (stk["gemm_ms"] * 1e-3) / 1e12 if stk["gemm_ms"] > 0 else None
    flops_est, nnz32, nred = flops, f32.getFactorNNZ(), f32.n_reduced()
    sym = None
    if rank == 0 and world == 1 and not args.no_cpu:
        sym = (f32.supernodes(), f32.conversionPlan(), f32._row_maps()[1])
    # the FP32 handle is released before the FP64 arm (the largest workloads do not
    # hold both factorizations at once)
    del f32
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    out64 = {}
    if not args.no_fp64:
        try:
            f64, _ = make(False)
            X64 = torch.empty_like(B_dev)
            K64 = max(1, min(args.steps, 3))
            tot64, _, _ = timed(f64, K64, 1, pK, pB, C.c_void_p(X64.data_ptr()), D)
            ms64 = tot64 / K64
            st64 = f64.stats()
            out64 = {"fp64_plain_solves_per_s": world * 1000.0 / ms64, "fp64_plain_ms_per_step": ms64,
                     "fp64_factor_ms": st64["factor_ms"], "fp64_solve_ms": st64["solve_ms"],
                     "fp64_residual": residual(f64, X64),
                     "speedup_fp32_refine_vs_fp64_plain": ms64 / ms32}
            del f64
        except (_lib.MFSError, torch.OutOfMemoryError) as e:
            # the FP64 factorization of the largest workloads may not fit beside the inputs
            out64 = {"fp64_plain": f"unavailable: {str(e)[:160]}"}

    peak = peaks["bf16_tflops_sustained"]
    half = args.tc == 5
    split16 = args.tc in (0, 6)
    # DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) over the GEMM launches
    # of one factorization of the full-size workload (per operand mode, group width 4)
    traffic_by_mode = {(2, True): GEMM_TRAFFIC_SPLIT16_CONFIG2, (2, False): 89.9e9}
    gemm_traffic = (traffic_by_mode.get((args.config, split16)) if ((half or split16) and args.k is None
                                                                   and args.group in (0, 4)) else None)
    roofline = {"bound": "tensor", "achieved": gemm_tf, "peak": peak, "unit": "TFLOP/s",
                "frac": (gemm_tf / peak) if gemm_tf else None, "traffic": gemm_traffic,
                "traffic_unit": "DRAM bytes per factorization over the same GEMM launches (ncu capture of this workload)",
                "kernel": ("gemm_tma_kernel (tcgen05 kind::f16, split hi/lo FP16 operands: three MMAs per k slice, "
                           "TMA-fed Schur updates) + gemm_tc_kernel (split-TF32 row solves)" if split16 else
                           "gemm_tma_kernel (tcgen05 kind::f16, TMA-fed Schur updates) + gemm_tc_kernel (row solves)"
                           if half else "gemm_tc_kernel / gemm_tma_kernel (tcgen05 kind::tf32)"),
                "launches": stk["gemm_launches"], "kernel_ms_per_factorization": stk["gemm_ms"],
                "kernel_flops_per_factorization": stk["gemm_flops"],
                "note": f"algorithmic flops of the launches' tasks / CUDA-event time per launch, summed over one "
                        f"factorization; peak = {peak_kind} sustained dense bf16 (the FP16 rate; TF32 is half of it); "
                        f"whole factorization sequence: {achieved_seq:.1f} TFLOP/s of the symbolic flop count"}

    result = {
        "metric": METRIC, "value": world * 1000.0 * 1.0 / ms32, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms32, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 factor / f64 refine", "data": "synthetic",
        "config": {"workload": f"config{args.config}:{wl.name}", "n_free_dofs": nred,
                   "tets": int(wl.tets.shape[0]), "nrhs": nrhs, "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (element Hessians %.2f GB)" % (wl.Ke.nbytes / 1e9),
                   **wl.info},
        "e2e": {"value": world * 1000.0 / e2e_ms, "unit": UNIT,
                "h2d_bytes_per_step": int(wl.Ke.nbytes + wl.rhs.nbytes), "d2h_bytes_per_step": int(wl.rhs.nbytes)},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "roofline": roofline,
        "residual": res32,
        "refine_iterations": st32["refine_iterations"], "perturbed_pivots": st32["perturbed_pivots"],
        "refactored_blocks": st32["refactored_blocks"], "split_escalations": st32["split_escalations"],
        "factor_ms": st32["factor_ms"], "solve_ms": st32["solve_ms"], "assemble_ms": st32["assemble_ms"],
        "factor_nnz": nnz32, "flops": flops_est, "symbolic_s": t_sym, "input_gen_s": t_gen,
        **out64,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        result["cpu_baseline"] = cpu_baseline(wl, sym, args)
    if rank == 0:
        return result
    return None


# ------------------------------------------------- config 4: learned PCG on a Newton sequence
def run_newton_sequence(args, rank, world, local, dist):
    """Learned-PCG form on the 30-step load ramp, beside FP32+refine and FP64 plain.

    Untimed: the network is trained on `--train-hessians` Hessians at seeded random
    loads (20 right-hand sides each, solutions from the FP64 factor). Timed: `--steps`
    load steps of the ramp (each its own Hessian, resident on the device); one step =
    assemble -> PCG with the learned G (cap 200, tolerance 1e-10) -> Cholesky fallback
    (FP32 factor + FP64 refinement) when PCG misses."""
    import torch
    from meshfemsparse_b200 import B200Factorizer, _lib, workloads
    from meshfemsparse_b200.learned import LearnedPreconditioner

    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    lib = _lib.load()
    D = _lib.MFS_DEVICE_POINTERS
    FULL = _lib.MFS_SOLVE_FULL
    t0 = time.time()
    seq = workloads.newton_sequence(k=args.k or 48, final_hessians=False)
    wl = seq.wl
    n_full, nrhs = wl.n_full, wl.nrhs
    stream = torch.cuda.current_stream()

    def make(single):
        f = B200Factorizer(single, refine=single, stream=stream.cuda_stream, device=local, refine_maxit=args.maxit)
        f.factorizeSymbolic(wl.H, wl.pins)
        f.setElements(wl.tets)
        return f

    f32, f64 = make(True), make(False)
    rng = np.random.default_rng(44)
    keep = np.ones(n_full, dtype=bool)
    keep[wl.pins] = False
    # ---- training data from the FP64 factor
    train = []
    for i in range(args.train_hessians):
        Ke = torch.from_numpy(seq.hessians(float(rng.uniform(0.0, seq.max_strain)), seed=1000 + i,
                                           device=dev).reshape(-1)).to(dev)
        Ax = torch.empty(int(f64._axlen), dtype=torch.float64, device=dev)
        _lib.check(lib.mfs_assemble(f64._h, C.c_void_p(Ke.data_ptr()), C.c_void_p(Ax.data_ptr()), D), f64._h, "asm")
        _lib.check(lib.mfs_numeric(f64._h, None, None, 0.0, 0), f64._h, "numeric")
        Bh = rng.normal(size=(20, n_full))
        Bh[:, ~keep] = 0.0
        B = torch.from_numpy(Bh).to(dev)
        X = torch.empty_like(B)
        _lib.check(lib.mfs_solve(f64._h, C.c_void_p(B.data_ptr()), C.c_void_p(X.data_ptr()), 20, n_full, FULL | D),
                   f64._h, "solve")
        train.append((Ax, B, X))
        del Ke
    t_data = time.time() - t0
    net = LearnedPreconditioner(device=local, seed=4)
    torch.cuda.synchronize()
    t1 = time.time()
    losses = []
    for it in range(args.train_steps):
        Ax, B, X = train[it % len(train)]
        losses.append(net.train_step(f32, B.data_ptr(), X.data_ptr(), lr=2e-3, Ax=Ax.data_ptr(),
                                     device_pointers=True, nrhs=20, ld=n_full))
    torch.cuda.synchronize()
    t_train = time.time() - t1
    del train
    # ---- the timed load steps (Hessians resident on the device)
    K = args.steps
    ts = [int(round(seq.steps * (i + 1) / K)) for i in range(K)]
    Kes = [torch.from_numpy(seq.hessians(seq.strain(t), device=dev).reshape(-1)).to(dev) for t in ts]
    B = torch.from_numpy(np.ascontiguousarray(wl.rhs.T)).to(dev)
    X = torch.empty_like(B)
    it_c = C.c_int32()

    def step_pcg(f, Ke, netp, Bp, Xp, flags):
        _lib.check(lib.mfs_assemble(f._h, Ke, None, flags), f._h, "assemble")
        _lib.check(lib.mfs_pcg_solve(f._h, netp, None, Bp, Xp, nrhs, n_full, FULL | flags, 200, 1e-10,
                                     C.byref(it_c)), f._h, "pcg")
        st = f.stats()
        return int(it_c.value), bool(st["pcg_fallback"])

    def step_factor(f, Ke, Bp, Xp, flags):
        _lib.check(lib.mfs_assemble(f._h, Ke, None, flags), f._h, "assemble")
        _lib.check(lib.mfs_numeric(f._h, None, None, 0.0, 0), f._h, "numeric")
        _lib.check(lib.mfs_solve(f._h, Bp, Xp, nrhs, n_full, FULL | flags), f._h, "solve")
        return f.stats()["refine_iterations"], False

    def run(fn, W, sample_clocks=False):
        for i in range(W):
            fn(i % K)
        torch.cuda.synchronize()
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        l0 = f32.stats()["kernel_launches"]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        info = [fn(i) for i in range(K)]
        e1.record(stream)
        torch.cuda.synchronize()
        launches = f32.stats()["kernel_launches"] - l0
        clocks = sampler.stop() if sampler else None
        total = e0.elapsed_time(e1)
        total = max_over_ranks(total, dist, dev)
        return total / K, info, launches, clocks

    pB, pX = C.c_void_p(B.data_ptr()), C.c_void_p(X.data_ptr())
    ms_l, info_l, launches, clocks = run(lambda i: step_pcg(f32, C.c_void_p(Kes[i].data_ptr()), net._p, pB, pX, D),
                                         args.warmup, sample_clocks=True)

    def residual(f):
        Y = torch.empty_like(X)
        _lib.check(lib.mfs_apply(f._h, pX, C.c_void_p(Y.data_ptr()), nrhs, n_full, FULL | D), f._h, "apply")
        m = torch.from_numpy(keep).to(dev)
        R = (B - Y)[:, m]
        return float((R.norm(dim=1) / B[:, m].norm(dim=1)).max().item())

    res_l = residual(f32)
    ms_j, info_j, _, _ = run(lambda i: step_pcg(f32, C.c_void_p(Kes[i].data_ptr()), None, pB, pX, D), 1)
    ms_32, info_32, _, _ = run(lambda i: step_factor(f32, C.c_void_p(Kes[i].data_ptr()), pB, pX, D), 1)
    res_32 = residual(f32)
    ms_64, _, _, _ = run(lambda i: step_factor(f64, C.c_void_p(Kes[i].data_ptr()), pB, pX, D), 1)
    res_64 = residual(f64)
    # e2e of the learned form through host (pinned) buffers
    Ke_h = [k.cpu().pin_memory() for k in Kes[:min(K, 3)]]
    B_h = B.cpu().pin_memory()
    X_h = torch.empty_like(B_h).pin_memory()
    Ke_bytes = Kes[0].numel() * 8
    del Kes
    torch.cuda.empty_cache()
    Ke2 = Ke_h
    K2 = len(Ke2)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(K2):
        step_pcg(f32, C.c_void_p(Ke2[i].data_ptr()), net._p, C.c_void_p(B_h.data_ptr()), C.c_void_p(X_h.data_ptr()), 0)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / K2

    peaks, peak_kind = measured_peaks()
    result = {
        "metric": METRIC, "value": world * 1000.0 / ms_l, "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": args.warmup, "ms_per_step": ms_l, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 network / f64 PCG", "data": "synthetic",
        "config": {"workload": f"config4:{wl.name}", "n_free_dofs": f32.n_reduced(), "tets": int(wl.tets.shape[0]),
                   "nrhs": nrhs, "parallelism": f"replicas{world}", "load_steps_timed": ts,
                   "l2": "inputs larger than L2 (element Hessians %.2f GB per step)" % (Ke_bytes / 1e9),
                   **wl.info},
        "e2e": {"value": world * 1000.0 / e2e_ms, "unit": UNIT, "h2d_bytes_per_step": int(Ke_bytes + B.numel() * 8),
                "d2h_bytes_per_step": int(B.numel() * 8)},
        "gpu_launches": int(launches), "clocks": clocks,
        "roofline": None,
        "residual": res_l,
        "learned_pcg": {"iterations": [i for i, _ in info_l], "fallbacks": int(sum(fb for _, fb in info_l)),
                        "cap": 200},
        "jacobi_pcg": {"solves_per_s": 1000.0 / ms_j, "iterations": [i for i, _ in info_j],
                       "fallbacks": int(sum(fb for _, fb in info_j))},
        "fp32_refine": {"solves_per_s": 1000.0 / ms_32, "refine_iterations": [i for i, _ in info_32],
                        "residual": res_32},
        "fp64_plain_solves_per_s": world * 1000.0 / ms_64, "fp64_plain_ms_per_step": ms_64, "fp64_residual": res_64,
        "speedup_learned_pcg_vs_fp64_plain": ms_64 / ms_l, "speedup_fp32_refine_vs_fp64_plain": ms_64 / ms_32,
        "training": {"hessians": args.train_hessians, "pairs": 20 * args.train_hessians, "steps": args.train_steps,
                     "seconds": t_train, "data_seconds": t_data, "loss_first": float(np.mean(losses[:10])),
                     "loss_last": float(np.mean(losses[-10:]))},
        "peaks": peak_kind,
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        wl.Ke = Ke2[-1].numpy().reshape(-1, 12, 12)
        result["cpu_baseline"] = cpu_baseline(wl, (f32.supernodes(), f32.conversionPlan(), f32._row_maps()[1]), args)
    return result if rank == 0 else None


# -------------------------------------------------------------- CPU legs
def cpu_step(wl, sn, plan, prr, threads):
    """One complete Newton step of the workload on the host cores with the oracle port
    (FP64 multifrontal factorization + supernodal solve, OpenBLAS dense kernels, all
    host threads): element assembly, value injection, numeric factorization of the
    whole tree and the multi-RHS solve. Returns the stage times and the pivot status."""
    from oracle import pyoracle
    w, d, fr, pan, col0 = pyoracle.panel_layout(sn)
    pyoracle.set_range(0, -1)
    t = time.time()
    Ax = pyoracle.assemble(wl.H.numBlocks, wl.H.Ap, wl.H.Ai, wl.tets, wl.Ke)
    t_asm = time.time() - t
    t = time.time()
    vals = pyoracle.inject(plan["entries"], sn["vb"], 3, Ax, int(pan[-1]))
    t_inj = time.time() - t
    t = time.time()
    fail = pyoracle.mf_factor(sn, vals, threads)
    t_fac = time.time() - t
    n = int(w.sum())
    keep = prr >= 0
    t = time.time()
    B = np.zeros((n, wl.rhs.shape[1]))
    B[prr[keep]] = wl.rhs[keep]                     # pins removed, permuted reduced order
    X = pyoracle.mf_solve(sn, vals, B, threads)
    x_full = np.zeros_like(wl.rhs)
    x_full[keep] = X[prr[keep]]
    t_sol = time.time() - t
    return {"total": t_asm + t_inj + t_fac + t_sol, "asm": t_asm, "inject": t_inj, "factor": t_fac,
            "solve": t_sol, "pivot_failure": int(fail)}


def cpu_baseline(wl, sym, args):
    """The oracle port timed on one complete step of the same workload (no sampling,
    no extrapolation) on all host threads. sym: (supernodes, conversion plan, row map)
    of the factorizer's symbolic analysis."""
    from oracle import pyoracle
    pyoracle.load_blas()
    threads = int(pyoracle.load().orc_max_threads())
    r = cpu_step(wl, sym[0], sym[1], sym[2], threads)
    return {"value": 1.0 / r["total"], "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"one complete step of the same workload (nrhs={wl.nrhs}): CPU assembly, injection, "
                      f"FP64 multifrontal factorization of the whole tree and supernodal solve with OpenBLAS; "
                      f"{r['asm']:.2f}s asm, {r['inject']:.2f}s inject, {r['factor']:.2f}s factor, "
                      f"{r['solve']:.2f}s solve",
            "pivot_failure": r["pivot_failure"]}


def run_reference(args, rank, world, dist):
    """The CPU reference arm: complete steps of the workload (assembly, injection, whole-tree
    FP64 factorization, solve) with the oracle port on all host threads. One untimed
    warm-up step, then timed complete steps until --steps are done or --cpu-seconds of
    timed work is spent (at least one); `steps` reports the steps actually timed."""
    if rank != 0:
        return
    from meshfemsparse_b200 import B200Factorizer, workloads
    from oracle import pyoracle
    wl = workloads.build(args.config, k=args.k, device=None)
    f = B200Factorizer(False, device=-1)        # host-only analysis (ordering, supernodes, plan)
    f.factorizeSymbolic(wl.H, wl.pins)
    sn, plan, prr = f.supernodes(), f.conversionPlan(), f._row_maps()[1]
    pyoracle.load_blas()
    threads = int(pyoracle.load().orc_max_threads())
    warm = cpu_step(wl, sn, plan, prr, threads) if args.warmup > 0 else None
    runs = []
    t_start = time.time()
    while len(runs) < args.steps:
        runs.append(cpu_step(wl, sn, plan, prr, threads))
        if time.time() - t_start + runs[-1]["total"] > args.cpu_seconds:
            break
    ms = 1000.0 * float(np.mean([r["total"] for r in runs]))
    value = 1000.0 / ms
    stages = {k: float(np.mean([r[k] for r in runs])) for k in ("asm", "inject", "factor", "solve")}
    sample = (f"complete steps of the workload (nrhs={wl.nrhs}): CPU assembly, injection, FP64 multifrontal "
              f"factorization of the whole tree and supernodal solve with OpenBLAS; mean of {len(runs)} timed "
              f"step(s): " + ", ".join(f"{v:.2f}s {k}" for k, v in stages.items()))
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
           "steps": len(runs), "warmup": 1 if warm else 0, "steps_requested": args.steps,
           "warmup_requested": args.warmup, "ms_per_step": ms, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": f"config{args.config}:{wl.name}", "nrhs": wl.nrhs, **wl.info},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                            "pivot_failure": runs[-1]["pivot_failure"]},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def config4_summary(args, rank, world, local, dist):
    """A short run of the config-4 arm (learned PCG on the Newton load ramp, beside
    FP32+refine and FP64 plain on the same steps), summarized for the default line."""
    import copy
    a = copy.copy(args)
    a.config, a.k, a.steps, a.warmup, a.no_cpu = 4, None, 3, 3, True
    a.train_hessians = min(args.train_hessians, 4)
    r = run_newton_sequence(a, rank, world, local, dist)
    if r is None:
        return None
    keep = ("value", "ms_per_step", "residual", "learned_pcg", "jacobi_pcg", "fp32_refine", "fp64_plain_solves_per_s",
            "fp64_plain_ms_per_step", "fp64_residual", "speedup_learned_pcg_vs_fp64_plain",
            "speedup_fp32_refine_vs_fp64_plain", "training", "steps", "warmup", "e2e")
    out = {k: r[k] for k in keep if k in r}
    out["workload"] = r["config"]["workload"]
    out["n_free_dofs"] = r["config"]["n_free_dofs"]
    out["unit"] = UNIT
    return out


def main():
    args = parse()
    rank, world, local, dist = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, rank, world, dist)
        elif args.config == 4:
            result = run_newton_sequence(args, rank, world, local, dist)
            if result is not None:
                print(json.dumps(result), flush=True)
        else:
            result = run_b200(args, rank, world, local, dist)
            if (result is not None and args.config == 2 and world == 1 and not args.no_config4
                    and not args.profile and args.k is None):
                import torch
                torch.cuda.empty_cache()
                result["config4"] = config4_summary(args, rank, world, local, dist)
            if result is not None:
                print(json.dumps(result), flush=True)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
