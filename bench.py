#!/usr/bin/env python
"""Benchmark: time to FP64 relative residual 1e-8 on the 256^3 HPCCG matrix.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 256]

One step = one complete solve of A x = b on the 27-point generate_matrix
operator (MPI/src/SparseMatrix.F90:68-185) at n^3 (default 256^3: 16,777,216
rows, 449,455,096 nonzeros), b = A x* with x* i.i.d. U[-1,1) from the project's
counter-based generator (seed 1234), x0 = 0, FP64 CG (MPI/src/numerics.F90:41-162)
stopped when ||r|| < 1e-8 ||b||; the FP64 true residual is checked afterwards.
Inputs (5.4 GB of matrix) are far larger than the 126 MB L2, so no flush is
needed between steps.

Solvers timed: plain FP64 CG (the reference's algorithm), and FP64 iterative
refinement around an FP32 or BF16-value inner CG, each on the stored matrix
(column-major ELL copy of the CSR, the reference's representation); then the
same FP64 CG and the FP32 refinement with the matrix-free stencil SpMV (the
operator checked equal to the CSR entry by entry; FP64 results bit-identical),
and, unless --no-learned, the flexible PCG with the U-Net trained in-run.  `value` is the device time
of one solve of the fastest solver whose FP64 true residual meets 1e-8 (CUDA
events on the library stream, max over ranks); config.methods lists every
solver.  `e2e` is the same solve through the host-array C-ABI call
(hpccg_gpu_cg / hpccg_gpu_solve_mixed) with b and x0 copied from pinned host
memory and x copied back inside the timed region.  `roofline` covers the
dominant kernel of that solver.  `cpu_baseline` times whole solves of the same
system by the CPU oracle (a C restatement of the reference, OpenMP over all
host cores; one-thread figure beside it).

N > 1 GPUs run independent replicas (the path does not shard at one rank:
no collective in the data path); each rank solves its own system and the
reported time is the max over ranks.

`--impl reference` times the reference's algorithm on the host cores instead
(the Fortran reference cannot be compiled here: no Fortran compiler; the C
restatement in oracle/ is used) and prints the same JSON line with
"impl": "reference".
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "hpccg-f90_b200"))

METRIC = ("s to rel-res 1e-8 @256^3 (FP64 true residual), best of FP64 CG / mixed-precision IR "
          "(stored-matrix ELL or checked matrix-free stencil SpMV)")
SEED_XSTAR = 1234
REL_TOL = 1e-8


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), float(d.get("bf16_tflops", 1590.0)), "measured"
    return 6650.0, 1590.0, "fallback"


def _bf16_sustained():
    """(burst, sustained, source) BF16 dense TFLOP/s from MEASURED_PEAKS.json, else the fallback figures."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        burst = float(d.get("bf16_tflops", 1590.0))
        return burst, float(d.get("bf16_tflops_sustained", burst)), "measured"
    return 1590.0, 1400.0, "fallback"


# The U-Net's 3x3x3 convolutions as (input channels, level): level l runs on the grid coarsened
# 2^l times per axis (csrc/unet.cu, kLayers), each layer 16 output channels; plus the 16 -> 1
# projection at level 0.
UNET_CONVS = [(1, 0), (16, 0), (16, 1), (16, 1), (16, 2), (16, 2), (16, 3), (16, 3), (32, 2), (16, 2),
              (32, 1), (16, 1), (32, 0)]


def unet_forward_flop(nx: int, ny: int, nz: int) -> float:
    """Multiply-add FLOPs (2 per MAC) of one U-Net forward pass on an nx x ny x nz grid."""
    vox = nx * ny * nz
    return float(sum(2 * 27 * cin * 16 * vox / 8 ** lvl for cin, lvl in UNET_CONVS) + 2 * 16 * vox)


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(value: float, backend_device=None) -> float:
    """Max of a float over all ranks of the default process group (or the value itself)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=backend_device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.lines:
            return None
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _traffic_from_profile(name="spmv_dot_fp64_256.txt", key="dram_bytes_per_launch_full_size"):
    """DRAM bytes per launch of a kernel at full size, from a committed ncu summary."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------------------------------
# CPU side: the oracle (a C restatement of the reference) timed on the host cores
# ---------------------------------------------------------------------------------------

def _cpu_problem(n: int):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # the checker / CPU baseline only

    A, x, _, _ = oracle.generate_matrix(n, n, n)
    xstar = oracle.uniform_pm1(SEED_XSTAR, A.nrow)
    b = oracle.spmv(A, xstar, omp=True)
    return oracle, A, b


def cpu_reference_time(n: int, solves: int, warmup: int, solves_1thread: int = 1):
    """Seconds per complete solve to rel-res 1e-8 of the oracle CG (the reference's loop,
    MPI/src/numerics.F90:91-147) with OpenMP on all host cores: the median of `solves` whole
    solves after `warmup` untimed ones.  r, p and Ap are allocated and first-touched once,
    outside the timed region.  The same for the sequential build (one thread), median of
    `solves_1thread` whole solves."""
    oracle, A, b = _cpu_problem(n)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    tol = REL_TOL * float(np.sqrt(np.dot(b, b)))
    x = np.zeros(A.nrow)

    def timed(omp, count, skip):
        work = oracle.CgWork(A, omp=omp)
        out, iters = [], None
        for s in range(skip + count):
            x[:] = 0.0
            t = time.perf_counter()
            iters, _ = work.solve(b, x, 1000, tol)
            dt = time.perf_counter() - t
            if s >= skip:
                out.append(dt)
        return out, iters

    per_solve, iters = timed(True, solves, warmup)
    relres = oracle.true_relres(A, b, x)
    per_solve_1t, iters_1t = timed(False, solves_1thread, 0) if solves_1thread > 0 else ([], None)
    return {"value": float(np.median(per_solve)), "per_solve_s": per_solve, "iters": iters, "cores": cores,
            "relres": relres, "value_1thread": float(np.median(per_solve_1t)) if per_solve_1t else None,
            "per_solve_1thread_s": per_solve_1t, "iters_1thread": iters_1t}


def _host_cpu():
    """The host's CPU model, logical CPUs and the CPUs this process may run on."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        usable = os.cpu_count()
    return {"cpu_model": model, "nproc": usable, "logical_cpus": os.cpu_count()}


def _cpu_sample(r, n):
    s = (f"whole solves to FP64 rel-res 1e-8 of the C restatement of MPI/src CG at {n}^3 ({r['iters']} iterations, "
         f"true rel-res {r['relres']:.2e}): median of {len(r['per_solve_s'])} on {r['cores']} OpenMP threads")
    if r["per_solve_1thread_s"]:
        s += f"; value_1thread: median of {len(r['per_solve_1thread_s'])} on the sequential build"
    return s + "; work arrays allocated once outside the timed region"


def run_reference(args):
    ws, rank, _ = _dist()
    if ws > 1:  # every rank joins (gloo: no GPU work in this arm); rank 0 alone times and prints
        import datetime

        import torch.distributed as dist

        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        ws = dist.get_world_size()
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    r = cpu_reference_time(args.n, args.steps, args.warmup, args.ref_1thread_solves)
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": "s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["value"] * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.n}^3 27-point HPCCG matrix, x* U[-1,1) seed 1234, b = A x*, x0 = 0, FP64 CG to ||r||/||b|| <= 1e-8",
                   "reference_build": "unavailable (Fortran 90; no Fortran compiler in this image) -> C restatement of MPI/src",
                   "iterations": r["iters"], "per_solve_s": r["per_solve_s"]},
        "cpu_baseline": {"value": r["value"], "unit": "s", "cores": r["cores"], "kind": "port",
                         "sample": _cpu_sample(r, args.n), "value_1thread": r["value_1thread"], **_host_cpu()},
        "e2e": {"value": r["value"], "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------------------

def _fp64_relres(M, d_x, d_b, bnorm, scratch):
    """FP64 true residual ||b - A x|| / ||b|| with the library's own kernels."""
    M.spmv(d_x, scratch)
    M.waxpby(1.0, d_b, -1.0, scratch, scratch)
    return float(np.sqrt(M.ddot1(scratch))) / bnorm


def batch_workload(hp, torch, args):
    """The batched-solve workload: 64 systems with (nx, ny, nz) uniform in [16, 96] (seed 7),
    x*_s U[-1,1) (seed 7+s), b_s = A_s x*_s, every system to FP64 rel-res 1e-8.  Times the
    stacked persistent solve (FP64 CG and FP32 refinement) against the same systems solved one
    after another with the single-system FP64 CG graph."""
    sizes = hp.batch_sizes(7, 64, 16, 96)
    B = hp.Batch.generated(sizes)
    xs = B.stack([hp.uniform_pm1_host(7 + s, int(B.nrows[s])) for s in range(B.nsys)])
    d_xs = torch.from_numpy(xs).cuda()
    d_b = torch.empty_like(d_xs)
    B.spmv(d_xs, d_b)
    d_x = torch.zeros_like(d_b)
    out = {"systems": int(B.nsys), "rows": int(B.nrows.sum()), "stacked_rows": int(B.stacked_rows),
           "sizes": "nx,ny,nz uniform in [16,96], seed 7"}
    for name, prec in (("fp64", hp.PREC_FP64), ("fp32_ir", hp.PREC_FP32)):
        times = []
        for rep in range(args.warmup + args.steps):
            d_x.zero_()
            iters, relres, outer, rc = B.solve(d_b, d_x, prec, REL_TOL)
            if rep >= args.warmup:
                times.append(B.last_solve_ms())
        err = max(float((d_x[B.offsets[s]:B.offsets[s] + B.nrows[s]] - d_xs[B.offsets[s]:B.offsets[s] + B.nrows[s]])
                        .abs().max()) for s in range(B.nsys))
        out[name] = {"ms": float(np.median(times)), "status": int(rc), "max_relres": float(relres.max()),
                     "iters_min_max": [int(iters.min()), int(iters.max())], "max_abs_err_vs_xstar": err}
        if name == "fp64":
            fp64_iters = iters.copy()
    out["schedule"] = list(B.get_schedule())
    B.set_spmv(hp.SPMV_STENCIL)  # matrix-free rows, same iterates in FP64
    for name, prec in (("fp64_stencil", hp.PREC_FP64), ("fp32_ir_stencil", hp.PREC_FP32)):
        times = []
        for rep in range(args.warmup + args.steps):
            d_x.zero_()
            iters, relres, outer, rc = B.solve(d_b, d_x, prec, REL_TOL)
            if rep >= args.warmup:
                times.append(B.last_solve_ms())
        err = max(float((d_x[B.offsets[s]:B.offsets[s] + B.nrows[s]] - d_xs[B.offsets[s]:B.offsets[s] + B.nrows[s]])
                        .abs().max()) for s in range(B.nsys))
        out[name] = {"ms": float(np.median(times)), "status": int(rc), "max_relres": float(relres.max()),
                     "iters_min_max": [int(iters.min()), int(iters.max())], "max_abs_err_vs_xstar": err}
        if name == "fp64_stencil":  # the matrix-free rows repeat the stored rows' sums: same iterations
            out[name]["iters_equal_stored"] = bool(np.array_equal(iters, fp64_iters))
            assert out[name]["iters_equal_stored"], "matrix-free FP64 batch took other iteration counts"
    out["schedule_stencil"] = list(B.get_schedule())
    seq = 0.0
    for s, (nx, ny, nz) in enumerate(sizes):
        M = hp.Matrix.generated(int(nx), int(ny), int(nz))
        bs = d_b[B.offsets[s]:B.offsets[s] + B.nrows[s]]
        xsol = torch.zeros_like(bs)
        M.cg_device(bs, xsol, 1000, REL_TOL * float(torch.linalg.vector_norm(bs)), history=False)
        xsol.zero_()
        M.cg_device(bs, xsol, 1000, REL_TOL * float(torch.linalg.vector_norm(bs)), history=False)
        seq += M.last_solve_ms()
        M.close()
    out["sequential_fp64_cg_ms"] = seq
    out["speedup_fp64_vs_sequential"] = seq / out["fp64"]["ms"]
    B.close()
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist

    import hpccg_b200 as hp

    ws, rank, local = _dist()
    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local if ws > 1 else 0)
    torch.cuda.set_device(dev)
    n = args.n
    nz = args.nz or n  # an n x n x nz grid (cubic unless --nz is given)
    N = n * n * nz
    cubic = nz == n
    grid_name = f"{n}^3" if cubic else f"{n}x{n}x{nz}"
    d_x = torch.zeros(N, dtype=torch.float64, device=dev)
    M = hp.Matrix.generated(n, n, nz, d_x, None, None)
    xstar = torch.empty(N, dtype=torch.float64, device=dev)
    M.uniform_pm1(SEED_XSTAR, xstar)
    d_b = torch.empty_like(xstar)
    M.spmv(xstar, d_b)  # b = A x* (bit-identical to the reference's spmv order)
    bnorm = float(np.sqrt(M.ddot1(d_b)))
    tol = REL_TOL * bnorm
    scratch = torch.empty_like(d_b)
    max_iter = 1000
    for prec in (hp.PREC_FP32, hp.PREC_BF16):
        M.set_mixed_rows_per_thread(prec, 4)

    # Each solver: a device solve returning (info dict, kernel launches), run
    # with the SpMV kind listed beside it.
    def fp64_cg():
        it, _, _, st = M.cg_device(d_b, d_x, max_iter, tol, history=False)
        assert st == hp.HPCCG_OK, st
        return {"iterations": it}, 2 + 3 * it

    def mixed(prec):
        def run():
            info, st = M.solve_mixed_device(d_b, d_x, prec, REL_TOL)
            assert st == hp.HPCCG_OK, st
            # inner iteration: three kernels, or one fused pass (plus the first pass of each inner solve)
            fused = M.get_spmv()[0] == hp.SPMV_STENCIL and M.mixed_fused()
            inner = info.inner_iters + info.outer_iters if fused else 3 * info.inner_iters
            # b.b (its own kernel unless fused into the first residual), residuals, inner start/end
            launches = (0 if fused else 1) + (info.outer_iters + 1) + 2 * info.outer_iters + inner
            return {"outer": info.outer_iters, "inner": info.inner_iters, "device_relres": info.relres}, launches
        return run

    ELL, STENCIL = hp.SPMV_AUTO, hp.SPMV_STENCIL
    methods = [("fp64_cg", "plain FP64 CG (reference operation order), one CUDA graph", fp64_cg, ELL),
               ("fp32_ir", "FP64 iterative refinement, FP32 inner CG", mixed(hp.PREC_FP32), ELL),
               ("bf16_ir", "FP64 iterative refinement, inner CG on BF16 values / FP32 vectors", mixed(hp.PREC_BF16),
                ELL),
               ("fp64_cg_stencil", "plain FP64 CG with the matrix-free stencil SpMV (bit-identical to fp64_cg)",
                fp64_cg, STENCIL),
               ("fp32_ir_stencil", "FP64 iterative refinement (FP64 stencil residual), FP32 matrix-free inner CG "
                "(one fused TMA pass per iteration when nx % 4 == 0)", mixed(hp.PREC_FP32), STENCIL)]
    learned_info = None
    if not args.no_learned and cubic:
        from hpccg_b200 import learned

        t0 = time.time()
        net, hist = learned.train_preconditioner(64, seed=1, rhs=64, rounds=3, steps=args.train_steps)
        learned_info = {"train_s": time.time() - t0, "train_grid": "64^3", "train_rhs": 64, "rounds": 3,
                        "steps_per_round": args.train_steps, "loss_first": float(np.mean(hist[:5])),
                        "loss_last": float(np.mean(hist[-20:])), "params": net.nparams}

        def learned_fcg():
            info, st = learned.solve_fcg(M, net, n, d_b, d_x, REL_TOL, max_iter)
            assert st == hp.HPCCG_OK, st
            return ({"iterations": info.iters, "nn_applies": info.nn_applies, "fallback": info.fallback},
                    4 + 25 * info.iters)

        def learned_mixed():
            info, st = learned.solve_mixed_fcg(M, net, (n, n, nz), d_b, d_x, REL_TOL)
            assert st == hp.HPCCG_OK, st
            return ({"outer": info.outer_iters, "inner": info.inner_iters, "nn_applies": info.nn_applies,
                     "fallback": info.fallback}, 3 + 6 * info.inner_iters + 3 * info.outer_iters)

        methods.append(("learned_fcg", "flexible PCG (FP64, matrix-free stencil SpMV) with the trained U-Net "
                        "preconditioner (BF16 tensor cores)", learned_fcg, STENCIL))
        methods.append(("learned_mixed_fcg", "FP64 iterative refinement (FP64 stencil residual) around the "
                        "U-Net-preconditioned flexible CG in FP32 vectors (matrix-free FP32 operator)",
                        learned_mixed, STENCIL))
    results = {}
    clk_summary = None
    if args.methods:
        keep = set(args.methods.split(",")) | {"fp64_cg", "fp64_cg_stencil"}  # the speed-up baselines
        methods = [m for m in methods if m[0] in keep]
    for name, desc, fn, kind in methods:
        M.set_spmv(kind)
        for _ in range(args.warmup):
            d_x.zero_()
            fn()
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()
        times, launches = [], 0
        with ClockSampler(torch.cuda.current_device()) as clk:
            for _ in range(args.steps):
                d_x.zero_()
                info, nl = fn()
                times.append(M.last_solve_ms())
                launches += nl
        torch.cuda.synchronize()
        if ws > 1:
            dist.barrier()
        ms = max_over_ranks(float(np.median(times)), dev)
        relres = _fp64_relres(M, d_x, d_b, bnorm, scratch)
        err = float((d_x - xstar).abs().max().item())
        results[name] = {"ms": ms, "method": desc, "true_relres": relres, "max_abs_err_vs_xstar": err,
                         "gpu_launches": launches, "clocks": clk.summary(), "spmv_kernel": list(M.get_spmv()),
                         **info}
    if learned_info is not None:
        # the learned method on its own workload: Gaussian-random-field right-hand side
        grf = learned.gaussian_random_field(M, n, 4242, torch)
        M.set_spmv(STENCIL)
        d_x.zero_()
        it_plain, _, _, _ = M.cg_device(grf, d_x, max_iter, REL_TOL * float(torch.linalg.vector_norm(grf)),
                                        history=False)
        plain_grf_ms = M.last_solve_ms()
        d_x.zero_()
        info, _ = learned.solve_fcg(M, net, n, grf, d_x, REL_TOL, max_iter)
        learned_info.update({"grf_rhs": {"plain_fp64_cg_iters": it_plain, "plain_fp64_cg_ms": plain_grf_ms,
                                         "learned_fcg_iters": info.iters, "learned_fcg_ms": M.last_solve_ms(),
                                         "relres": info.relres, "fallback": info.fallback}})
        grf_mixed = {}
        for name, nn in (("plain_fp32_ir", None), ("learned_mixed_fcg", net)):
            d_x.zero_()
            mi, _ = learned.solve_mixed_fcg(M, nn, n, grf, d_x, REL_TOL)
            grf_mixed[name] = {"ms": M.last_solve_ms(), "outer": mi.outer_iters, "inner": mi.inner_iters,
                               "nn_applies": mi.nn_applies, "relres": mi.relres, "fallback": mi.fallback}
        d_x.zero_()
        mi, _ = M.solve_mixed_device(grf, d_x, hp.PREC_FP32, REL_TOL)
        grf_mixed["fp32_ir_stencil"] = {"ms": M.last_solve_ms(), "outer": mi.outer_iters,
                                        "inner": mi.inner_iters, "relres": mi.relres}
        learned_info["grf_rhs"]["mixed"] = grf_mixed
        d_in = torch.randn(N, dtype=torch.float32, device=dev)
        d_out = torch.empty_like(d_in)
        learned_info["unet_forward_ms"] = net.time_forward(d_in, d_out, n, n, n, 3)
    batch_info = batch_workload(hp, torch, args) if not args.no_batch else None
    ok = {k: v for k, v in results.items() if v["true_relres"] <= REL_TOL}
    head = min(ok, key=lambda k: ok[k]["ms"])
    plain_ms = results["fp64_cg"]["ms"]
    head_kind = STENCIL if head.endswith("_stencil") or head.startswith("learned") else ELL

    # end to end through the host-array C-ABI call of the headline solver, pinned host buffers
    h_b = torch.empty(N, dtype=torch.float64, pin_memory=True)
    h_b.copy_(d_b)
    h_x = torch.zeros(N, dtype=torch.float64, pin_memory=True)
    xb, bb = h_x.numpy(), h_b.numpy()
    e2e = []
    M.set_spmv(head_kind)
    for s in range(args.warmup + args.steps):
        xb[:] = 0.0
        t0 = time.perf_counter()
        if head.startswith("fp64_cg"):
            M.cg(bb, xb, max_iter, tol, history=False)
        elif head.startswith("learned"):
            h_bd = torch.from_numpy(bb).to(dev)
            d_xe = torch.zeros_like(h_bd)
            if head == "learned_fcg":
                learned.solve_fcg(M, net, n, h_bd, d_xe, REL_TOL, max_iter)
            else:
                learned.solve_mixed_fcg(M, net, n, h_bd, d_xe, REL_TOL)
            xb[:] = d_xe.cpu().numpy()
        else:
            M.solve_mixed(bb, xb, hp.PREC_BF16 if head == "bf16_ir" else hp.PREC_FP32, REL_TOL)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            e2e.append(dt)
    e2e_s = max_over_ranks(float(np.median(e2e)), dev)

    # rooflines (CUDA events on the library stream around back-to-back launches)
    hbm, _, peak_kind = _peaks()
    nnz = M.nnz
    M.set_spmv(ELL)
    kms64 = M.time_cg_kernels(reps=20)
    alg64 = 12 * nnz + 20 * N + 4
    roof64 = {"bound": "hbm", "kernel": "k_cg_spmv_dot (FP64 SpMV + p.Ap)", "kernel_ms": kms64[1],
              "alg_bytes_per_launch": alg64, "achieved": alg64 / (kms64[1] * 1e-3) / 1e9, "peak": hbm,
              "unit": "GB/s", "peak_source": peak_kind,
              "traffic": _traffic_from_profile() if n == 256 and cubic else None}
    roof64["frac"] = roof64["achieved"] / hbm
    roofs = {"fp64_cg": roof64}
    for name, prec, vb in (("fp32_ir", hp.PREC_FP32, 4), ("bf16_ir", hp.PREC_BF16, 2)):
        km = M.time_mixed_kernels(prec, 20)
        alg = (4 + vb) * nnz + 12 * N + 4
        roofs[name] = {"bound": "hbm", "kernel": f"k_mp_spmv_dot ({name[:4].upper()} values, FP32 vectors, + p.Ap)",
                       "kernel_ms": km[1], "alg_bytes_per_launch": alg, "achieved": alg / (km[1] * 1e-3) / 1e9,
                       "peak": hbm, "unit": "GB/s", "peak_source": peak_kind, "traffic": None,
                       "inner_iteration_ms": sum(km)}
        roofs[name]["frac"] = roofs[name]["achieved"] / hbm
    M.set_spmv(STENCIL)
    kst = M.time_cg_kernels(reps=20)
    alg = 16 * N + 4  # x read once, y written; A is not stored
    roofs["fp64_cg_stencil"] = {"bound": "hbm",
                                "kernel": "k_cg_spmv_dot<StratStencilTma> (matrix-free FP64 SpMV + p.Ap, "
                                          "reference term order, p by TMA)",
                                "kernel_ms": kst[1], "alg_bytes_per_launch": alg,
                                "achieved": alg / (kst[1] * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                                "peak_source": peak_kind,
                                "traffic": _traffic_from_profile("stencil_spmv_256.txt") if n == 256 and cubic else None,
                                "iteration_ms": sum(kst)}
    roofs["fp64_cg_stencil"]["frac"] = roofs["fp64_cg_stencil"]["achieved"] / hbm
    fused = M.mixed_fused()
    km = M.time_mixed_kernels(hp.PREC_FP32, 20)
    if fused:  # one pass reads r, p, d and writes r, p, d (FP32), plus four FP64 partials per CTA
        alg = 24 * N + 32
        kname = "k_mp_iter_tma (one fused FP32 matrix-free inner-CG pass, TMA-fed: r, p, d in and out)"
        traffic = _traffic_from_profile("inner_cg_pass_256.txt", "iter_dram_bytes_per_launch_full_size")
    else:
        alg = 8 * N + 4
        kname = ("k_mp_spmv_dot_tma (matrix-free FP32 SpMV, TMA-fed, + p.Ap)" if n % 4 == 0
                 else "k_mp_spmv_dot<StratLpStencil> (matrix-free FP32 SpMV + p.Ap)")
        traffic = _traffic_from_profile("stencil_spmv_256.txt", "fp32_tma_dram_bytes_per_launch_full_size")
    roofs["fp32_ir_stencil"] = {"bound": "hbm", "kernel": kname,
                                "kernel_ms": km[1], "alg_bytes_per_launch": alg,
                                "achieved": alg / (km[1] * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                                "peak_source": peak_kind, "traffic": traffic if n == 256 and cubic else None,
                                "inner_iteration_ms": km[1] if fused else sum(km)}
    roofs["fp32_ir_stencil"]["frac"] = roofs["fp32_ir_stencil"]["achieved"] / hbm
    if fused:  # the outer cycle's FP64 residual: x and b read (FP64), r written (FP32)
        alg = 20 * N + 32
        res = {"bound": "hbm", "kernel": "k_mp_residual_tma (FP64 r = b - A x, x and b by TMA, r stored FP32, "
                                         "+ r.r)",
               "kernel_ms": km[0], "alg_bytes_per_launch": alg, "achieved": alg / (km[0] * 1e-3) / 1e9,
               "peak": hbm, "unit": "GB/s", "peak_source": peak_kind,
               "traffic": _traffic_from_profile("refinement_residual_256.txt") if n == 256 and cubic else None}
        res["frac"] = res["achieved"] / hbm
        roofs["fp32_ir_stencil_residual"] = res
    if learned_info is not None:
        # the network's dominant work: the 3x3x3 convolutions on the tensor cores, against the
        # sustained BF16 peak (the forward pass runs inside a seconds-long solve)
        flop = unet_forward_flop(n, n, nz)
        fms = learned_info["unet_forward_ms"]
        _, bf16_sust, bf16_kind = _bf16_sustained()
        conv = {"bound": "tensor", "kernel": "U-Net forward pass (k_conv3_row tcgen05 convolutions, BF16 in, "
                "FP32 accumulate; the 1-channel input layer on tcgen05 too when nx % 128 == 0 "
                "(k_conv3_in1_tc), else on CUDA cores; pooling and upsampling)",
                "kernel_ms": fms, "flop_per_launch": flop, "achieved": flop / (fms * 1e-3) / 1e12,
                "peak": bf16_sust, "unit": "TFLOP/s", "peak_source": bf16_kind, "traffic": None}
        conv["frac"] = conv["achieved"] / bf16_sust
        roofs["learned_fcg"] = conv
        roofs["learned_mixed_fcg"] = conv

    if rank != 0:
        if ws > 1:
            dist.destroy_process_group()
        return 0

    cpu = None
    if not args.no_cpu_baseline and cubic:
        c = cpu_reference_time(n, 3, 1, args.ref_1thread_solves)
        cpu = {"value": c["value"], "unit": "s", "cores": c["cores"], "kind": "port",
               "value_1thread": c["value_1thread"], "iterations": c["iters"], "sample": _cpu_sample(c, n),
               **_host_cpu()}
    hr = results[head]
    line = {
        "metric": METRIC, "value": hr["ms"] / 1e3, "unit": "s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": hr["ms"], "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if head.startswith("fp64") or head == "learned_fcg"
        else "f32/bf16 inner, f64 outer",
        "data": "synthetic",
        "config": {"workload": f"{grid_name} 27-point HPCCG matrix ({N} rows, {nnz} nonzeros), x* U[-1,1) seed 1234, "
                               f"b = A x*, x0 = 0, solved to FP64 ||b - A x|| <= 1e-8 ||b||",
                   "method": head, "speedup_vs_plain_gpu_cg": plain_ms / hr["ms"],
                   "speedup_vs_plain_gpu_cg_stencil": results["fp64_cg_stencil"]["ms"] / hr["ms"],
                   "methods": results, "learned": learned_info, "batch": batch_info,
                   "l2": f"every pass streams more than the 126 MB L2 (the vectors alone: {N} rows x 8 B = "
                         f"{8 * N / 1e6:.0f} MB in FP64; the matrix-free inner pass moves 24 B a row, the stored "
                         f"matrix {(12 * nnz + 4 * (N + 1)) / 1e9:.1f} GB); no flush",
                   "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU",
                   "spmv_kernel": results[head]["spmv_kernel"]},
        "roofline": roofs[head], "roofline_all": roofs,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 16 * N, "d2h_bytes_per_step": 8 * N,
                "call": "hpccg_gpu_cg" if head.startswith("fp64_cg") else
                ("hpccg_gpu_solve_fcg" if head == "learned_fcg" else
                 "hpccg_gpu_solve_mixed_fcg" if head == "learned_mixed_fcg" else "hpccg_gpu_solve_mixed")},
        "gpu_launches": hr["gpu_launches"],
        "clocks": hr["clocks"],
    }
    print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()
    return 0


def _relaunch(nproc: int, argv: list[str]) -> int:
    """`--gpus N` without a launcher: start N ranks of this script under torch.distributed.run
    (one process per GPU, rendezvous on 127.0.0.1) and return their exit status."""
    import socket

    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    # torch.distributed.run's own parser would read a bare "--n" as an abbreviation of its options
    argv = ["--grid" if a == "--n" else ("--grid=" + a[4:] if a.startswith("--n=") else a) for a in argv]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *argv]
    return subprocess.run(cmd).returncode


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", "--grid", dest="n", type=int, default=256)
    ap.add_argument("--nz", type=int, default=0, help="planes of an n x n x nz grid (default n; profiling cases)")
    ap.add_argument("--ref-1thread-solves", type=int, default=1,
                    help="whole one-thread oracle solves for cpu_baseline.value_1thread (0: skip)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip training/timing the learned preconditioner")
    ap.add_argument("--train-steps", type=int, default=400)
    ap.add_argument("--methods", default="", help="comma-separated subset of solvers to time (default: all)")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-system batched-solve workload")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    ws_env = os.environ.get("WORLD_SIZE")
    if ws_env is None and args.gpus > 1:
        return _relaunch(args.gpus, sys.argv[1:] if argv is None else list(argv))
    if int(ws_env or 1) != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but the launcher started WORLD_SIZE={ws_env} ranks", file=sys.stderr)
        return 2
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
