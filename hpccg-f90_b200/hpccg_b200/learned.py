"""Learned preconditioner pipeline: data from the GPU CG, training, solving.

Every numerical step runs in the library's own kernels through the C-ABI:
the FP64 CG that generates residual->error pairs (hpccg_gpu_cg_device), the
U-Net forward/backward/Adam (hpccg_unet_*), and the flexible PCG in FP64
(hpccg_gpu_solve_fcg) or in FP32 inside FP64 refinement
(hpccg_gpu_solve_mixed_fcg).  torch provides device memory and, for the synthetic
right-hand sides only, the FFT that shapes white noise into a Gaussian random
field.
"""
from __future__ import annotations

import ctypes
import math
import time

import numpy as np

from . import (HPCCG_ERR_NOT_CONVERGED, HPCCG_OK, Matrix, Unet, _check, _dptr, _lib, _sync_torch)


class FcgInfo(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int32), ("nn_applies", ctypes.c_int32), ("fallback", ctypes.c_int32),
                ("status", ctypes.c_int32), ("relres", ctypes.c_double)]


_lib.hpccg_gpu_solve_fcg.restype = ctypes.c_int
_lib.hpccg_gpu_solve_fcg.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_int32,
                                     ctypes.c_void_p]


class MixedFcgInfo(ctypes.Structure):
    _fields_ = [("outer_iters", ctypes.c_int32), ("inner_iters", ctypes.c_int32), ("nn_applies", ctypes.c_int32),
                ("fallback", ctypes.c_int32), ("status", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("relres", ctypes.c_double)]


_lib.hpccg_gpu_solve_mixed_fcg.restype = ctypes.c_int
_lib.hpccg_gpu_solve_mixed_fcg.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                           ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                           ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p]


def gaussian_random_field(M: Matrix, n: int, seed: int, torch):
    """RHS with power spectrum |k|^-2 on an n^3 grid (k = 0 removed), unit RMS, FP64.

    White noise comes from the project's counter-based generator (Box-Muller on
    two uniform streams); the spectral shaping uses an FFT."""
    N = n ** 3
    u1 = torch.empty(N, dtype=torch.float64, device="cuda")
    u2 = torch.empty_like(u1)
    M.uniform_pm1(seed, u1)
    M.uniform_pm1(seed ^ 0x5DEECE66D, u2)
    a = (u1 + 1.0) * 0.5  # [0, 1)
    rad = torch.sqrt(-2.0 * torch.log1p(-a))  # Box-Muller radius, finite for a in [0, 1)
    w = (rad * torch.cos(math.pi * (u2 + 1.0))).reshape(n, n, n)
    W = torch.fft.rfftn(w)
    k = torch.fft.fftfreq(n, device="cuda", dtype=torch.float64) * n
    kr = torch.fft.rfftfreq(n, device="cuda", dtype=torch.float64) * n
    kk = torch.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + kr[None, None, :] ** 2)
    amp = torch.where(kk > 0, 1.0 / torch.clamp(kk, min=1e-12), torch.zeros_like(kk))
    f = torch.fft.irfftn(W * amp, s=(n, n, n)).reshape(-1).contiguous()
    return f / torch.sqrt((f * f).mean())


def make_pairs(M: Matrix, n: int, seeds, ks, torch):
    """Residual->error pairs from the GPU CG: for each GRF right-hand side b and
    each k in ks, x_k = k CG iterations from 0, r_k = b - A x_k, e_k = x - x_k
    with x from CG to ||r|| < 1e-12 ||b||.  Pairs are scaled by 1/rms(r_k).
    Returns FP32 tensors (inputs, targets) of shape [len(seeds)*len(ks), n^3]."""
    N = n ** 3
    ins, tgts = [], []
    x = torch.zeros(N, dtype=torch.float64, device="cuda")
    xk = torch.zeros_like(x)
    r = torch.empty_like(x)
    for sd in seeds:
        b = gaussian_random_field(M, n, sd, torch)
        bn = float(torch.linalg.vector_norm(b))
        x.zero_()
        M.cg_device(b, x, 2000, 1e-12 * bn, history=False)
        for k in ks:
            xk.zero_()
            if k > 0:
                M.cg_device(b, xk, k, 0.0, history=False)
            M.spmv(xk, r)
            M.waxpby(1.0, b, -1.0, r, r)
            s = float(torch.sqrt((r * r).mean()))
            if not s > 0:
                continue
            ins.append((r / s).float())
            tgts.append(((x - xk) / s).float())
    return torch.stack(ins), torch.stack(tgts)


def fcg_pairs(M: Matrix, net: Unet, n: int, seeds, ks, torch):
    """Residual->error pairs from the flexible PCG with the current network: the
    residuals the preconditioner meets when it is used (x_k = k FCG iterations
    from 0), so later training rounds cover them."""
    N = n ** 3
    ins, tgts = [], []
    x = torch.zeros(N, dtype=torch.float64, device="cuda")
    xk = torch.zeros_like(x)
    r = torch.empty_like(x)
    for sd in seeds:
        b = gaussian_random_field(M, n, sd, torch)
        bn = float(torch.linalg.vector_norm(b))
        x.zero_()
        M.cg_device(b, x, 2000, 1e-12 * bn, history=False)
        for k in ks:
            xk.zero_()
            solve_fcg(M, net, n, b, xk, rel_tol=1e-14, max_iter=k)
            M.spmv(xk, r)
            M.waxpby(1.0, b, -1.0, r, r)
            s = float(torch.sqrt((r * r).mean()))
            if not s > 0:
                continue
            ins.append((r / s).float())
            tgts.append(((x - xk) / s).float())
    return torch.stack(ins), torch.stack(tgts)


def train_preconditioner(n: int = 64, seed: int = 1, rhs: int = 64, rounds: int = 3, steps: int = 400,
                         batch: int = 4, lr: float = 2e-3, log=None):
    """Train the U-Net as an FCG preconditioner on n^3 grids.

    Training round 0 learns from plain-CG residual->error pairs of `rhs` Gaussian random
    field right-hand sides; each further round adds pairs from FCG runs with
    the current network.  Loss: energy norm of the HPCCG operator."""
    import torch

    M = Matrix.generated(n, n, n)
    net = Unet(seed)
    net.set_loss(1)
    seeds = list(range(1000 * seed, 1000 * seed + rhs))
    ins, tgts = make_pairs(M, n, seeds, [0, 1, 2, 3, 5, 8, 12, 20, 30], torch)
    hist = []
    for rnd in range(rounds):
        hist += train(net, ins, tgts, n, steps, batch=batch, lr=lr * (0.7 ** rnd), seed=rnd, log=log)
        if rnd + 1 < rounds:
            sub = seeds[rnd::rounds][: max(8, rhs // rounds)]
            fi, ft = fcg_pairs(M, net, n, sub, [2, 4, 6, 9, 12, 16, 22, 30], torch)
            ins, tgts = torch.cat([ins, fi]), torch.cat([tgts, ft])
            if log:
                log(f"round {rnd}: {fi.shape[0]} FCG pairs added, {ins.shape[0]} total")
    return net, hist


def train(net: Unet, inputs, targets, n: int, steps: int, batch: int = 4, lr: float = 2e-3, seed: int = 0,
          time_budget_s: float | None = None, log=None):
    """Adam on the mean squared error of net(r_k) against e_k, cosine learning-rate decay."""
    import torch

    g = torch.Generator(device="cpu").manual_seed(seed)
    npairs = inputs.shape[0]
    losses = []
    t0 = time.time()
    for step in range(steps):
        idx = torch.randint(0, npairs, (batch,), generator=g)
        xb = inputs[idx.cuda()].contiguous()
        yb = targets[idx.cuda()].contiguous()
        loss = net.loss_grad(xb, yb, n, n, n, batch)
        cur = lr * 0.5 * (1 + math.cos(math.pi * step / max(1, steps)))
        net.adam_step(max(cur, lr * 0.02))
        losses.append(loss)
        if log and (step % 50 == 0 or step == steps - 1):
            log(f"step {step} loss {loss:.4e} lr {cur:.2e} t {time.time() - t0:.1f}s")
        if time_budget_s is not None and time.time() - t0 > time_budget_s:
            break
    return losses


def solve_fcg(M: Matrix, net: Unet | None, n: int, d_b, d_x, rel_tol: float = 1e-8, max_iter: int = 2000):
    """Flexible PCG with the network (net=None: plain CG through the same code).
    Returns (FcgInfo, status)."""
    _sync_torch()
    info = FcgInfo()
    rc = _lib.hpccg_gpu_solve_fcg(M.handle, None if net is None else net.handle, n, n, n, _dptr(d_b), _dptr(d_x),
                                  rel_tol, max_iter, ctypes.byref(info))
    _check(rc, "solve_fcg", allow=(HPCCG_OK, HPCCG_ERR_NOT_CONVERGED))
    return info, rc


def solve_mixed_fcg(M: Matrix, net: Unet | None, n, d_b, d_x, rel_tol: float = 1e-8, max_outer: int = 20,
                    max_inner: int = 1000):
    """FP64 iterative refinement around the network-preconditioned flexible CG in FP32
    (hpccg_gpu_solve_mixed_fcg; net=None: plain FP32 CG).  n: the grid edge or (nx, ny, nz).
    Returns (MixedFcgInfo, status)."""
    nx, ny, nz = (n, n, n) if isinstance(n, int) else n
    _sync_torch()
    info = MixedFcgInfo()
    rc = _lib.hpccg_gpu_solve_mixed_fcg(M.handle, None if net is None else net.handle, nx, ny, nz, _dptr(d_b),
                                        _dptr(d_x), rel_tol, max_outer, max_inner, ctypes.byref(info))
    _check(rc, "solve_mixed_fcg", allow=(HPCCG_OK, HPCCG_ERR_NOT_CONVERGED))
    return info, rc


def _main(argv=None):
    """Command line: time the U-Net forward pass (random weights) on an n^3 grid,
    or train the preconditioner and report its FCG iteration gain.

        python -m hpccg_b200.learned forward --n 128 --reps 5
        python -m hpccg_b200.learned train --n 64 --steps 400
    """
    import argparse
    import json

    import torch

    ap = argparse.ArgumentParser(prog="python -m hpccg_b200.learned")
    ap.add_argument("cmd", choices=["forward", "train"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--seed", type=int, default=1)
    a = ap.parse_args(argv)
    if a.cmd == "forward":
        net = Unet(a.seed)
        d_in = torch.randn(a.n ** 3, dtype=torch.float32, device="cuda")
        d_out = torch.empty_like(d_in)
        net.forward(d_in, d_out, a.n, a.n, a.n)  # first call sizes the workspace
        ms = net.time_forward(d_in, d_out, a.n, a.n, a.n, a.reps)
        print(json.dumps({"unet_forward_ms": ms, "n": a.n, "params": net.nparams}))
        return 0
    net, hist = train_preconditioner(a.n, seed=a.seed, steps=a.steps)
    M = Matrix.generated(a.n, a.n, a.n)
    b = gaussian_random_field(M, a.n, 4242, torch)
    x = torch.zeros_like(b)
    plain, _ = solve_fcg(M, None, a.n, b, x)
    x.zero_()
    lrn, _ = solve_fcg(M, net, a.n, b, x)
    print(json.dumps({"loss_first": float(np.mean(hist[:5])), "loss_last": float(np.mean(hist[-20:])),
                      "plain_iters": plain.iters, "learned_iters": lrn.iters, "relres": lrn.relres}))
    return 0


if __name__ == "__main__":
    import sys

    sys.exit(_main())
