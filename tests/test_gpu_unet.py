"""The U-Net kernels against the float64 numpy oracle (oracle/unet_oracle.py).

Bars: a conv layer on tcgen05 (BF16 operands, FP32 accumulation) matches the
oracle on the same BF16-rounded operands within 1e-3 relative to the output
scale (plus BF16 output rounding, 2^-8 relative); the CUDA-core conv matches
with FP32 weights; the full forward pass matches within 3e-2 of the output
scale (BF16 activations between layers); every layer's gradient block matches
the oracle's within 6e-2 relative (norm of the difference over norm).
"""
import numpy as np
import pytest

import unet_oracle as uo
import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch

    import hpccg_b200 as hp
    return torch, hp


def _bf16_tensor(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda().to(torch.bfloat16).contiguous()


def to_planar(x):
    """[b,z,y,x,16] channels-last -> the kernels' row-planar [b,z,y,half,x,8]."""
    b, z, y, nx, c = x.shape
    return np.ascontiguousarray(x.reshape(b, z, y, nx, 2, 8).transpose(0, 1, 2, 4, 3, 5))


def from_planar(p):
    b, z, y, _, nx, _ = p.shape
    return p.transpose(0, 1, 2, 4, 3, 5).reshape(b, z, y, nx, 16)


SHAPES = [(16, 16, 16, 1), (32, 8, 8, 2), (128, 4, 2, 1), (8, 8, 8, 3), (64, 16, 8, 1), (256, 3, 5, 2)]


@pytest.mark.parametrize("nx,ny,nz,nb", SHAPES)
@pytest.mark.parametrize("nin", [1, 2])
@pytest.mark.parametrize("epi", [0, 1, 2, 3])
def test_conv_layer_tc_and_cc(env, nx, ny, nz, nb, nin, epi):
    torch, hp = env
    rng = np.random.default_rng(nx * 131 + nin * 7 + epi)
    xs = [uo.bf16_round(rng.normal(0, 1, (nb, nz, ny, nx, 16))) for _ in range(nin)]
    W = rng.normal(0, 0.1, (27, 16 * nin, 16)).astype(np.float32)
    b = rng.normal(0, 0.1, 16).astype(np.float32)
    proj = rng.normal(0, 0.3, 17).astype(np.float32)
    x = np.concatenate(xs, -1).astype(np.float64)
    dW, db, dp = (torch.from_numpy(v).cuda() for v in (W, b, proj))
    din = [_bf16_tensor(torch, to_planar(v)) for v in xs] + [None]
    for path, Wref in ((0, uo.bf16_round(W)), (2, uo.bf16_round(W)), (1, W)):
        pre = uo.conv3(x, Wref.astype(np.float64))
        if epi == 3:
            want = pre
            out = torch.empty((nb, nz, ny, 2, nx, 8), dtype=torch.float32, device="cuda")
        elif epi == 2:
            want = np.maximum(pre + b, 0) @ proj[:16].astype(np.float64) + proj[16]
            out = torch.empty((nb, nz, ny, nx), dtype=torch.float32, device="cuda")
        else:
            want = pre + b
            if epi == 0:
                want = np.maximum(want, 0)
            out = torch.empty((nb, nz, ny, 2, nx, 8), dtype=torch.bfloat16, device="cuda")
        hp.conv3_layer(din[0], din[1], dW, db, dp, epi, path, out, nx, ny, nz, nb)
        got = out.float().cpu().numpy().astype(np.float64)
        if epi != 2:
            got = from_planar(got)
        scale = np.abs(want).max() + 1e-30
        tol = 1e-3 * scale + (2.0 ** -8 * np.abs(want) if epi in (0, 1) else 0)
        assert np.all(np.abs(got - want) <= tol), (path, np.abs(got - want).max(), scale)


@pytest.mark.parametrize("nx,ny,nz,nb", [(128, 4, 2, 1), (256, 3, 5, 2), (128, 1, 1, 1), (64, 4, 4, 1)])
@pytest.mark.parametrize("epi", [0, 1])
def test_input_layer_tc_and_cc(env, nx, ny, nz, nb, epi):
    """The 1-channel input layer: tcgen05 (BF16 input and weights rounded as the kernel rounds them,
    FP32 accumulation; 128-voxel rows) and CUDA cores (FP32) against the oracle conv, within the
    bars of the 16-channel layers; grids whose nx is not a multiple of 128 have no tensor-core path."""
    torch, hp = env
    rng = np.random.default_rng(nx * 7 + ny + epi)
    x = rng.normal(0, 1, (nb, nz, ny, nx)).astype(np.float32)
    W = rng.normal(0, 0.2, (27, 1, 16)).astype(np.float32)
    b = rng.normal(0, 0.1, 16).astype(np.float32)
    dW, db = torch.from_numpy(W).cuda(), torch.from_numpy(b).cuda()
    din = torch.from_numpy(x).cuda()
    for path in (0, 1):
        xr, Wr = (uo.bf16_round(x), uo.bf16_round(W)) if path == 0 else (x, W)
        want = uo.conv3(xr[..., None].astype(np.float64), Wr.astype(np.float64)) + b
        if epi == 0:
            want = np.maximum(want, 0)
        out = torch.empty((nb, nz, ny, 2, nx, 8), dtype=torch.bfloat16, device="cuda")
        if path == 0 and nx % 128:
            with pytest.raises(hp.HpccgError) as e:
                hp.conv3_layer(din, None, dW, db, None, epi, path, out, nx, ny, nz, nb, nin=0)
            assert e.value.code == hp.HPCCG_ERR_UNSUPPORTED
            continue
        hp.conv3_layer(din, None, dW, db, None, epi, path, out, nx, ny, nz, nb, nin=0)
        got = from_planar(out.float().cpu().numpy().astype(np.float64))
        scale = np.abs(want).max() + 1e-30
        tol = 1e-3 * scale + 2.0 ** -8 * np.abs(want)
        assert np.all(np.abs(got - want) <= tol), (path, np.abs(got - want).max(), scale)


def _net_and_params(hp, seed=3):
    net = hp.Unet(seed)
    p = net.get_params().astype(np.float64)
    # non-trivial biases so every ReLU sees both signs
    rng = np.random.default_rng(seed)
    p = p + rng.normal(0, 0.02, p.size)
    net.set_params(p.astype(np.float32))
    return net, net.get_params().astype(np.float64)


def test_forward_matches_oracle(env):
    torch, hp = env
    net, p = _net_and_params(hp)
    assert net.nparams == 104337
    rng = np.random.default_rng(5)
    r = rng.normal(0, 1, (2, 16, 16, 16))
    want = uo.forward(p, r)
    din = torch.from_numpy(r.astype(np.float32)).cuda()
    dout = torch.empty_like(din)
    net.forward(din, dout, 16, 16, 16, 2)
    got = dout.cpu().numpy()
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= 3e-2 * scale, (np.abs(got - want).max(), scale)


def test_gradients_match_oracle(env):
    torch, hp = env
    net, p = _net_and_params(hp, seed=9)
    rng = np.random.default_rng(6)
    r = rng.normal(0, 1, (1, 16, 16, 16))
    t = rng.normal(0, 0.05, (1, 16, 16, 16))
    loss_ref, g_ref = uo.loss_grad(p, r, t)
    din = torch.from_numpy(r.astype(np.float32)).cuda()
    dt = torch.from_numpy(t.astype(np.float32)).cuda()
    loss, g = net.loss_grad(din, dt, 16, 16, 16, 1, want_grad=True)
    assert loss == pytest.approx(loss_ref, rel=5e-2)
    off, n = uo.offsets()
    for l in range(14):
        a, b = off[l], (off[l + 1] if l < 13 else n)
        ref = g_ref[a:b]
        err = np.linalg.norm(g[a:b] - ref) / (np.linalg.norm(ref) + 1e-30)
        assert err <= 6e-2, (l, err)


def test_trained_network_reduces_fcg_iterations(env):
    """What the trained network gains: FCG iterations to FP64 rel-res 1e-8 on
    held-out Gaussian-random-field right-hand sides, against plain CG through
    the same solver (net = None).  Trained on 64^3 grids as the bench does."""
    torch, hp = env
    from hpccg_b200 import learned

    net, hist = learned.train_preconditioner(64, seed=2, rhs=48, rounds=3, steps=300, batch=4)
    assert np.mean(hist[-20:]) < 0.5 * np.mean(hist[:5])
    for n in (64, 96):
        M = hp.Matrix.generated(n, n, n)
        for sd in (77, 78):
            b = learned.gaussian_random_field(M, n, sd, torch)
            x = torch.zeros_like(b)
            plain, st0 = learned.solve_fcg(M, None, n, b, x)
            x.zero_()
            fcg, st1 = learned.solve_fcg(M, net, n, b, x)
            assert st0 == hp.HPCCG_OK and st1 == hp.HPCCG_OK
            assert fcg.relres <= 1e-8 and plain.relres <= 1e-8
            assert fcg.iters <= 0.6 * plain.iters, (n, sd, fcg.iters, plain.iters)
            # the same network inside mixed precision: FP32 flexible CG in FP64 refinement,
            # against plain FP32 CG through the same solver; the oracle checks the result
            bh = b.cpu().numpy()
            runs = {}
            for name, nn in (("plain", None), ("learned", net)):
                x.zero_()
                info, st = learned.solve_mixed_fcg(M, nn, n, b, x)
                assert st == hp.HPCCG_OK, name
                rel = oracle.grid_true_relres(n, n, n, bh, x.cpu().numpy())
                assert rel <= 1e-8 * (1 + 1e-6), (name, rel)
                assert info.relres == pytest.approx(rel, rel=1e-6)
                runs[name] = info
            assert runs["learned"].nn_applies > 0
            assert runs["learned"].inner_iters <= 0.6 * runs["plain"].inner_iters, (
                n, sd, runs["learned"].inner_iters, runs["plain"].inner_iters)
