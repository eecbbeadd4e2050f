"""CPU oracle for the learned preconditioner (TEST INFRASTRUCTURE ONLY).

A float64 numpy restatement of the project's U-Net (the reference has no
learned part): 3x3x3 zero-padded convolutions on channels-last tensors
[batch][z][y][x][c], 2x2x2 average pooling, nearest 2x upsampling, ReLU, the
16->1 projection, the mean-squared-error loss and the full backward pass.
The parameter vector layout matches hpccg_unet_get_params: per layer
W[27][cin][16] then bias[16]; then projection weights[16] and bias[1].
Tap t = (dz+1)*9 + (dy+1)*3 + (dx+1) reads the input at (z+dz, y+dy, x+dx).
"""
from __future__ import annotations

import numpy as np

# (cin, level) per layer, in parameter order; layers 8, 10, 12 read two 16-channel inputs.
LAYERS = [(1, 0), (16, 0), (16, 1), (16, 1), (16, 2), (16, 2), (16, 3), (16, 3), (32, 2), (16, 2), (32, 1),
          (16, 1), (32, 0)]


def offsets():
    off, o = [], 0
    for cin, _ in LAYERS:
        off.append(o)
        o += 27 * cin * 16 + 16
    off.append(o)
    return off, o + 17


def unpack(params):
    off, n = offsets()
    assert len(params) == n
    Ws, bs = [], []
    for l, (cin, _) in enumerate(LAYERS):
        w = params[off[l]:off[l] + 27 * cin * 16].reshape(27, cin, 16)
        Ws.append(w.astype(np.float64))
        bs.append(params[off[l] + 27 * cin * 16: off[l + 1]].astype(np.float64))
    proj = params[off[-1]:off[-1] + 17].astype(np.float64)
    return Ws, bs, proj


def _pad(x):
    return np.pad(x, ((0, 0), (1, 1), (1, 1), (1, 1), (0, 0)))


def conv3(x, W, b=None):
    """x [B,Z,Y,X,cin], W [27,cin,cout] -> [B,Z,Y,X,cout] (zero padding)."""
    B, Z, Y, X, _ = x.shape
    xp = _pad(x)
    out = np.zeros((B, Z, Y, X, W.shape[2]))
    for t in range(27):
        dz, dy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
        sl = xp[:, 1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X, :]
        out += sl @ W[t]
    if b is not None:
        out += b
    return out


def conv3_grads(x, W, dy):
    """Gradients of conv3 w.r.t. x, W and bias, given dL/d(out) = dy."""
    B, Z, Y, X, _ = x.shape
    xp = _pad(x)
    dxp = np.zeros_like(xp)
    dW = np.zeros_like(W)
    for t in range(27):
        dz, dyy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
        sl = (slice(None), slice(1 + dz, 1 + dz + Z), slice(1 + dyy, 1 + dyy + Y), slice(1 + dx, 1 + dx + X))
        dW[t] = np.einsum("bzyxc,bzyxo->co", xp[sl], dy)
        dxp[sl] += dy @ W[t].T
    return dxp[:, 1:-1, 1:-1, 1:-1, :], dW, dy.sum(axis=(0, 1, 2, 3))


def pool(x):
    B, Z, Y, X, C = x.shape
    return x.reshape(B, Z // 2, 2, Y // 2, 2, X // 2, 2, C).mean(axis=(2, 4, 6))


def pool_bwd(d):
    return np.repeat(np.repeat(np.repeat(d, 2, axis=1), 2, axis=2), 2, axis=3) / 8.0


def up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, axis=1), 2, axis=2), 2, axis=3)


def up_bwd(d):
    B, Z, Y, X, C = d.shape
    return d.reshape(B, Z // 2, 2, Y // 2, 2, X // 2, 2, C).sum(axis=(2, 4, 6))


def relu(x):
    return np.maximum(x, 0.0)


def forward(params, r, keep=False):
    """r [B,Z,Y,X] -> out [B,Z,Y,X]; keep=True also returns the activations."""
    Ws, bs, proj = unpack(params)
    a = {}
    x = r[..., None].astype(np.float64)
    a["in"] = x
    a["e1a"] = relu(conv3(x, Ws[0], bs[0]))
    a["e1b"] = relu(conv3(a["e1a"], Ws[1], bs[1]))
    a["d1"] = pool(a["e1b"])
    a["e2a"] = relu(conv3(a["d1"], Ws[2], bs[2]))
    a["e2b"] = relu(conv3(a["e2a"], Ws[3], bs[3]))
    a["d2"] = pool(a["e2b"])
    a["e3a"] = relu(conv3(a["d2"], Ws[4], bs[4]))
    a["e3b"] = relu(conv3(a["e3a"], Ws[5], bs[5]))
    a["d3"] = pool(a["e3b"])
    a["e4a"] = relu(conv3(a["d3"], Ws[6], bs[6]))
    a["e4b"] = relu(conv3(a["e4a"], Ws[7], bs[7]))
    a["u3"] = up(a["e4b"])
    a["c3a"] = relu(conv3(np.concatenate([a["e3b"], a["u3"]], -1), Ws[8], bs[8]))
    a["c3b"] = relu(conv3(a["c3a"], Ws[9], bs[9]))
    a["u2"] = up(a["c3b"])
    a["c2a"] = relu(conv3(np.concatenate([a["e2b"], a["u2"]], -1), Ws[10], bs[10]))
    a["c2b"] = relu(conv3(a["c2a"], Ws[11], bs[11]))
    a["u1"] = up(a["c2b"])
    a["c1"] = relu(conv3(np.concatenate([a["e1b"], a["u1"]], -1), Ws[12], bs[12]))
    out = a["c1"] @ proj[:16] + proj[16]
    return (out, a) if keep else out


def apply_A(d):
    """The generate_matrix operator on each grid of d [B,Z,Y,X]: 27 d - sum of in-grid neighbours."""
    dp = np.pad(d, ((0, 0), (1, 1), (1, 1), (1, 1)))
    Z, Y, X = d.shape[1:]
    s = np.zeros_like(d)
    for t in range(27):
        dz, dy, dx = t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1
        s += dp[:, 1 + dz:1 + dz + Z, 1 + dy:1 + dy + Y, 1 + dx:1 + dx + X]
    return 28.0 * d - s


def loss_grad(params, r, target, kind=0):
    """Loss (0: mean squared error, 1: energy norm d.(A d)/n) and its gradient."""
    off, n = offsets()
    Ws, bs, proj = unpack(params)
    out, a = forward(params, r, keep=True)
    N = out.size
    if kind == 1:
        Ad = apply_A(target - out)
        loss = float(((target - out) * Ad).sum() / N)
        dout = -2.0 * Ad / N
    else:
        loss = float(((out - target) ** 2).mean())
        dout = 2.0 * (out - target) / N
    g = np.zeros(n)
    g[off[-1]:off[-1] + 16] = np.einsum("bzyxc,bzyx->c", a["c1"], dout)
    g[off[-1] + 16] = dout.sum()

    def put(l, dW, db):
        cin = LAYERS[l][0]
        g[off[l]:off[l] + 27 * cin * 16] = dW.reshape(-1)
        g[off[l] + 27 * cin * 16:off[l + 1]] = db

    d = (dout[..., None] * proj[:16]) * (a["c1"] > 0)
    dx, dW, db = conv3_grads(np.concatenate([a["e1b"], a["u1"]], -1), Ws[12], d)
    put(12, dW, db)
    g_e1b, g_u1 = dx[..., :16], dx[..., 16:]
    d = up_bwd(g_u1) * (a["c2b"] > 0)
    dx, dW, db = conv3_grads(a["c2a"], Ws[11], d)
    put(11, dW, db)
    d = dx * (a["c2a"] > 0)
    dx, dW, db = conv3_grads(np.concatenate([a["e2b"], a["u2"]], -1), Ws[10], d)
    put(10, dW, db)
    g_e2b, g_u2 = dx[..., :16], dx[..., 16:]
    d = up_bwd(g_u2) * (a["c3b"] > 0)
    dx, dW, db = conv3_grads(a["c3a"], Ws[9], d)
    put(9, dW, db)
    d = dx * (a["c3a"] > 0)
    dx, dW, db = conv3_grads(np.concatenate([a["e3b"], a["u3"]], -1), Ws[8], d)
    put(8, dW, db)
    g_e3b, g_u3 = dx[..., :16], dx[..., 16:]
    d = up_bwd(g_u3) * (a["e4b"] > 0)
    dx, dW, db = conv3_grads(a["e4a"], Ws[7], d)
    put(7, dW, db)
    d = dx * (a["e4a"] > 0)
    dx, dW, db = conv3_grads(a["d3"], Ws[6], d)
    put(6, dW, db)
    d = (g_e3b + pool_bwd(dx)) * (a["e3b"] > 0)
    dx, dW, db = conv3_grads(a["e3a"], Ws[5], d)
    put(5, dW, db)
    d = dx * (a["e3a"] > 0)
    dx, dW, db = conv3_grads(a["d2"], Ws[4], d)
    put(4, dW, db)
    d = (g_e2b + pool_bwd(dx)) * (a["e2b"] > 0)
    dx, dW, db = conv3_grads(a["e2a"], Ws[3], d)
    put(3, dW, db)
    d = dx * (a["e2a"] > 0)
    dx, dW, db = conv3_grads(a["d1"], Ws[2], d)
    put(2, dW, db)
    d = (g_e1b + pool_bwd(dx)) * (a["e1b"] > 0)
    dx, dW, db = conv3_grads(a["e1a"], Ws[1], d)
    put(1, dW, db)
    d = dx * (a["e1a"] > 0)
    _, dW, db = conv3_grads(a["in"], Ws[0], d)
    put(0, dW, db)
    return loss, g


def bf16_round(x):
    """Round float values to the nearest BF16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)
