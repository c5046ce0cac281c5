"""FP64 numpy restatement of the warm-start network's operations and of the whole network's
forward and backward pass (macroflow3d_b200/csrc/nn.cuh, kernels_nn.cuh).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the CUDA kernels' values and
gradients on tiny shapes.  The product (macroflow3d_b200) never imports this module.  The
network has no counterpart in the reference (its initial guess is the x-linear head,
src/physics/flow/solve_head.cu:29-73); parity here is against this restatement of the
mathematics, checked on its own by adjoint identities and finite differences.

Arrays are numpy float64 of shape (nz, ny, nx, C) (channels innermost, as on the device);
weights are (cout, 27, cin) with tap t = (dz+1)*9 + (dy+1)*3 + (dx+1).
"""
from __future__ import annotations

import numpy as np

TAPS = [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]  # (dz, dy, dx)

LAYERS = [(16, 16, 1), (16, 16, 1), (16, 32, 1), (32, 32, 1), (32, 64, 1), (64, 64, 1),
          (64, 64, 1), (64, 64, 1), (128, 64, 1), (96, 32, 1), (48, 16, 1), (16, 16, 0)]
TARGET_SCALE = 0.1


def _shift(x, dz, dy, dx):
    """s[z, y, x] = x[z + dz, y + dy, x + dx] with zeros outside."""
    nz, ny, nx = x.shape[:3]
    out = np.zeros_like(x)
    zs, ys, xs = slice(max(0, -dz), min(nz, nz - dz)), slice(max(0, -dy), min(ny, ny - dy)), \
        slice(max(0, -dx), min(nx, nx - dx))
    zt, yt, xt = slice(max(0, dz), min(nz, nz + dz)), slice(max(0, dy), min(ny, ny + dy)), \
        slice(max(0, dx), min(nx, nx + dx))
    out[zs, ys, xs] = x[zt, yt, xt]
    return out


def conv3d(x, w, b=None):
    """y[v, co] = sum_t sum_ci x[v + off(t), ci] w[co, t, ci] (+ b[co])."""
    y = np.zeros(x.shape[:3] + (w.shape[0],))
    for t, (dz, dy, dx) in enumerate(TAPS):
        y += _shift(x, dz, dy, dx) @ w[:, t, :].T
    if b is not None:
        y += b
    return y


def conv3d_dgrad(g, w):
    """Adjoint of conv3d in x: dx[v, ci] = sum_t sum_co g[v - off(t), co] w[co, t, ci]."""
    dx = np.zeros(g.shape[:3] + (w.shape[2],))
    for t, (dz, dy, dxo) in enumerate(TAPS):
        dx += _shift(g, -dz, -dy, -dxo) @ w[:, t, :]
    return dx


def conv3d_wgrad(x, g):
    """dw[co, t, ci] = sum_v g[v, co] x[v + off(t), ci]; db[co] = sum_v g[v, co]."""
    cin, cout = x.shape[3], g.shape[3]
    dw = np.zeros((cout, 27, cin))
    G = g.reshape(-1, cout)
    for t, (dz, dy, dx) in enumerate(TAPS):
        dw[:, t, :] = G.T @ _shift(x, dz, dy, dx).reshape(-1, cin)
    return dw, G.sum(axis=0)


def flip_weights(w):
    """W'[ci, t, co] = W[co, 26 - t, ci]: conv3d(g, W') == conv3d_dgrad(g, W)."""
    return np.ascontiguousarray(w[:, ::-1, :].transpose(2, 1, 0))


def pool(x):
    nz, ny, nx, c = x.shape
    return x.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2, c).mean(axis=(1, 3, 5))


def pool_bwd(g):
    return np.repeat(np.repeat(np.repeat(g, 2, 0), 2, 1), 2, 2) / 8.0


def up(x):
    return np.repeat(np.repeat(np.repeat(x, 2, 0), 2, 1), 2, 2)


def up_bwd(g):
    nz, ny, nx, c = g.shape
    return g.reshape(nz // 2, 2, ny // 2, 2, nx // 2, 2, c).sum(axis=(1, 3, 5))


def net_input(lnK, hw=1.0, he=0.0):
    nz, ny, nx = lnK.shape
    x = np.zeros((nz, ny, nx, 16))
    hl = hw + (he - hw) * (np.arange(nx) + 0.5) / nx
    x[..., 0] = 0.5 * lnK
    x[..., 1] = (hl - 0.5 * (hw + he))[None, None, :]
    return x, np.broadcast_to(hl, lnK.shape)


def split_params(p):
    """Flat parameter vector (the device order: per layer W then b) -> [(W, b)]."""
    out, o = [], 0
    for cin, cout, _ in LAYERS:
        n = cout * 27 * cin
        out.append((p[o:o + n].reshape(cout, 27, cin), p[o + n:o + n + cout]))
        o += n + cout
    assert o == p.size
    return out


def forward(params, lnK, hw=1.0, he=0.0):
    """Returns (out, cache); out[..., 0] predicts (h - h_lin) / TARGET_SCALE."""
    P = split_params(params)
    relu = lambda z: np.maximum(z, 0.0)
    x, hl = net_input(lnK, hw, he)
    c = {"in": x}
    c["a0"] = relu(conv3d(x, *P[0]))
    c["e0"] = relu(conv3d(c["a0"], *P[1]))
    c["p0"] = pool(c["e0"])
    c["a2"] = relu(conv3d(c["p0"], *P[2]))
    c["e1"] = relu(conv3d(c["a2"], *P[3]))
    c["p1"] = pool(c["e1"])
    c["a4"] = relu(conv3d(c["p1"], *P[4]))
    c["e2"] = relu(conv3d(c["a4"], *P[5]))
    c["p2"] = pool(c["e2"])
    c["a6"] = relu(conv3d(c["p2"], *P[6]))
    c["e3"] = relu(conv3d(c["a6"], *P[7]))
    c["c2"] = np.concatenate([up(c["e3"]), c["e2"]], axis=3)
    c["d2"] = relu(conv3d(c["c2"], *P[8]))
    c["c1"] = np.concatenate([up(c["d2"]), c["e1"]], axis=3)
    c["d1"] = relu(conv3d(c["c1"], *P[9]))
    c["c0"] = np.concatenate([up(c["d1"]), c["e0"]], axis=3)
    c["d0"] = relu(conv3d(c["c0"], *P[10]))
    out = conv3d(c["d0"], *P[11])
    c["hl"] = hl
    return out, c


def loss_and_grad(params, lnK, h, hw=1.0, he=0.0):
    """Mean squared error of out[..., 0] against (h - h_lin) / TARGET_SCALE, and its gradient
    in the flat parameter order."""
    P = split_params(params)
    out, c = forward(params, lnK, hw, he)
    V = lnK.size
    d = out[..., 0] - (h - c["hl"]) / TARGET_SCALE
    loss = float((d * d).mean())
    gout = np.zeros_like(out)
    gout[..., 0] = 2.0 * d / V
    mask = lambda g, a: g * (a > 0)
    grads = [None] * 12

    def lay(i, x, g):
        grads[i] = conv3d_wgrad(x, g)
        return conv3d_dgrad(g, P[i][0])

    g = mask(lay(11, c["d0"], gout), c["d0"])
    gc0 = lay(10, c["c0"], g)
    acc0 = gc0[..., 32:].copy()
    g = mask(up_bwd(gc0[..., :32]), c["d1"])
    gc1 = lay(9, c["c1"], g)
    acc1 = gc1[..., 64:].copy()
    g = mask(up_bwd(gc1[..., :64]), c["d2"])
    gc2 = lay(8, c["c2"], g)
    acc2 = gc2[..., 64:].copy()
    g = mask(up_bwd(gc2[..., :64]), c["e3"])
    g = mask(lay(7, c["a6"], g), c["a6"])
    gp2 = lay(6, c["p2"], g)
    g = mask(acc2 + pool_bwd(gp2), c["e2"])
    g = mask(lay(5, c["a4"], g), c["a4"])
    gp1 = lay(4, c["p1"], g)
    g = mask(acc1 + pool_bwd(gp1), c["e1"])
    g = mask(lay(3, c["a2"], g), c["a2"])
    gp0 = lay(2, c["p0"], g)
    g = mask(acc0 + pool_bwd(gp0), c["e0"])
    g = mask(lay(1, c["a0"], g), c["a0"])
    lay(0, c["in"], g)
    flat = np.concatenate([np.concatenate([dw.ravel(), db]) for dw, db in grads])
    return loss, flat
