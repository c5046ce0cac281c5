"""The FP64 restatement of the warm-start network (oracle/nn_oracle.py), pinned on its own:
the data gradient is the adjoint of the convolution, the flipped-weight convolution equals it,
the weight gradient matches a directional difference, and the whole network's gradient
matches central differences of its loss.  CPU only."""
import numpy as np

from oracle import nn_oracle as N


def _rng(s):
    return np.random.default_rng(s)


def test_dgrad_is_the_adjoint_and_the_flipped_convolution():
    r = _rng(1)
    x = r.normal(size=(4, 5, 6, 16))
    w = r.normal(size=(32, 27, 16))
    g = r.normal(size=(4, 5, 6, 32))
    lhs = float((N.conv3d(x, w) * g).sum())
    rhs = float((x * N.conv3d_dgrad(g, w)).sum())
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)
    np.testing.assert_allclose(N.conv3d(g, N.flip_weights(w)), N.conv3d_dgrad(g, w), rtol=1e-12, atol=1e-12)


def test_wgrad_matches_directional_derivative():
    r = _rng(2)
    x = r.normal(size=(3, 4, 5, 16))
    g = r.normal(size=(3, 4, 5, 16))
    w = r.normal(size=(16, 27, 16))
    dw = r.normal(size=w.shape)
    db = r.normal(size=16)
    gw, gb = N.conv3d_wgrad(x, g)
    # the convolution is linear in (w, b): the directional derivative is exact
    lhs = float(((N.conv3d(x, w + dw, db) - N.conv3d(x, w)) * g).sum())
    rhs = float((gw * dw).sum() + (gb * db).sum())
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_network_gradient_matches_central_differences():
    r = _rng(3)
    n = 8
    lnK = r.normal(size=(n, n, n))
    h = 1.0 - (np.arange(n) + 0.5)[None, None, :] / n + 0.05 * r.normal(size=(n, n, n))
    sizes = [ci * co * 27 + co for ci, co, _ in N.LAYERS]
    p = np.concatenate([r.normal(size=k) * 0.15 for k in sizes])
    loss, grad = N.loss_and_grad(p, lnK, h)
    for k in range(3):
        d = r.normal(size=p.size)
        eps = 1e-6
        lp, _ = N.loss_and_grad(p + eps * d, lnK, h)
        lm, _ = N.loss_and_grad(p - eps * d, lnK, h)
        fd = (lp - lm) / (2 * eps)
        an = float(grad @ d)
        assert abs(fd - an) <= 1e-5 * max(abs(an), 1e-12), (fd, an)
