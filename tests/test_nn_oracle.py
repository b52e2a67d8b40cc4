"""The learned warm start's CPU oracle (oracle/conv_oracle.py), pinned without a GPU: the convolution against a
direct loop, the gradients against central finite differences, the bf16 rounding against torch's."""
import numpy as np
import pytest

from oracle import conv_oracle as O


def _direct_conv(x, W):
    nb, Z, Y, X, _ = x.shape
    y = np.zeros((nb, Z, Y, X, W.shape[2]))
    for b in range(nb):
        for z in range(Z):
            for yy in range(Y):
                for xx in range(X):
                    for t, (dz, dy, dx) in enumerate(O.taps()):
                        zs, ys, xs = z + dz, yy + dy, xx + dx
                        if 0 <= zs < Z and 0 <= ys < Y and 0 <= xs < X:
                            y[b, z, yy, xx] += x[b, zs, ys, xs] @ W[t]
    return y


def test_tap_order():
    t = O.taps()
    assert t[0] == (-1, -1, -1) and t[13] == (0, 0, 0) and t[26] == (1, 1, 1)
    assert t[1] == (-1, -1, 0) and t[3] == (-1, 0, -1) and t[9] == (0, -1, -1)   # x fastest, then y, then z


def test_conv_matches_direct_loop():
    rng = np.random.default_rng(0)
    x = rng.normal(size=(2, 3, 4, 5, 3))
    W = rng.normal(size=(27, 3, 2))
    assert np.allclose(O.conv_forward(x, W), _direct_conv(x, W), atol=1e-12)


def test_backward_data_and_wgrad_are_adjoints():
    """<conv(x), g> = <x, conv^T(g)> = <W, wgrad(x, g)>."""
    rng = np.random.default_rng(1)
    x = rng.normal(size=(2, 4, 3, 5, 3))
    W = rng.normal(size=(27, 3, 4))
    g = rng.normal(size=(2, 4, 3, 5, 4))
    lhs = (O.conv_forward(x, W) * g).sum()
    assert np.isclose(lhs, (x * O.conv_backward_data(g, W)).sum(), rtol=1e-12)
    assert np.isclose(lhs, (W * O.conv_wgrad(x, g)).sum(), rtol=1e-12)


def test_network_gradients_match_finite_differences():
    rng = np.random.default_rng(2)
    params = O.init_params(seed=3)
    x = rng.normal(size=(1, 4, 5, 3, 7))
    target = rng.normal(size=(1, 4, 5, 3, 3))
    weight = rng.uniform(0, 1, size=(1, 4, 5, 3))
    loss, _, grads = O.loss_and_grads(x, target, weight, params, quantize=False)
    eps = 1e-6
    for li in range(4):
        W, b = params[li]
        for _ in range(4):
            idx = tuple(rng.integers(0, s) for s in W.shape)
            Wp = W.copy(); Wp[idx] += eps
            Wm = W.copy(); Wm[idx] -= eps
            pp = list(params); pp[li] = (Wp, b)
            pm = list(params); pm[li] = (Wm, b)
            fd = (O.loss_and_grads(x, target, weight, pp, False)[0] - O.loss_and_grads(x, target, weight, pm, False)[0]) / (2 * eps)
            assert abs(fd - grads[li][0][idx]) <= 1e-6 + 1e-5 * abs(fd), (li, idx, fd, grads[li][0][idx])
        k = int(rng.integers(0, len(b)))
        bp = b.copy(); bp[k] += eps
        bm = b.copy(); bm[k] -= eps
        pp = list(params); pp[li] = (W, bp)
        pm = list(params); pm[li] = (W, bm)
        fd = (O.loss_and_grads(x, target, weight, pp, False)[0] - O.loss_and_grads(x, target, weight, pm, False)[0]) / (2 * eps)
        assert abs(fd - grads[li][1][k]) <= 1e-6 + 1e-5 * abs(fd), (li, k)


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(4)
    vals = np.concatenate([rng.normal(size=2000) * 10.0 ** rng.integers(-6, 6, 2000),
                           [1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -1.0 - 2 ** -8, 0.0, 65504.0, 3.0e38]])
    ours = O.bf16(vals)
    ref = torch.tensor(vals, dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(ours, ref)
    assert O.bf16(np.array([1.0 + 2 ** -8]))[0] == 1.0                 # tie to even
    assert O.bf16(np.array([1.0 + 3 * 2 ** -8]))[0] == 1.0 + 2 ** -6   # tie to even (upwards)
