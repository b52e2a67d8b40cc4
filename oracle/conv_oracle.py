"""CPU ORACLE — test infrastructure only, never on the product path.

Float64 numpy forward and backward of the learned warm start's network (four 3x3x3 convolutions, 7 -> 32 -> 32
-> 32 -> 3 channels, ReLU between layers, weighted squared-error loss), the checker of the tensor-core kernels
in ``mpmsnow_b200/csrc/mpm_conv.cu``.  The reference has no learned part (its initial guess is the uniform
velocity of ``src/MpmSim/Grid.cpp:911-947``), so there is no reference file to follow here: this restates the
convolution and its gradients from their definitions, and ``tests/test_nn_oracle.py`` pins the gradients with
central finite differences.

Layout (the kernels' layout): activations ``[batch][z][y][x][channel]``; weights ``W[t][cin][cout]`` with tap
``t = 9 (dz + 1) + 3 (dy + 1) + (dx + 1)``; ``y[v] = sum_t x[v + off(t)] W[t]`` with zeros outside the volume.

``quantize=True`` rounds to bfloat16 (round-to-nearest-even) exactly where the kernels store bf16: the network
input, the weights, every hidden activation, the output gradient and the back-propagated gradients, so the
oracle and the kernels differ only by fp32 summation order.
"""
from __future__ import annotations

import numpy as np

LAYERS = [(7, 32, True), (32, 32, True), (32, 32, True), (32, 3, False)]  # (cin, cout, relu)
PADS = [(16, 32), (32, 32), (32, 32), (32, 16)]


def taps():
    return [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]


def bf16(a):
    """Round float values to bfloat16 (nearest, ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = r.astype(np.uint32).view(np.float32).astype(np.float64)
    return np.where(np.isfinite(f), out, f.astype(np.float64))


def shift(x, dz, dy, dx):
    """s[b, z, y, x] = x[b, z + dz, y + dy, x + dx] (zero outside the volume)."""
    out = np.zeros_like(x)
    _, Z, Y, X, _ = x.shape

    def rng(n, d):
        return slice(max(0, -d), min(n, n - d)), slice(max(0, d), min(n, n + d))

    (zo, zi), (yo, yi), (xo, xi) = rng(Z, dz), rng(Y, dy), rng(X, dx)
    out[:, zo, yo, xo] = x[:, zi, yi, xi]
    return out


def conv_forward(x, W, b=None):
    """y = sum_t shift(x, off(t)) W[t] (+ b)."""
    y = np.zeros(x.shape[:4] + (W.shape[2],))
    for t, (dz, dy, dx) in enumerate(taps()):
        y += shift(x, dz, dy, dx) @ W[t]
    if b is not None:
        y += b
    return y


def conv_backward_data(dy, W):
    """dx[u] = sum_t dy[u - off(t)] W[t]^T."""
    dx = np.zeros(dy.shape[:4] + (W.shape[1],))
    for t, (dz, dyy, dxx) in enumerate(taps()):
        dx += shift(dy, -dz, -dyy, -dxx) @ W[t].T
    return dx


def conv_wgrad(x, dy):
    """dW[t] = sum_v x[v + off(t)]^T dy[v]."""
    cin, cout = x.shape[-1], dy.shape[-1]
    dW = np.zeros((27, cin, cout))
    dy2 = dy.reshape(-1, cout)
    for t, (dz, dyy, dxx) in enumerate(taps()):
        dW[t] = shift(x, dz, dyy, dxx).reshape(-1, cin).T @ dy2
    return dW


def init_params(seed=0, scale=1.0):
    """He-initialised weights W[t][cin][cout] and zero biases, unpadded, float64."""
    rng = np.random.default_rng(seed)
    params = []
    for cin, cout, _ in LAYERS:
        W = rng.normal(0.0, scale * np.sqrt(2.0 / (27 * cin)), (27, cin, cout))
        params.append((W, np.zeros(cout)))
    return params


def forward(x, params, quantize=True):
    """Returns the output (fp64) and the stored activations [input, a1, a2, a3]."""
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    acts = [q(x)]
    h = acts[0]
    for li, ((W, b), (_, _, relu)) in enumerate(zip(params, LAYERS)):
        z = conv_forward(h, q(W), b)
        if relu:
            h = q(np.maximum(z, 0.0))
            acts.append(h)
        else:
            return z, acts
    raise AssertionError


def loss_and_grads(x, target, weight, params, quantize=True):
    """Weighted squared error L = sum_v w_v |y_v - t_v|^2 / sum_v w_v and its gradients (dW, db per layer)."""
    q = bf16 if quantize else (lambda a: np.asarray(a, dtype=np.float64))
    y, acts = forward(x, params, quantize)
    inv = 1.0 / weight.sum()
    d = y - target
    loss = float((weight[..., None] * d * d).sum() * inv)
    g = q(2.0 * weight[..., None] * d * np.float32(inv))
    grads = [None] * len(params)
    for li in range(len(params) - 1, -1, -1):
        W, b = params[li]
        grads[li] = (conv_wgrad(acts[li], g), g.reshape(-1, g.shape[-1]).sum(0))
        if li == 0:
            break
        g = conv_backward_data(g, q(W))
        g = q(np.where(acts[li] > 0, g, 0.0))
    return loss, y, grads
