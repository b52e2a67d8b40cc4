"""Learned warm start of the implicit solve: the network, its training on the GPU and its use in the step.

No counterpart in the reference, whose initial guess is one uniform velocity per body (``Grid.cpp:911-947``).
A 4-layer 3x3x3 convolutional network (16 -> 32 -> 32 -> 32 -> 3 channels, ReLU, bf16 weights and activations,
fp32 accumulation on the tensor cores) maps a body grid's node features — mass, explicit momentum p* and the
internal-force velocity increment ("stress" channels), the relative stiffness of the Jacobi diagonal, and the
last two steps' corrections (h1 and its change h1 - h2) — to the correction of the guess p*/m + h1 towards the
solved grid velocity on heavy nodes (the light shell that the B-spline stencil adds around the material keeps
the history: its solved velocity is barely determined).  Conjugate residuals still runs to the same relative residual from the predicted guess, so a poor
prediction costs iterations, never accuracy.

Every computation goes through the C-ABI's ``mpm_nn_*`` kernels (``mpmsnow_b200/csrc/mpm_conv.cu``); torch only
holds device memory.  Weights are fp32 masters, padded to the kernels' channel widths, with Adam moments; the
bf16 packs the kernels read are rebuilt after every update.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi

CIN_PAD = (16, 32, 32, 32)
COUT_PAD = (32, 32, 32, 16)
COUT = (32, 32, 32, 3)
CIN = (16, 32, 32, 32)
N_FEAT = 16


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _check(rc, what):
    if rc != 0:
        raise capi.MpmError(rc, what)


class WarmStartNet:
    """The network on one CUDA device: fp32 master weights, Adam state, bf16 packs, and training/inference."""

    def __init__(self, seed=0, device="cuda", init_scale=1.0, out_init_scale=0.1):
        import torch
        self.torch = torch
        self.L = capi.load()
        self.device = torch.device(device)
        self.stream = torch.cuda.current_stream(self.device)
        # flat parameters: W1..W4 ([27][cin_pad][cout_pad] each), then b1..b4 (32 each)
        self.wsz = [27 * CIN_PAD[i] * COUT_PAD[i] for i in range(4)]
        self.woff = np.concatenate([[0], np.cumsum(self.wsz)]).astype(int)
        self.boff = [int(self.woff[4]) + 32 * i for i in range(4)]
        self.n_params = int(self.woff[4]) + 128
        host = np.zeros(self.n_params, dtype=np.float32)
        rng = np.random.default_rng(seed)
        for i in range(4):
            W = np.zeros((27, CIN_PAD[i], COUT_PAD[i]), dtype=np.float32)
            std = init_scale * np.sqrt(2.0 / (27 * CIN[i])) * (out_init_scale if i == 3 else 1.0)
            W[:, :CIN[i], :COUT[i]] = rng.normal(0.0, std, (27, CIN[i], COUT[i]))
            host[self.woff[i]:self.woff[i + 1]] = W.reshape(-1)
        self.params = torch.from_numpy(host).to(self.device)
        self.grads = torch.zeros_like(self.params)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.adam_step = 0
        self.packs_f = [torch.empty(self.wsz[i], dtype=torch.bfloat16, device=self.device) for i in range(4)]
        self.packs_b = [torch.empty(self.wsz[i], dtype=torch.bfloat16, device=self.device) for i in range(4)]
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.loss_acc = torch.zeros(1, dtype=torch.float64, device=self.device)
        self.feature_scale = np.ones(N_FEAT, dtype=np.float32)
        self.output_scale = 1.0
        self.light_mass = 0.05
        self.density = 400.0
        self.use_history = False
        self._bufs = {}
        self.pack()

    # --- parameters -----------------------------------------------------------------------------------------
    def W(self, i):
        return self.params[self.woff[i]:self.woff[i + 1]]

    def b(self, i):
        return self.params[self.boff[i]:self.boff[i] + 32]

    def dW(self, i):
        return self.grads[self.woff[i]:self.woff[i + 1]]

    def db(self, i):
        return self.grads[self.boff[i]:self.boff[i] + 32]

    def set_params(self, weights_list, biases_list):
        """Unpadded float weights W[t][cin][cout] and biases per layer (e.g. from the oracle)."""
        host = np.zeros(self.n_params, dtype=np.float32)
        for i, (W, bb) in enumerate(zip(weights_list, biases_list)):
            Wp = np.zeros((27, CIN_PAD[i], COUT_PAD[i]), dtype=np.float32)
            Wp[:, :W.shape[1], :W.shape[2]] = W
            host[self.woff[i]:self.woff[i + 1]] = Wp.reshape(-1)
            host[self.boff[i]:self.boff[i] + len(bb)] = bb
        self.params.copy_(self.torch.from_numpy(host))
        self.pack()

    def host_params(self):
        """(weights [MPM_WARM_START_WEIGHTS], biases [MPM_WARM_START_BIASES]) as the C-ABI's mpm_warm_start wants."""
        p = self.params.cpu().numpy()
        w = p[:self.woff[4]].copy()
        b = np.concatenate([p[self.boff[i]:self.boff[i] + COUT[i]] for i in range(4)]).astype(np.float32)
        return w, b

    def state_dict(self):
        w, b = self.host_params()
        return {"weights": w, "biases": b, "feature_scale": self.feature_scale.copy(),
                "output_scale": np.float32(self.output_scale), "light_mass": np.float32(self.light_mass),
                "density": np.float32(self.density), "use_history": np.int32(self.use_history)}

    def load_state_dict(self, d):
        host = np.zeros(self.n_params, dtype=np.float32)
        host[:self.woff[4]] = d["weights"]
        o = 0
        for i in range(4):
            host[self.boff[i]:self.boff[i] + COUT[i]] = d["biases"][o:o + COUT[i]]
            o += COUT[i]
        self.params.copy_(self.torch.from_numpy(host))
        fs = np.zeros(N_FEAT, dtype=np.float32)
        fs[:len(d["feature_scale"])] = d["feature_scale"]     # earlier models had fewer input channels
        self.feature_scale = fs
        self.output_scale = float(d["output_scale"])
        self.light_mass = float(d["light_mass"])
        self.density = float(d["density"])
        self.use_history = int(d["use_history"]) if "use_history" in d else 0
        self.pack()

    def pack(self):
        s = C.c_void_p(self.stream.cuda_stream)
        for i in range(4):
            _check(self.L.mpm_nn_pack_weights(_ptr(self.W(i)), CIN_PAD[i], COUT_PAD[i], CIN_PAD[i], COUT_PAD[i],
                                              _ptr(self.packs_f[i]), _ptr(self.packs_b[i]), s), "pack")

    # --- buffers --------------------------------------------------------------------------------------------
    def _buf(self, name, n, ch, dtype):
        t = self._bufs.get(name)
        if t is None or t.numel() < n * ch or t.dtype != dtype:
            t = self.torch.empty(max(n, 1) * ch, dtype=dtype, device=self.device)
            self._bufs[name] = t
        return t[:n * ch]

    # --- forward / backward ---------------------------------------------------------------------------------
    def forward(self, x, dims, keep=False):
        """x: bf16 [nvox * 16] features; dims = (nx, ny, nz, batch).  Returns fp32 [nvox, 3]."""
        nx, ny, nz, nb = dims
        n = nx * ny * nz * nb
        s = C.c_void_p(self.stream.cuda_stream)
        bf = self.torch.bfloat16
        acts = [x]
        h = x
        for i in range(3):
            y = self._buf(f"a{i + 1}", n, 32, bf)
            _check(self.L.mpm_nn_conv3d(_ptr(h), CIN_PAD[i], _ptr(self.packs_f[i]), _ptr(self.b(i)), COUT[i], COUT_PAD[i],
                                        1, 0, None, _ptr(y), None, 0, nx, ny, nz, nb, _ptr(self.err), s), "conv")
            acts.append(y)
            h = y
        out = self._buf("out", n, 3, self.torch.float32)
        _check(self.L.mpm_nn_conv3d(_ptr(h), 32, _ptr(self.packs_f[3]), _ptr(self.b(3)), 3, 16, 0, 0, None, None,
                                    _ptr(out), 3, nx, ny, nz, nb, _ptr(self.err), s), "conv")
        if keep:
            self._acts = acts
        return out.view(n, 3)

    def loss_backward(self, x, dims, target, weight):
        """Forward, weighted squared error against target ([nvox, 3] fp32, weight [nvox] fp32) and the gradients
        (accumulated into self.grads, which the caller zeroes).  Returns the loss as a device scalar."""
        nx, ny, nz, nb = dims
        n = nx * ny * nz * nb
        s = C.c_void_p(self.stream.cuda_stream)
        bf = self.torch.bfloat16
        y = self.forward(x, dims, keep=True)
        acts = self._acts
        wsum = float(weight.sum().item())
        self.loss_acc.zero_()
        g = self._buf("g16", n, 16, bf)
        _check(self.L.mpm_nn_mse(_ptr(y), 3, _ptr(target), _ptr(weight), n, 1.0 / max(wsum, 1e-30), _ptr(g),
                                 _ptr(self.loss_acc), s), "mse")
        gin, gin_pad = g, 16
        for i in range(3, -1, -1):
            _check(self.L.mpm_nn_conv3d_wgrad(_ptr(acts[i]), CIN_PAD[i], _ptr(gin), gin_pad, _ptr(self.dW(i)), nx, ny, nz,
                                              nb, _ptr(self.err), s), "wgrad")
            _check(self.L.mpm_nn_bias_grad(_ptr(gin), gin_pad, COUT[i], n, _ptr(self.db(i)), s), "bias grad")
            if i == 0:
                break
            gout = self._buf(f"g{i}", n, 32, bf)
            _check(self.L.mpm_nn_conv3d(_ptr(gin), gin_pad, _ptr(self.packs_b[i]), None, CIN[i], CIN_PAD[i], 0, 1,
                                        _ptr(acts[i]), _ptr(gout), None, 0, nx, ny, nz, nb, _ptr(self.err), s), "dgrad")
            gin, gin_pad = gout, 32
        return self.loss_acc

    def adam(self, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        self.adam_step += 1
        s = C.c_void_p(self.stream.cuda_stream)
        _check(self.L.mpm_nn_adam(_ptr(self.params), _ptr(self.grads), _ptr(self.m), _ptr(self.v), self.n_params, lr,
                                  beta1, beta2, eps, self.adam_step, weight_decay, s), "adam")
        self.pack()

    def check_err(self):
        e = int(self.err.item())
        if e:
            raise RuntimeError(f"tensor-core wait timed out in a convolution kernel (flag {e})")

    # --- the step ---------------------------------------------------------------------------------------------
    def install(self, sim_handle, min_nodes=4096, network=True, use_history=None, extrapolate=False):
        """Install into a C-ABI handle (mpm_set_warm_start).  network=False installs the guess without the network
        (p*/m, plus the history if used; with extrapolate, plus the linear extrapolation h1 - h2)."""
        hist = int(self.use_history if use_history is None else use_history)
        if extrapolate and not network and hist:
            hist = 2
        install_guess(sim_handle, self.feature_scale, self.output_scale, self.light_mass, self.density, min_nodes,
                      hist, self.host_params() if network else None)


def install_guess(sim_handle, feature_scale=None, output_scale=1.0, light_mass=0.05, density=400.0, min_nodes=0,
                  use_history=False, params=None):
    """mpm_set_warm_start with an optional network (params = (weights, biases) as host_params returns)."""
    L = capi.load()
    ws = capi.MpmWarmStart()
    keep = []
    if params is not None:
        wc = np.ascontiguousarray(params[0], dtype=np.float32)
        bc = np.ascontiguousarray(params[1], dtype=np.float32)
        keep += [wc, bc]
        ws.weights = wc.ctypes.data_as(C.POINTER(C.c_float))
        ws.biases = bc.ctypes.data_as(C.POINTER(C.c_float))
    fs = np.ones(N_FEAT, dtype=np.float32) if feature_scale is None else np.asarray(feature_scale, dtype=np.float32)
    for k in range(N_FEAT):
        ws.feature_scale[k] = float(fs[k])
    ws.output_scale = float(output_scale)
    ws.light_mass = float(light_mass)
    ws.density = float(density)
    ws.min_nodes = int(min_nodes)
    ws.use_history = int(use_history)
    _check(L.mpm_set_warm_start(sim_handle, C.byref(ws)), "mpm_set_warm_start")


def features(L, mass, pstar, force, diag, history, normals, dt, h, density, light_mass, gravity, feature_scale, out,
             stream):
    """Node features of captured grid arrays (device tensors; the history record h1 and the contact normals may be
    None) into out (bf16 [n * 16])."""
    g = np.ascontiguousarray(gravity, dtype=np.float32)
    fs = np.ascontiguousarray(feature_scale, dtype=np.float32)
    _check(L.mpm_nn_features(_ptr(mass), _ptr(pstar), _ptr(force), _ptr(diag), _ptr(history), _ptr(normals),
                             mass.numel(), dt, h, density, light_mass, g.ctypes.data_as(C.c_void_p),
                             fs.ctypes.data_as(C.c_void_p), _ptr(out), C.c_void_p(stream.cuda_stream)), "features")
