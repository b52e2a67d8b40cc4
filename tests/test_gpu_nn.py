"""The learned warm start's tensor-core kernels against the float64 CPU oracle — needs a B200.

Each convolution kernel (forward, backward data, weight gradient; every channel-width pair the network uses),
the whole network's loss and gradients, training on the GPU, and the warm start inside the step (which must
leave the solve's result unchanged to the solver tolerance).
"""
import ctypes as C

import numpy as np
import pytest

from oracle import conv_oracle as O

pytestmark = pytest.mark.gpu

PAIRS = [(16, 32, 7, 32), (32, 32, 32, 32), (32, 16, 32, 3), (16, 16, 16, 16)]   # cin_pad, cout_pad, cin, cout


def _lib():
    from mpmsnow_b200 import build, capi
    build.build()
    return capi.load()


def _bf(a):
    import torch
    return torch.tensor(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16).cuda().contiguous()


def _f32(a):
    import torch
    return torch.tensor(np.ascontiguousarray(a, dtype=np.float32)).cuda().contiguous()


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _pack(L, W, cin_pad, cout_pad):
    import torch
    n = 27 * cin_pad * cout_pad
    wf = torch.empty(n, dtype=torch.bfloat16, device="cuda")
    wb = torch.empty(n, dtype=torch.bfloat16, device="cuda")
    Wd = _f32(W)
    assert L.mpm_nn_pack_weights(_p(Wd), cin_pad, cout_pad, cin_pad, cout_pad, _p(wf), _p(wb), None) == 0
    torch.cuda.synchronize()
    return wf, wb


def _layer(rng, cin_pad, cout_pad, cin, cout):
    W = np.zeros((27, cin_pad, cout_pad))
    W[:, :cin, :cout] = rng.normal(0, 0.2, (27, cin, cout))
    b = np.zeros(cout_pad)
    b[:cout] = rng.normal(0, 0.1, cout)
    return W, b


@pytest.mark.parametrize("cin_pad,cout_pad,cin,cout", PAIRS)
def test_conv_forward_matches_oracle(cin_pad, cout_pad, cin, cout):
    import torch
    L = _lib()
    rng = np.random.default_rng(cin_pad * 100 + cout_pad)
    dims = (9, 7, 5, 2)                       # 630 voxels: 5 M tiles, the last one partial
    nx, ny, nz, nb = dims
    x = np.zeros((nb, nz, ny, nx, cin_pad))
    x[..., :cin] = rng.normal(size=(nb, nz, ny, nx, cin))
    W, b = _layer(rng, cin_pad, cout_pad, cin, cout)
    xq, Wq = O.bf16(x), O.bf16(W)
    wf, _ = _pack(L, W, cin_pad, cout_pad)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    for relu in (0, 1):
        ref = O.conv_forward(xq, Wq) + b
        if relu:
            ref = np.maximum(ref, 0)
        y32 = torch.zeros(630 * cout, dtype=torch.float32, device="cuda")
        ybf = torch.full((630 * cout_pad,), 7.0, dtype=torch.bfloat16, device="cuda")
        xd, bd = _bf(x), _f32(b)     # held: a pointer to a freed temporary could be reused by the next allocation
        rc = L.mpm_nn_conv3d(_p(xd), cin_pad, _p(wf), _p(bd), cout, cout_pad, relu, 0, None, _p(ybf), _p(y32),
                             cout, nx, ny, nz, nb, _p(err), None)
        assert rc == 0
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        got = y32.cpu().numpy().reshape(nb, nz, ny, nx, cout)
        scale = np.abs(ref).max()
        assert np.abs(got - ref[..., :cout]).max() <= 2e-6 * scale * np.sqrt(27 * cin)
        gbf = ybf.float().cpu().numpy().reshape(nb, nz, ny, nx, cout_pad)
        assert np.all(gbf[..., cout:] == 0)
        # bf16 output = the fp32 result rounded (a rounding flip at most where the two sums straddle a tie)
        assert np.mean(gbf[..., :cout] == O.bf16(got)) > 0.999


@pytest.mark.parametrize("cin_pad,cout_pad,cin,cout", PAIRS)
def test_conv_backward_data_matches_oracle(cin_pad, cout_pad, cin, cout):
    import torch
    L = _lib()
    rng = np.random.default_rng(7 + cin_pad + cout_pad)
    nx, ny, nz, nb = 6, 11, 4, 3
    n = nx * ny * nz * nb
    W, _ = _layer(rng, cin_pad, cout_pad, cin, cout)
    g = np.zeros((nb, nz, ny, nx, cout_pad))
    g[..., :cout] = rng.normal(size=(nb, nz, ny, nx, cout))
    act = np.zeros((nb, nz, ny, nx, cin_pad))
    act[..., :cin] = np.maximum(rng.normal(size=(nb, nz, ny, nx, cin)), 0)   # about half the mask zero
    gq, Wq, aq = O.bf16(g), O.bf16(W), O.bf16(act)
    ref = np.where(aq > 0, O.conv_backward_data(gq, Wq), 0.0)
    _, wb = _pack(L, W, cin_pad, cout_pad)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    y32 = torch.zeros(n * cin, dtype=torch.float32, device="cuda")
    ybf = torch.full((n * cin_pad,), 3.0, dtype=torch.bfloat16, device="cuda")
    gd, ad = _bf(g), _bf(act)
    rc = L.mpm_nn_conv3d(_p(gd), cout_pad, _p(wb), None, cin, cin_pad, 0, 1, _p(ad), _p(ybf), _p(y32), cin,
                         nx, ny, nz, nb, _p(err), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    got = y32.cpu().numpy().reshape(nb, nz, ny, nx, cin)
    assert np.abs(got - ref[..., :cin]).max() <= 2e-6 * np.abs(ref).max() * np.sqrt(27 * cout)
    assert np.all(ybf.float().cpu().numpy().reshape(nb, nz, ny, nx, cin_pad)[..., cin:] == 0)


@pytest.mark.parametrize("cin_pad,cout_pad,cin,cout", PAIRS)
def test_conv_weight_gradient_matches_oracle(cin_pad, cout_pad, cin, cout):
    import torch
    L = _lib()
    rng = np.random.default_rng(11 + cin_pad * cout_pad)
    nx, ny, nz, nb = 13, 11, 9, 2             # 2,574 voxels: two CTAs along the voxels, a partial 64-voxel stage
    x = np.zeros((nb, nz, ny, nx, cin_pad))
    x[..., :cin] = rng.normal(size=(nb, nz, ny, nx, cin))
    g = np.zeros((nb, nz, ny, nx, cout_pad))
    g[..., :cout] = rng.normal(size=(nb, nz, ny, nx, cout))
    xq, gq = O.bf16(x), O.bf16(g)
    ref = O.conv_wgrad(xq, gq)
    dw = torch.full((27 * cin_pad * cout_pad,), 0.5, dtype=torch.float32, device="cuda")   # accumulates
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    xd, gd = _bf(x), _bf(g)
    rc = L.mpm_nn_conv3d_wgrad(_p(xd), cin_pad, _p(gd), cout_pad, _p(dw), nx, ny, nz, nb, _p(err), None)
    assert rc == 0
    db = torch.zeros(cout_pad, dtype=torch.float32, device="cuda")
    assert L.mpm_nn_bias_grad(_p(gd), cout_pad, cout, nx * ny * nz * nb, _p(db), None) == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    got = dw.cpu().numpy().reshape(27, cin_pad, cout_pad) - 0.5
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max() * 10
    assert np.allclose(db.cpu().numpy()[:cout], gq.reshape(-1, cout_pad).sum(0)[:cout], rtol=1e-4, atol=1e-3)


def test_network_loss_and_gradients_match_oracle():
    """The whole network through WarmStartNet (forward, mse, backward) against the oracle with the kernels'
    bf16 storage points: loss, output and every layer's weight and bias gradient."""
    import torch

    from mpmsnow_b200.learned import WarmStartNet
    _lib()
    rng = np.random.default_rng(21)
    params = O.init_params(seed=5)
    params = [(W, rng.normal(0, 0.05, b.shape)) for W, b in params]
    net = WarmStartNet(seed=0)
    net.set_params([W for W, _ in params], [b for _, b in params])
    nx, ny, nz, nb = 10, 9, 8, 2
    n = nx * ny * nz * nb
    x7 = rng.normal(size=(nb, nz, ny, nx, 7))
    x16 = np.zeros((nb, nz, ny, nx, 16))
    x16[..., :7] = x7
    target = rng.normal(size=(nb, nz, ny, nx, 3)) * 0.3
    weight = rng.uniform(0, 1, size=(nb, nz, ny, nx)) * (rng.uniform(size=(nb, nz, ny, nx)) > 0.3)
    loss_ref, y_ref, grads_ref = O.loss_and_grads(x7, target, weight, params, quantize=True)
    net.grads.zero_()
    loss = net.loss_backward(_bf(x16).view(-1), (nx, ny, nz, nb), _f32(target.reshape(n, 3)), _f32(weight.reshape(n)))
    torch.cuda.synchronize()
    net.check_err()
    y = net._bufs["out"][:n * 3].cpu().numpy().reshape(nb, nz, ny, nx, 3)
    assert np.abs(y - y_ref).max() <= 1e-3 * np.abs(y_ref).max()
    assert abs(float(loss.item()) - loss_ref) <= 1e-3 * loss_ref
    for i, (dW_ref, db_ref) in enumerate(grads_ref):
        dW = net.dW(i).cpu().numpy().reshape(27, O.PADS[i][0], O.PADS[i][1])
        cin, cout = dW_ref.shape[1], dW_ref.shape[2]
        assert np.all(dW[:, cin:, :] == 0) and np.all(dW[:, :, cout:] == 0)
        rel = np.linalg.norm(dW[:, :cin, :cout] - dW_ref) / np.linalg.norm(dW_ref)
        assert rel < 5e-3, (i, rel)
        db = net.db(i).cpu().numpy()[:cout]
        assert np.linalg.norm(db - db_ref) <= 5e-3 * np.linalg.norm(db_ref) + 1e-7, i


def test_training_on_the_gpu_reduces_the_loss():
    """A teacher network's outputs on random inputs, learned by a freshly initialised network with Adam."""
    import torch

    from mpmsnow_b200.learned import WarmStartNet
    _lib()
    rng = np.random.default_rng(31)
    teacher = O.init_params(seed=9, scale=0.7)
    nx, ny, nz, nb = 12, 12, 12, 4
    n = nx * ny * nz * nb
    x7 = rng.normal(size=(nb, nz, ny, nx, 7))
    y_t, _ = O.forward(x7, teacher, quantize=False)
    x16 = np.zeros((nb, nz, ny, nx, 16))
    x16[..., :7] = x7
    xd, td = _bf(x16).view(-1), _f32(y_t.reshape(n, 3))
    wd = torch.ones(n, dtype=torch.float32, device="cuda")
    net = WarmStartNet(seed=1)
    losses = []
    for it in range(300):
        net.grads.zero_()
        loss = net.loss_backward(xd, (nx, ny, nz, nb), td, wd)
        net.adam(lr=2e-3)
        if it % 50 == 0 or it == 299:
            losses.append(float(loss.item()))
    net.check_err()
    assert losses[-1] < 0.4 * losses[0], losses


def test_in_step_inference_matches_the_whole_volume():
    """The step evaluates each layer only on the output blocks within reach of the heavy nodes, the only nodes
    that read the network's output (the last layer at those nodes, layer l within 3 - l of them).  At every
    heavy node the step's correction x0 - p*/m equals the network run over the whole volume on the same
    features."""
    import torch
    from mpmsnow_b200 import learned
    from mpmsnow_b200 import sim as M
    from mpmsnow_b200.learned import WarmStartNet
    from mpmsnow_b200.warm_start_train import contact_normals
    from tests.gpu_helpers import slab_scene
    L = _lib()
    sc = slab_scene()
    warm = M.from_scene(sc)
    net = WarmStartNet(seed=3, out_init_scale=0.5)
    net.feature_scale[:] = 1.0
    net.output_scale = 0.05
    net.install(warm._h, min_nodes=0, use_history=False)
    warm.advance(sc["dt"], M.SquareMagnitudeTermination(60, 1e-5), stop_phase=1)  # first step: no history
    nx, ny, nz = (int(v) for v in warm.grid_info(0)["n"])
    G = nx * ny * nz
    dev = "cuda:0"
    arrays = {k: warm.grid_get(0, k) for k in ("masses", "explicitMomenta", "forces", "diag", "x0", "nodeCollided")}
    m, ps, f, d = (torch.from_numpy(arrays[k]).to(dev) for k in ("masses", "explicitMomenta", "forces", "diag"))
    info = warm.grid_info(0)
    cap = {"n": (nx, ny, nz), "mn": info["min"], "h": sc["h"], "flag": arrays["nodeCollided"]}
    nrm_host = contact_normals(cap, sc["colliders"])
    assert np.abs(nrm_host).sum() > 0          # the contact normals are among the features
    nrm = torch.from_numpy(nrm_host).to(dev)
    gravity = np.sum(np.asarray(sc["gravity"], dtype=np.float32), 0)
    feat = torch.empty(G * 16, dtype=torch.bfloat16, device=dev)
    torch.cuda.synchronize()
    learned.features(L, m, ps, f, d, None, nrm, sc["dt"], sc["h"], net.density, net.light_mass, gravity, net.feature_scale,
                     feat, net.stream)
    y = net.forward(feat, (nx, ny, nz, 1))
    net.stream.synchronize()
    y = y.float().cpu().numpy().reshape(G, 3)
    net.check_err()
    h = np.float32(sc["h"])
    mass = arrays["masses"]
    rel = mass * (np.float32(1) / (np.float32(net.density) * h * h * h)) / np.float32(net.light_mass)
    heavy = (mass > 0) & (rel >= 1.0 + 1e-4)          # clear of the threshold's rounding
    assert heavy.sum() > 1000 and (mass > 0).sum() > heavy.sum()
    v = arrays["explicitMomenta"].reshape(-1, 3)[heavy].astype(np.float64) / mass[heavy, None]
    corr = arrays["x0"].reshape(-1, 3)[heavy].astype(np.float64) - v
    ref = np.float64(net.output_scale) * (sc["h"] / sc["dt"]) * y[heavy].astype(np.float64)
    assert np.abs(ref).max() > 0
    err = np.abs(corr - ref).max()
    assert err <= 1e-5 * np.abs(v).max() + 1e-4 * np.abs(ref).max(), (err, np.abs(ref).max(), np.abs(v).max())


def test_warm_start_in_the_step_keeps_the_solution():
    """A network installed into the step replaces the initial guess; CR still converges to the tolerance, so
    positions after a few steps agree with the plain step's to the solver's accuracy."""
    from mpmsnow_b200 import sim as M
    from mpmsnow_b200.learned import WarmStartNet
    from tests.gpu_helpers import rel_err, slab_scene
    _lib()
    sc = slab_scene()
    term = M.SquareMagnitudeTermination(200, 1e-6)
    plain = M.from_scene(sc)
    warm = M.from_scene(sc)
    net = WarmStartNet(seed=2, out_init_scale=0.5)     # an untrained network: a poor guess, never a wrong answer
    net.feature_scale[:] = 1.0
    net.output_scale = 0.05
    net.install(warm._h, min_nodes=0)
    M.profile_enable(warm, True)
    its_p, its_w = [], []
    for _ in range(4):
        its_p.append(plain.advance(sc["dt"], term)["iterations"][0])
        st = warm.advance(sc["dt"], term)
        its_w.append(st["iterations"][0])
        assert all(e == 0 for e in st["exit"])
    p0 = plain.particleData().variable("p").copy()
    p1 = warm.particleData().variable("p").copy()
    assert rel_err(p1, p0) < 1e-5, rel_err(p1, p0)
    prof = {p["name"]: p for p in M.profile_read(warm)}
    assert prof["warm_start_net"]["launches"] == 4        # one profiled phase per step (6 kernels)
    x0 = warm.grid_get(0, "x0").reshape(-1, 3)
    m = warm.grid_get(0, "masses")
    ps = warm.grid_get(0, "explicitMomenta").reshape(-1, 3)
    assert np.all(x0[m == 0] == 0)
    assert not np.allclose(x0[m > 0], ps[m > 0] / m[m > 0, None])   # the network's correction is applied
