"""Training data, training and evaluation of the learned warm start, all on the GPU.

The plain solver generates its own training pairs: scenes are stepped with the reference's uniform initial guess,
and after every step whose solve converged each body's grid gives the network input (node mass, explicit
momentum p*, forces, Jacobi diagonal) and target (the solved velocity x minus p*/m on heavy nodes, in units of
h/dt).  Volumes are cut into
24^3 windows at a stride of 16 whose central 16^3 nodes carry the loss (each output there sees its whole 9^3
receptive field inside the window, as it does in the step), on the heavy nodes.

  python -m mpmsnow_b200.warm_start_train --family snowball --out warm_start_snowball.npz
  python -m mpmsnow_b200.warm_start_train --family slab --out warm_start_slab.npz

Scene families (seeded, synthetic):
  snowball  snowball drops: radius U[0.05, 0.2] m, downward speed U[0, 5] m/s, E0 log-uniform [5e4, 5e5] Pa,
            50k-200k particles, h = 0.01 m, dt = 5e-4 s, ground plane y = 0; training seeds 1000-1199,
            held-out seeds 2000-2019.
  slab      sections of the 30-degree slab (34 x 86 cells across at h = 1/171 m, 2 x 2 x 2 jittered particles per
            cell, E0 log-uniform [1e5, 2e5] Pa) of 10-30 cells length, dt = 2.5e-4 s; other seeds than the
            headline slab's.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from . import scenes as S

WIN = 24
CORE = 16
HALO = (WIN - CORE) // 2


# --- scenes ---------------------------------------------------------------------------------------------------
def snowball_drop(seed):
    rng = np.random.default_rng(seed)
    r = float(rng.uniform(0.05, 0.2))
    speed = float(rng.uniform(0.0, 5.0))
    e0 = float(math.exp(rng.uniform(math.log(5e4), math.log(5e5))))
    n = int(rng.integers(50_000, 200_001))
    gap = float(rng.uniform(0.0, 0.02))
    sc = S.snowball(n=n, radius=r, centre=(0.0, r + gap, 0.0), velocity=(0.0, -speed, 0.0), h=0.01, dt=5e-4,
                    seed=seed)
    sc["snow"] = (e0,) + tuple(S.SNOW[1:])
    sc["name"] = f"snowball_drop_{seed}"
    return sc


def slab_section(seed):
    rng = np.random.default_rng(seed)
    length = int(rng.integers(10, 31))
    sc = S.slab(cells=(length, 34, 86), h=1.0 / 171, seed_jitter=seed, seed_e0=seed + 7919)
    sc["name"] = f"slab_section_{seed}_{length}"
    return sc


FAMILIES = {
    "snowball": {"scene": snowball_drop, "train": range(1000, 1200), "test": range(2000, 2020), "steps": 40,
                 "capture_from": 2, "capture_every": 2},
    "slab": {"scene": slab_section, "train": range(3000, 3024), "test": range(4000, 4004), "steps": 60,
             "capture_from": 1, "capture_every": 3},
}


# --- capture --------------------------------------------------------------------------------------------------
def capture_bodies(sim, tol, min_nodes=512, full=True):
    """Host copies of every body's grid after a step whose solve converged to tol: dims, masses, explicit
    momenta, solution, and (full) forces, Jacobi diagonal and collision flags."""
    out = []
    st = sim.last_stats
    for b in range(min(st["n_bodies"], 64)):
        if st["exit"][b] != 0 or not st["rNorm2"][b] <= tol * tol * st["bNorm2"][b]:
            continue  # not converged (or a trivial solve): no target
        info = sim.grid_info(b)
        n3 = [int(v) for v in info["n"]]
        if n3[0] * n3[1] * n3[2] < min_nodes:
            continue
        c = {"body": b, "n": n3, "mn": info["min"].astype(np.float64), "m": sim.grid_get(b, "masses"),
             "ps": sim.grid_get(b, "explicitMomenta"), "x": sim.grid_get(b, "solution")}
        if full:
            c["f"] = sim.grid_get(b, "forces")
            c["d"] = sim.grid_get(b, "diag")
            c["flag"] = sim.grid_get(b, "nodeCollided")
        out.append(c)
    return out


def history_record(c, density, light_mass):
    """What the step records after a solve (mpm_nn.h): x - p*/m on heavy nodes, x on light ones, NaN without mass."""
    m = c["m"].astype(np.float64)
    x = c["x"].reshape(-1, 3).astype(np.float64)
    ps = c["ps"].reshape(-1, 3).astype(np.float64)
    has = m > 0
    heavy = has & (m / (density * c["h"] ** 3) >= light_mass)
    out = np.full_like(x, np.nan)
    out[heavy] = x[heavy] - ps[heavy] / m[heavy, None]
    light = has & ~heavy
    out[light] = x[light]
    return out.astype(np.float32)


def contact_normals(c, colliders):
    """The outward normal of the collider each node collided with in the explicit update (nodeCollided >= 0), 0
    elsewhere, as the step's features take them, in the same separately rounded float32 operations (node position
    h i + min, the gradient, its norm, the division): planes and cylinders, the training scenes' colliders."""
    f32 = np.float32
    nx, ny, nz = c["n"]
    flag = np.asarray(c["flag"]).reshape(-1)
    out = np.zeros((flag.size, 3), dtype=f32)
    idx = np.nonzero(flag >= 0)[0]
    if idx.size:
        ijk = np.stack([idx % nx, (idx // nx) % ny, idx // (nx * ny)], 1).astype(f32)
        pos = f32(c["h"]) * ijk + np.asarray(c["mn"], dtype=f32)[None, :]
        for o, col in enumerate(colliders):
            sel = flag[idx] == o
            if not sel.any():
                continue
            if col["kind"] == 0:
                g = np.broadcast_to(np.asarray(col["c"][:3], dtype=f32), (int(sel.sum()), 3))
            elif col["kind"] == 1:
                p = pos[sel]
                g = np.stack([p[:, 0] - f32(col["c"][0]), np.zeros(len(p), dtype=f32), p[:, 2] - f32(col["c"][1])], 1)
            else:
                raise ValueError("contact normals of sampled colliders are not restated here")
            nn = np.sqrt((g[:, 0] * g[:, 0] + g[:, 1] * g[:, 1]) + g[:, 2] * g[:, 2])
            out[idx[sel]] = g / nn[:, None]
    return out.reshape(-1)


def map_history(prev, c):
    """A previous record of the same body on the current grid (integer shift of the origins), NaN outside."""
    n, pn = c["n"], prev["n"]
    off = np.rint((c["mn"] - prev["mn"]) / c["h"]).astype(int)
    src = prev["hist"].reshape(pn[2], pn[1], pn[0], 3)
    out = np.full((n[2], n[1], n[0], 3), np.nan, dtype=np.float32)
    zi, yi, xi = np.arange(n[2]) + off[2], np.arange(n[1]) + off[1], np.arange(n[0]) + off[0]
    vz, vy, vx = (zi >= 0) & (zi < pn[2]), (yi >= 0) & (yi < pn[1]), (xi >= 0) & (xi < pn[0])
    out[np.ix_(vz, vy, vx)] = src[np.ix_(zi[vz], yi[vy], xi[vx])]
    return out.reshape(-1)


def generate(family, seeds, max_iters=60, tol=1e-5, log=print, density=S.DENSITY, light_mass=0.05):
    """Step each scene of the family with the plain solver; returns captures (with the previous step's history
    record of the same body mapped onto the capture's grid, where there is one, and the contact normals) and
    per-scene stats."""
    from . import sim as M
    fam = FAMILIES[family]
    caps, meta = [], []
    for seed in seeds:
        sc = fam["scene"](seed)
        sim = M.from_scene(sc)
        term = M.SquareMagnitudeTermination(max_iters, tol)
        t0 = time.time()
        n_caps = 0
        prev = {}   # per body: the history record of the previous step
        g = np.sum(np.asarray(sc["gravity"], dtype=np.float32), 0)
        for step in range(fam["steps"]):
            sim.advance(sc["dt"], term)
            want = step >= fam["capture_from"] and (step - fam["capture_from"]) % fam["capture_every"] == 0
            now = {}
            for c in capture_bodies(sim, tol, full=want):
                c.update(h=sc["h"], dt=sc["dt"], gravity=g)
                c["hist"] = history_record(c, density, light_mass)
                if want:
                    c["hist_prev"] = map_history(prev[c["body"]], c) if c["body"] in prev else None
                    c["nrm"] = contact_normals(c, sc["colliders"])
                    caps.append(c)
                    n_caps += 1
                now[c["body"]] = {"n": c["n"], "mn": c["mn"], "hist": c["hist"]}
            prev = now
        meta.append({"seed": seed, "particles": int(sc["x"].shape[0]), "captures": n_caps,
                     "seconds": round(time.time() - t0, 2)})
        del sim
    log(f"[{family}] {len(seeds)} scenes, {len(caps)} captured grids")
    return caps, meta


# --- normalisation and windows ----------------------------------------------------------------------------------
def classes(m, h, density, light_mass):
    """Nodes with mass, heavy nodes (mass at least light_mass of density h^3) and the mass in that unit."""
    mh = m / (density * h ** 3)
    has = m > 0
    return has, has & (mh >= light_mass), mh


def raw_channels(c, density, light_mass, use_history=False):
    """Unscaled features (16) and target (3) of a capture, float64 numpy: for normalisation statistics."""
    m = c["m"].astype(np.float64)
    ps = c["ps"].reshape(-1, 3).astype(np.float64)
    f = c["f"].reshape(-1, 3).astype(np.float64)
    d = c["d"].reshape(-1, 3).astype(np.float64)
    x = c["x"].reshape(-1, 3).astype(np.float64)
    h, dt = c["h"], c["dt"]
    has, heavy, mh = classes(m, h, density, light_mass)
    inv = np.where(heavy, 1.0 / np.where(heavy, m, 1.0), 0.0)
    v = ps * inv[:, None]
    acc = (dt * f * inv[:, None] - dt * c["gravity"][None, :]) * heavy[:, None]
    stiff = (d - m[:, None]) * inv[:, None]
    hist = np.zeros_like(x)
    if use_history and c.get("hist_prev") is not None:
        hp = c["hist_prev"].reshape(-1, 3).astype(np.float64)
        ok = heavy & ~np.isnan(hp[:, 0])
        hist[ok] = hp[ok]
    nrm = c["nrm"].reshape(-1, 3).astype(np.float64) * heavy[:, None]
    feat = np.concatenate([mh[:, None] * has[:, None], v * dt / h, acc * dt / h, stiff, hist * dt / h, nrm], 1)
    target = (x - v - hist) * dt / h * heavy[:, None]
    return feat, target, has, heavy


def normalisation(caps, density=S.DENSITY, light_mass=0.05, use_history=False):
    """Feature scales (inverse RMS over heavy nodes) and the output scale (RMS of the heavy nodes' targets), so
    that every input channel and the output are of unit size."""
    sq = np.zeros(16)
    tq = 0.0
    cnt = 0
    for c in caps:
        feat, target, has, heavy = raw_channels(c, density, light_mass, use_history)
        sq += (feat[heavy] ** 2).sum(0)
        tq += (target[heavy] ** 2).sum()
        cnt += int(heavy.sum())
    rms = np.sqrt(sq / max(cnt, 1))
    feature_scale = np.where(rms > 0, 1.0 / np.maximum(rms, 1e-30), 1.0).astype(np.float32)
    out = float(np.sqrt(tq / max(3 * cnt, 1))) or 1.0
    return feature_scale, out


def windows(caps, net, density=S.DENSITY, stiffness_weight=False):
    """Device tensors of every 24^3 window with mass in its core: features (bf16 [T, 24^3 * 16]), targets
    (fp32 [T, 24^3, 3], in the units of the network output) and loss weights (fp32 [T, 24^3]: 1 on the core's
    heavy nodes, or with stiffness_weight their Jacobi diagonal over their mass, d / m averaged over the axes,
    so that the loss weighs a node's error as the implicit matrix's diagonal does)."""
    import torch
    import torch.nn.functional as F

    from . import learned
    L = net.L
    dev = net.device
    Xs, Ys, Ws = [], [], []
    core = torch.zeros(WIN, WIN, WIN, device=dev)
    core[HALO:HALO + CORE, HALO:HALO + CORE, HALO:HALO + CORE] = 1.0
    for c in caps:
        nx, ny, nz = c["n"]
        G = nx * ny * nz
        m = torch.from_numpy(c["m"]).to(dev)
        ps = torch.from_numpy(c["ps"]).to(dev)
        f = torch.from_numpy(c["f"]).to(dev)
        d = torch.from_numpy(c["d"]).to(dev)
        x = torch.from_numpy(c["x"]).to(dev).view(G, 3)
        hp = None
        if net.use_history and c.get("hist_prev") is not None:
            hp = torch.from_numpy(np.ascontiguousarray(c["hist_prev"])).to(dev)
        nrm = torch.from_numpy(np.ascontiguousarray(c["nrm"])).to(dev)
        feat = torch.empty(G * 16, dtype=torch.bfloat16, device=dev)
        learned.features(L, m, ps, f, d, hp, nrm, c["dt"], c["h"], density, net.light_mass, c["gravity"],
                         net.feature_scale, feat, net.stream)
        has, heavy, _ = classes(m, c["h"], density, net.light_mass)
        v = ps.view(G, 3) / torch.where(has, m, torch.ones_like(m))[:, None] * has[:, None]
        base = v
        if hp is not None:
            hv = hp.view(G, 3)
            base = v + torch.where(torch.isnan(hv), torch.zeros_like(hv), hv)
        tgt = (x - base) * (c["dt"] / c["h"] / net.output_scale) * heavy[:, None]
        wgt = heavy.float()
        if stiffness_weight:
            dm = d.view(G, 3).mean(1) / torch.where(has, m, torch.ones_like(m))
            wgt = wgt * dm / dm[heavy].mean().clamp_min(1e-30)
        # pad by the halo (and up to a multiple of the core) and cut windows
        px, py, pz = [(-n) % CORE for n in (nx, ny, nz)]
        fv = F.pad(feat.view(nz, ny, nx, 16), (0, 0, HALO, HALO + px, HALO, HALO + py, HALO, HALO + pz))
        tv = F.pad(tgt.view(nz, ny, nx, 3), (0, 0, HALO, HALO + px, HALO, HALO + py, HALO, HALO + pz))
        wv = F.pad(wgt.view(nz, ny, nx), (HALO, HALO + px, HALO, HALO + py, HALO, HALO + pz))
        for z0 in range(0, nz + pz, CORE):
            for y0 in range(0, ny + py, CORE):
                for x0 in range(0, nx + px, CORE):
                    w = wv[z0:z0 + WIN, y0:y0 + WIN, x0:x0 + WIN] * core
                    if float(w.sum()) <= 0:
                        continue
                    Xs.append(fv[z0:z0 + WIN, y0:y0 + WIN, x0:x0 + WIN].reshape(-1))
                    Ys.append(tv[z0:z0 + WIN, y0:y0 + WIN, x0:x0 + WIN].reshape(-1, 3))
                    Ws.append(w.reshape(-1))
    return torch.stack(Xs), torch.stack(Ys), torch.stack(Ws)


# --- training ---------------------------------------------------------------------------------------------------
def train(net, X, Y, Wt, iters=3000, batch=16, lr=2e-3, seed=0, log=print, val=None):
    """Adam with a cosine learning-rate decay over random batches of windows.  Returns the loss history."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    T = X.shape[0]
    hist = []
    dims = (WIN, WIN, WIN, batch)
    for it in range(iters):
        idx = torch.randint(0, T, (batch,), generator=g).to(X.device)
        net.grads.zero_()
        loss = net.loss_backward(X[idx].reshape(-1), dims, Y[idx].reshape(-1, 3).contiguous(),
                                 Wt[idx].reshape(-1).contiguous())
        net.adam(lr=lr * 0.5 * (1 + math.cos(math.pi * it / iters)))
        if it % 100 == 0 or it == iters - 1:
            hist.append((it, float(loss.item())))
            if val is not None and (it % 500 == 0 or it == iters - 1):
                hist[-1] = hist[-1] + (evaluate_loss(net, *val, batch=batch),)
            log(f"  iter {it} loss {hist[-1][1:]}")
    net.check_err()
    return hist


def evaluate_loss(net, X, Y, Wt, batch=16):
    import torch
    tot, wsum = 0.0, 0.0
    for i in range(0, X.shape[0], batch):
        xb, yb, wb = X[i:i + batch], Y[i:i + batch], Wt[i:i + batch]
        k = xb.shape[0]
        y = net.forward(xb.reshape(-1), (WIN, WIN, WIN, k))
        d = (y.view(k, -1, 3) - yb) ** 2
        tot += float((d.sum(-1) * wb).sum())
        wsum += float(wb.sum())
    return tot / max(wsum, 1e-30)


# --- evaluation in the step ---------------------------------------------------------------------------------------
def compare_in_step(family, seeds, net, steps=None, max_iters=60, tol=1e-5, min_nodes=0, log=print, base_only=True):
    """Plain vs learned warm start on each scene and, with base_only, the same guess without the network (p*/m,
    plus the history when the model uses it) and, for history models, that guess with the fixed linear
    extrapolation h1 - h2: CR iterations per step and device time per step."""
    import torch

    from . import sim as M
    fam = FAMILIES[family]
    steps = steps or fam["steps"]
    rows = []
    for seed in seeds:
        sc = fam["scene"](seed)
        row = {"seed": seed, "particles": int(sc["x"].shape[0])}
        modes = [("plain", None), ("learned", True)]
        if base_only:
            modes += [("base_only", False)] + ([("extrapolated", "extrapolate")] if net.use_history else [])
        for mode, network in modes:
            sim = M.from_scene(sc)
            if network is not None:
                net.install(sim._h, min_nodes=min_nodes, network=network is True, extrapolate=network == "extrapolate")
            term = M.SquareMagnitudeTermination(max_iters, tol)
            its, ms = [], []
            stream = torch.cuda.ExternalStream(M.stream_ptr(sim))
            for _ in range(steps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                st = sim.advance(sc["dt"], term)
                e1.record(stream)
                e1.synchronize()
                ms.append(e0.elapsed_time(e1))
                its.append(st["total_iterations"])
            row[mode] = {"iterations_per_step": float(np.mean(its)), "ms_per_step": float(np.mean(ms)),
                         "iterations": its}
            del sim
        row["iteration_ratio"] = row["plain"]["iterations_per_step"] / max(row["learned"]["iterations_per_step"], 1e-9)
        row["time_ratio"] = row["plain"]["ms_per_step"] / max(row["learned"]["ms_per_step"], 1e-9)
        extra = ""
        if base_only:
            extra = (f", without the network {row['base_only']['iterations_per_step']:.1f} it "
                     f"{row['base_only']['ms_per_step']:.2f} ms")
            if "extrapolated" in row:
                extra += (f", linear extrapolation {row['extrapolated']['iterations_per_step']:.1f} it "
                          f"{row['extrapolated']['ms_per_step']:.2f} ms")
        log(f"  seed {seed}: plain {row['plain']['iterations_per_step']:.1f} it {row['plain']['ms_per_step']:.2f} ms, "
            f"learned {row['learned']['iterations_per_step']:.1f} it {row['learned']['ms_per_step']:.2f} ms{extra}")
        rows.append(row)
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--family", default="snowball", choices=sorted(FAMILIES))
    ap.add_argument("--out", required=True)
    ap.add_argument("--train-scenes", type=int, default=None)
    ap.add_argument("--test-scenes", type=int, default=None)
    ap.add_argument("--iters", type=int, default=3000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--report", default=None)
    ap.add_argument("--light-mass", type=float, default=0.05)
    ap.add_argument("--history", action="store_true", help="the previous step's correction as input and base")
    ap.add_argument("--stiffness-weight", action="store_true",
                    help="weigh each node's squared error by its Jacobi diagonal over its mass")
    args = ap.parse_args()
    import torch

    from .learned import WarmStartNet
    fam = FAMILIES[args.family]
    train_seeds = list(fam["train"])[:args.train_scenes]
    test_seeds = list(fam["test"])[:args.test_scenes]
    t0 = time.time()
    caps, meta = generate(args.family, train_seeds)
    t_gen = time.time() - t0
    net = WarmStartNet(seed=0)
    net.light_mass = args.light_mass
    net.use_history = args.history
    net.feature_scale, net.output_scale = normalisation(caps, light_mass=net.light_mass, use_history=net.use_history)
    net.density = S.DENSITY
    nval = max(1, len(caps) // 10)
    X, Y, Wt = windows(caps[nval:], net, stiffness_weight=args.stiffness_weight)
    Xv, Yv, Wv = windows(caps[:nval], net, stiffness_weight=args.stiffness_weight)
    print(f"windows: train {X.shape[0]}, validation {Xv.shape[0]}; data {t_gen:.1f}s", flush=True)
    torch.cuda.synchronize()
    t1 = time.time()
    hist = train(net, X, Y, Wt, iters=args.iters, batch=args.batch, lr=args.lr, val=(Xv, Yv, Wv))
    torch.cuda.synchronize()
    t_train = time.time() - t1
    np.savez(args.out, **net.state_dict())
    rows = compare_in_step(args.family, test_seeds, net)
    rep = {"family": args.family, "train_scenes": len(train_seeds), "captures": len(caps),
           "windows": int(X.shape[0]), "data_seconds": t_gen, "train_seconds": t_train, "iters": args.iters,
           "batch": args.batch, "loss_history": hist, "feature_scale": net.feature_scale.tolist(),
           "output_scale": net.output_scale, "light_mass": net.light_mass, "use_history": net.use_history,
           "test": rows,
           "mean_iteration_ratio": float(np.mean([r["iteration_ratio"] for r in rows])),
           "mean_time_ratio": float(np.mean([r["time_ratio"] for r in rows])),
           "mean_iterations": {k: float(np.mean([r[k]["iterations_per_step"] for r in rows]))
                               for k in ("plain", "learned", "base_only", "extrapolated") if k in rows[0]}}
    if args.report:
        with open(args.report, "w") as f:
            json.dump(rep, f, indent=1)
    print(json.dumps({k: v for k, v in rep.items() if k not in ("test", "loss_history")}), flush=True)


if __name__ == "__main__":
    main()
