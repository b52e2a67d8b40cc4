"""Generates the FP64-oracle fixtures of the benchmark configurations (test infrastructure).

The CPU oracle (``oracle/``, the restated reference step) runs a configuration's seeded scene for its steps in
FP64 (and, with ``--prec 32``, in FP32: the reference's own arithmetic) and keeps what the GPU parity tests of
``tests/test_gpu_config_fixtures.py`` compare against, small enough to commit:

* the displacement from the initial position of an evenly strided sample of particles (caller order), at each
  saved step, and their velocities at the last step;
* over ALL particles at each saved step: the largest coordinate magnitude and the largest displacement (the two
  scales the position error is stated against);
* the final grid velocities (absolute: frame velocity added) and masses of a strided sample of each body's nodes
  with mass, keyed by world node index ``round(min / h) + (i, j, k)``; with ``--nodes-like FIXTURE`` at that
  fixture's nodes instead (NaN where this run's grid has no such node), so that an FP32 run is compared with the
  FP64 run node by node;
* the oracle's CR iterations and body count per step.

  python tests/golden/make_config_fixtures.py --config c3 [--prec 64] [--threads 4] [--nodes-like c3_fp64.npz]

Scenes are regenerated from their seeds by ``mpmsnow_b200.scenes``; nothing else is read.  Runtimes on 4 host
threads: c3 (4,000,032 particles, 100 steps) about 2 h, c2 (1,000,000 particles, 200 steps) about 1 h, c5s (the
avalanche section, 100 steps) a few minutes.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# config name -> (scene factory, steps, steps whose positions are kept)
CONFIGS = {
    "c3": ("slab", 100, (50, 100)),
    "c2": ("two_snowballs", 200, (100, 200)),
    "c5s": ("avalanche_section", 100, (50, 100)),
}
N_SAMPLE_PARTICLES = 4096
N_SAMPLE_NODES = 4096


def scene(name):
    from mpmsnow_b200 import scenes as S
    return getattr(S, CONFIGS[name][0])()


def particle_sample(n):
    stride = max(1, n // N_SAMPLE_PARTICLES)
    return np.arange(0, n, stride, dtype=np.int64)[:N_SAMPLE_PARTICLES]


def grid_sample(mass, n3, mn, h, vel, fv, like=None):
    """Strided sample of the nodes with mass (or the world node indices `like`): world node index (3 ints),
    absolute velocity and mass (NaN velocity and zero mass where the grid has no such node)."""
    origin = np.rint(np.asarray(mn, dtype=np.float64) / h).astype(np.int64)
    n3 = np.asarray(n3, dtype=np.int64)
    if like is None:
        heavy = np.flatnonzero(mass > 0)
        stride = max(1, heavy.size // N_SAMPLE_NODES)
        sel = heavy[::stride][:N_SAMPLE_NODES]
        i = sel % n3[0]
        j = (sel // n3[0]) % n3[1]
        k = sel // (n3[0] * n3[1])
        idx = np.stack([i + origin[0], j + origin[1], k + origin[2]], 1).astype(np.int32)
        v = vel.reshape(-1, 3)[sel] + np.asarray(fv, dtype=np.float64)[None, :]
        return idx, v, np.asarray(mass, dtype=np.float64)[sel]
    idx = np.asarray(like, dtype=np.int64)
    loc = idx - origin[None, :]
    inside = np.all((loc >= 0) & (loc < n3[None, :]), axis=1)
    v = np.full((idx.shape[0], 3), np.nan)
    m = np.zeros(idx.shape[0])
    flat = loc[inside, 0] + n3[0] * (loc[inside, 1] + n3[1] * loc[inside, 2])
    v[inside] = vel.reshape(-1, 3)[flat] + np.asarray(fv, dtype=np.float64)[None, :]
    m[inside] = np.asarray(mass, dtype=np.float64)[flat]
    return idx.astype(np.int32), v, m


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", required=True, choices=sorted(CONFIGS))
    ap.add_argument("--prec", type=int, default=64, choices=(32, 64))
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=None)
    ap.add_argument("--nodes-like", default=None, help="sample the grids at this fixture's nodes")
    args = ap.parse_args()
    from oracle import oracle as O
    O.build()
    sc = scene(args.config)
    _, steps, save = CONFIGS[args.config]
    n = sc["x"].shape[0]
    p0 = sc["x"].astype(np.float64)
    sample = particle_sample(n)
    o = O.OracleSim(sc["x"], sc["m"], sc["h"], sc["snow"], sc["colliders"], sc["gravity"], prec=args.prec,
                    threads=args.threads, mu0=sc.get("mu0"), lambda0=sc.get("lambda0"))
    if "v" in sc and np.any(sc["v"]):
        o.set("v", sc["v"])
    out = {"sample": sample.astype(np.int32), "steps": np.array(sorted(save), dtype=np.int32)}
    iters, bodies = [], []
    t0 = time.time()
    for s in range(1, steps + 1):
        st = o.advance(sc["dt"], 60, 1e-5)
        iters.append(int(sum(st["iterations"])))
        bodies.append(int(st["n_bodies"]))
        print(json.dumps({"step": s, "bodies": st["n_bodies"], "ballistic": st["n_ballistic"],
                          "iterations": st["iterations"][:4], "t_s": round(time.time() - t0, 1)}), flush=True)
        if s in save:
            p = o.get("p")
            out[f"disp_step{s}"] = p[sample] - p0[sample]
            out[f"max_abs_step{s}"] = np.array(np.abs(p).max())
            out[f"max_disp_step{s}"] = np.array(np.linalg.norm(p - p0, axis=1).max())
    out["v_last"] = o.get("v")[sample]
    like = dict(np.load(args.nodes_like)) if args.nodes_like else None
    for b in range(o.num_grids()):
        info = o.grid_info(b)
        idx, v, m = grid_sample(o.grid_get(b, "masses"), info["n"], info["min"], sc["h"], o.grid_get(b, "velocities"),
                                info["frame_velocity"], None if like is None else like.get(f"grid{b}_node"))
        out[f"grid{b}_node"] = idx
        out[f"grid{b}_v"] = v
        out[f"grid{b}_m"] = m
    out["n_grids"] = np.array(o.num_grids())
    out["cr_iterations"] = np.array(iters, dtype=np.int32)
    out["n_bodies"] = np.array(bodies, dtype=np.int32)
    path = args.out or os.path.join(HERE, f"{args.config}_fp{args.prec}.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path}", flush=True)


if __name__ == "__main__":
    main()
