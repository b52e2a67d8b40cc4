"""Precision of the CUDA step on the headline slab (4,000,032 particles) against the FP64 oracle after 100 steps.

Test infrastructure, run by hand on a B200 (the oracle's positions are made by ``oracle/run_slab_reference.py``
on the host, ~1.5 h with 8 threads, and are too large to commit):

  python oracle/run_slab_reference.py --prec 64 --steps 100 --save 1,10,50,100 --out <dir>
  python tests/slab_precision.py --oracle-dir <dir> [--warm-start]

For each saved step it prints one JSON line: the maximum position error relative to the largest coordinate
(the criterion of the parity tests), the maximum and RMS error in metres, the largest displacement from the
initial positions, and the error relative to that displacement.  The oracle files may be float64 or float32
(``p_fp64_step<k>.npy``).
"""
import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--oracle-dir", required=True)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warm-start", action="store_true", help="step with the packaged slab warm-start model")
    args = ap.parse_args()
    from mpmsnow_b200 import build, scenes as S, sim as M
    build.build()
    sc = S.slab()
    sim = M.from_scene(sc)
    if args.warm_start:
        from mpmsnow_b200.learned import WarmStartNet
        net = WarmStartNet(seed=0)
        net.load_state_dict(dict(np.load(os.path.join(ROOT, "mpmsnow_b200", "warm_start_slab.npz"))))
        net.install(sim._h, min_nodes=0)
    term = M.SquareMagnitudeTermination(60, 1e-5)
    p0 = sc["x"].astype(np.float64)
    its = []
    for step in range(1, args.steps + 1):
        st = sim.advance(sc["dt"], term)
        its.append(st["total_iterations"])
        f = os.path.join(args.oracle_dir, f"p_fp64_step{step}.npy")
        if not os.path.exists(f):
            continue
        ref = np.load(f).astype(np.float64).reshape(-1, 3)
        p = sim.particleData().variable("p").astype(np.float64).reshape(-1, 3)
        d = np.abs(p - ref)
        disp = np.linalg.norm(ref - p0, axis=1).max()
        err = np.linalg.norm(p - ref, axis=1)
        print(json.dumps({"step": step, "particles": int(p.shape[0]), "warm_start": args.warm_start,
                          "rel_err_max": float(d.max() / np.abs(ref).max()), "err_max_m": float(err.max()),
                          "err_rms_m": float(np.sqrt((err ** 2).mean())), "max_displacement_m": float(disp),
                          "err_max_over_displacement": float(err.max() / max(disp, 1e-30)),
                          "cr_iterations_per_step_so_far": float(np.mean(its))}), flush=True)


if __name__ == "__main__":
    main()
