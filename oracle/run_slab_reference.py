"""CPU ORACLE run (test infrastructure): the headline slab (4,000,032 particles) stepped by the FP64 (or FP32)
restatement of the reference, saving particle positions at chosen steps.

  python oracle/run_slab_reference.py --prec 64 --steps 100 --save 10,50,100 --out <dir> [--threads N]

tests/slab_precision.py steps the CUDA path on the same scene and compares its positions against these files,
which states the precision of the 4 M configuration against the FP64 oracle after 100 steps.
"""
import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--prec", type=int, default=64)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--save", default="10,50,100")
    ap.add_argument("--out", required=True)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--length-cells", type=int, default=171)
    args = ap.parse_args()
    from mpmsnow_b200 import scenes as S
    from oracle import oracle as O
    O.build()
    sc = S.slab() if args.length_cells == 171 else S.slab(cells=(args.length_cells, 34, 86), h=1.0 / 171)
    os.makedirs(args.out, exist_ok=True)
    save = {int(s) for s in args.save.split(",") if s}
    t0 = time.time()
    sim = O.OracleSim(sc["x"], sc["m"], sc["h"], sc["snow"], sc["colliders"], sc["gravity"], prec=args.prec,
                      threads=args.threads, mu0=sc["mu0"], lambda0=sc["lambda0"])
    log = open(os.path.join(args.out, f"log_fp{args.prec}.txt"), "a")
    for s in range(1, args.steps + 1):
        st = sim.advance(sc["dt"], 60, 1e-5)
        print(f"step {s} bodies {st['n_bodies']} ballistic {st['n_ballistic']} iterations {st['iterations'][:4]} "
              f"t={time.time() - t0:.0f}s", file=log, flush=True)
        if s in save:
            np.save(os.path.join(args.out, f"p_fp{args.prec}_step{s}.npy"), sim.get("p").astype(np.float64))


if __name__ == "__main__":
    main()
