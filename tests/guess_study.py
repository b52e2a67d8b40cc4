"""Where the CR iterations left after the warm start's physical guess come from, on the FP64 oracle — a study
script run by hand on the CPU (not collected by pytest):

  python tests/guess_study.py [--length 20] [--steps 10] [--threads 8]

It steps a slab section (the headline slab's cross-section, ``--length`` cells long) with the FP64 oracle,
records each step's solution, stops the next step after the rhs and the Jacobi diagonal are built (Grid.cpp:
983-1002, 841-867), and runs conjugate residuals (ConjugateResiduals.cpp:19-160, the oracle's order of
operations, with the collision projection of Grid.cpp:778-818) from several initial guesses to the 1e-5
relative residual of the step, printing one JSON object:

* the reference's uniform guess (Grid.cpp:911-947) and the warm start's guess without the network: p*/m - vc on
  heavy nodes (mass >= 0.05 rho h^3) plus the previous step's correction mapped by the integer origin shift;
* that guess plus the best correction from a coarse space (Galerkin: minimising the operator-norm error over
  piecewise-constant fields on k^3-node blocks), the most a coarse-scale predictor could add;
* the guess's residual by node class (heavy, light, collided), and the guess with the exact solution put in on
  one class at a time.
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
    ap.add_argument("--length", type=int, default=20)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--threads", type=int, default=8)
    args = ap.parse_args()
    from mpmsnow_b200 import scenes as S
    from tests.gpu_helpers import oracle_sim

    sc = S.slab(cells=(args.length, 34, 86), h=1.0 / 171)
    h, dt = sc["h"], sc["dt"]
    o = oracle_sim(sc, prec=64, threads=args.threads)
    nrm = np.array(sc["colliders"][0]["c"][:3], dtype=np.float64)
    nrm /= np.linalg.norm(nrm)
    rho_h3 = 400.0 * h ** 3

    def base_of(m, ps, vc):
        heavy = m >= 0.05 * rho_h3
        out = np.zeros_like(ps)
        out.reshape(-1, 3)[heavy] = ps.reshape(-1, 3)[heavy] / m[heavy, None] - vc.reshape(-1, 3)[heavy]
        return out

    steps = []
    prev = None
    for _ in range(args.steps):
        st = o.advance(dt, 60, 1e-5)
        steps.append(st["iterations"][0])
        info = o.grid_info(0)
        m, ps, vc, x = (o.grid_get(0, k) for k in ("masses", "explicitMomenta", "vc", "solution"))
        prev = {"min": info["min"].copy(), "n": info["n"].copy(), "hist": x - base_of(m, ps, vc)}

    o.advance(dt, 60, 1e-5, stop_phase=1)
    info = o.grid_info(0)
    n = info["n"]
    b, d, m, ps, vc, x0 = (o.grid_get(0, k) for k in ("rhs", "diag", "masses", "explicitMomenta", "vc", "x0"))
    flags = o.grid_get(0, "nodeCollided").astype(int)
    has = (m > 0).reshape(n[2], n[1], n[0])

    def project(v):
        v = v.reshape(-1, 3).copy()
        v[flags == -2] = 0
        sel = flags >= 0
        v[sel] -= (v[sel] @ nrm)[:, None] * nrm[None, :]
        return v.reshape(-1)

    def A(v):
        return o.grid_apply(0, "A", v, dt)

    def cr(x, tol, max_iters=500):
        x = x.copy()
        thr = tol * tol * (b @ b)
        rpc = (b - A(x)) / d
        p = rpc.copy()
        Ap = A(p)
        rz = rpc @ Ap
        for i in range(max_iters + 1):
            pAp = Ap / d
            alpha = rz / (Ap @ pAp)
            x = project(x + alpha * p)
            rpc = rpc - alpha * pAp
            rr = rpc * d
            if i >= max_iters or rr @ rr < thr:
                return x, i
            Ar = A(rpc)
            rz_old, rz = rz, rpc @ Ar
            p = rpc + (rz / rz_old) * p
            Ap = Ar + (rz / rz_old) * Ap
        return x, max_iters

    # the previous step's correction on this step's grid (origins are multiples of h)
    off = np.rint((info["min"] - prev["min"]) / h).astype(int)
    hist = np.zeros((n[2], n[1], n[0], 3))
    ph = prev["hist"].reshape(prev["n"][2], prev["n"][1], prev["n"][0], 3)
    new_sl, old_sl = [], []
    for ax in (2, 1, 0):
        lo, hi = max(0, -off[ax]), min(n[ax], prev["n"][ax] - off[ax])
        new_sl.append(slice(lo, hi))
        old_sl.append(slice(lo + off[ax], hi + off[ax]))
    hist[tuple(new_sl)] = ph[tuple(old_sl)]
    guess = project(base_of(m, ps, vc) + hist.reshape(-1))
    xs, _ = cr(guess, 1e-12)

    def coarse(k, iters=80):
        nz, ny, nx = int(n[2]), int(n[1]), int(n[0])
        cz, cy, cx = -(-nz // k), -(-ny // k), -(-nx // k)

        def P(c):
            f = np.repeat(np.repeat(np.repeat(c.reshape(cz, cy, cx, 3), k, 0), k, 1), k, 2)[:nz, :ny, :nx]
            return project((f * has[..., None]).reshape(-1))

        def PT(f):
            g = project(f).reshape(nz, ny, nx, 3) * has[..., None]
            pad = np.zeros((cz * k, cy * k, cx * k, 3))
            pad[:nz, :ny, :nx] = g
            return pad.reshape(cz, k, cy, k, cx, k, 3).sum((1, 3, 5)).reshape(-1)

        rhs = PT(b - A(guess))
        c = np.zeros_like(rhs)
        r = rhs.copy()
        pdir = r.copy()
        rr = r @ r
        for _ in range(iters):
            Ap = PT(A(P(pdir)))
            alpha = rr / (pdir @ Ap)
            c += alpha * pdir
            r -= alpha * Ap
            rr_new = r @ r
            if rr_new < 1e-20 * (rhs @ rhs):
                break
            pdir = r + (rr_new / rr) * pdir
            rr = rr_new
        return P(c)

    res = {"particles": int(sc["x"].shape[0]), "grid": [int(v) for v in n], "iterations_of_the_steps": steps,
           "uniform guess": cr(x0, 1e-5)[1], "p*/m + history": cr(guess, 1e-5)[1],
           "relative residual of p*/m + history": float(np.linalg.norm(b - A(guess)) / np.linalg.norm(b))}
    for k in (2, 4, 8):
        g = project(guess + coarse(k))
        res[f"+ best coarse correction, {k}^3-node blocks"] = cr(g, 1e-5)[1]
        res[f"  its relative residual ({k}^3)"] = float(np.linalg.norm(b - A(g)) / np.linalg.norm(b))
    heavy = m >= 0.05 * rho_h3
    light = (m > 0) & ~heavy
    collided = flags != -1
    r0 = (b - A(guess)).reshape(-1, 3)
    tot = float(np.sum(r0 ** 2))
    for name, sel in (("heavy", heavy & ~collided), ("light", light & ~collided), ("collided", collided)):
        res[f"residual share, {name} nodes"] = float(np.sum(r0[sel] ** 2) / tot)
        res[f"node count, {name}"] = int(sel.sum())
        g = guess.reshape(-1, 3).copy()
        g[sel] = xs.reshape(-1, 3)[sel]
        res[f"exact on {name} nodes, the guess elsewhere"] = cr(project(g.reshape(-1)), 1e-5)[1]
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    main()
