"""Shared helpers of the GPU parity tests: one scene, two implementations (CUDA via the C-ABI, and the oracle)."""
import math

import numpy as np

from mpmsnow_b200 import scenes as S


def gpu_sim(scene, device=0):
    from mpmsnow_b200 import sim as M
    return M.from_scene(scene, device=device)


def oracle_sim(scene, prec=64, threads=1):
    from oracle import oracle as O
    sim = O.OracleSim(scene["x"], scene["m"], scene["h"], scene["snow"], scene["colliders"], scene["gravity"],
                      prec=prec, threads=threads, mu0=scene.get("mu0"), lambda0=scene.get("lambda0"),
                      dimension=scene.get("dimension", 3))
    if np.any(scene["v"]):
        sim.set("v", scene["v"])
    return sim


def impact_scene(n=3000, seed=7, height=0.105, speed=2.0, h=0.01, dt=5e-4):
    """A small snowball already touching the ground, moving down and sideways: contact, friction, plasticity."""
    sc = S.snowball(n=n, radius=0.1 * (n / 10000) ** (1 / 3), centre=(0.0, height, 0.0), velocity=(0.5, -speed, 0.2),
                    h=h, dt=dt, seed=seed)
    return sc


def slab_scene(cells=(24, 6, 12)):
    """The headline slab's shape at test size: a jittered 8-per-cell lattice resting on a 30 degree plane with
    per-particle E0 (13,824 particles at the default size); contact from the first step, well-conditioned."""
    return S.slab(cells=cells, h=0.5 / cells[0])


def oracle_threads():
    import os
    return max(1, min(16, os.cpu_count() or 1))


def two_body_scene(n_each=1500):
    a = S.sphere_points(n_each, 0.05, (-0.08, 0.06, 0.0), 31)
    b = S.sphere_points(n_each, 0.05, (0.08, 0.055, 0.01), 32)
    x = np.concatenate([a, b])
    v = np.concatenate([np.tile(np.float32((1.5, -1.0, 0.0)), (n_each, 1)),
                        np.tile(np.float32((-1.5, -0.5, 0.0)), (n_each, 1))])
    m = np.full(2 * n_each, S.DENSITY * 4 / 3 * math.pi * 0.05 ** 3 / n_each, dtype=np.float32)
    return {"name": "two_bodies", "x": x, "v": v, "m": m, "h": 0.01, "dt": 5e-4, "steps": 10, "snow": S.SNOW,
            "colliders": [S.plane((0.0, 1.0, 0.0, 0.0), 0.5)], "gravity": [S.GRAVITY]}


def moving_planes_scene():
    """The reference's implicit-update scene (TestGrid.cpp:456-536): 64 particles, two moving planes.  The
    reference builds that Grid directly; through Sim the particles must be closer than h to form one body
    (at exactly h apart every particle is ballistic, KdTree.inl:188), so the lattice spacing is 0.9 h."""
    h = 0.5
    rng = np.random.default_rng(17)
    distortion = rng.uniform(-1, 1, (3, 3)) * 0.001
    sp = 0.9 * h
    pts = [((i - 0.5) * sp, (j - 0.5) * sp, (k - 0.5) * sp) for i in range(4) for j in range(4) for k in range(4)]
    x = np.array(pts, dtype=np.float32)
    v = (0.1 + 0.01 * np.sin(2 * x.astype(np.float64))).astype(np.float32)
    F = np.stack([(np.eye(3) + distortion * math.cos(2 * p[0])) for p in x.astype(np.float64)]).astype(np.float32)
    return {"name": "moving_planes", "x": x, "v": v, "m": np.ones(64, dtype=np.float32), "h": h, "dt": 0.002,
            "steps": 1, "snow": (1.4e5, 0.2, 0.0, 1e5, 1e5), "F": F,
            "colliders": [S.plane((-1, -1, -1, 1), vel=(-0.1, -0.2, -0.3)), S.plane((-1, 0, 0, 1.5), vel=(-0.2, -0.1, -0.4))],
            "gravity": []}


def rel_err(a, b, scale=None):
    """max |a - b| relative to max |b| (or to a given scale, for arrays whose entries are all near zero)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if scale is None:
        scale = np.abs(b).max()
    return np.abs(a - b).max() / max(scale, 1e-30)
