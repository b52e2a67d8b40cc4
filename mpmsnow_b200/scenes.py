"""Seeded synthetic scenes with the shapes of the benchmark configurations.

No public dataset is involved: every scene is generated from a fixed seed with numpy.  All quantities are SI
(m, kg, s, Pa).  A scene is a dict with particle arrays (float32), the grid spacing, the time step, the snow
parameters in ``SnowConstitutiveModel``'s argument order ``(E, nu, xi, theta_c, theta_s)``
(SnowConstitutiveModel.h:13-18), colliders in the C-ABI's ``mpm_collider`` meaning, and gravity fields.
"""
from __future__ import annotations

import math

import numpy as np

SNOW = (1.4e5, 0.2, 10.0, 2.5e-2, 7.5e-3)   # E0, nu, xi, theta_c, theta_s
DENSITY = 400.0
GRAVITY = (0.0, -9.81, 0.0)


def plane(c, friction=0.5, sticky=False, vel=(0.0, 0.0, 0.0)):
    """``CollisionPlane(c, friction, sticky)`` (CollisionPlane.h:16), phi = c0 x + c1 y + c2 z + c3."""
    return {"kind": 0, "c": tuple(float(v) for v in c), "vel": tuple(vel), "friction": float(friction),
            "sticky": bool(sticky)}


def cylinder(cx, cz, radius, friction=0.5, sticky=False, vel=(0.0, 0.0, 0.0)):
    """Vertical solid cylinder collider (axis along y through (cx, cz)); no reference counterpart."""
    return {"kind": 1, "c": (float(cx), float(cz), float(radius), 0.0), "vel": tuple(vel),
            "friction": float(friction), "sticky": bool(sticky)}


def grid_collider(phi, origin, spacing, velocity=None, friction=0.5, sticky=False):
    """A collider sampled on a dense grid (the GPU form of the Houdini plugin's VDBCollisionObject): phi of shape
    (nz, ny, nx) at origin + spacing (i, j, k), optional velocity of shape (nz, ny, nx, 3)."""
    phi = np.ascontiguousarray(np.asarray(phi, dtype=np.float32))
    nz, ny, nx = phi.shape
    d = {"kind": 2, "c": tuple(float(o) for o in origin) + (float(spacing),), "vel": (0.0, 0.0, 0.0),
         "friction": float(friction), "sticky": bool(sticky), "dims": (nx, ny, nz), "phi": phi.reshape(-1)}
    if velocity is not None:
        d["grid_velocity"] = np.ascontiguousarray(np.asarray(velocity, dtype=np.float32)).reshape(-1)
    return d


def bowl_collider(centre=(0.0, 0.25, 0.0), radius=0.25, spacing=0.02, half_width=0.32, spin=0.0):
    """A spherical bowl sampled on a grid: phi = radius - |x - centre| (the snow is inside the sphere, the solid
    outside it), with an optional rigid spin about the vertical axis through the centre as sampled velocity."""
    n = int(round(2 * half_width / spacing)) + 1
    ax = np.arange(n) * spacing - half_width
    Z, Y, X = np.meshgrid(ax + centre[2], ax + centre[1], ax + centre[0], indexing="ij")
    phi = radius - np.sqrt((X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2)
    vel = None
    if spin:
        vel = np.stack([-spin * (Z - centre[2]), np.zeros_like(X), spin * (X - centre[0])], -1)
    origin = (centre[0] - half_width, centre[1] - half_width, centre[2] - half_width)
    return grid_collider(phi, origin, spacing, vel)


def sphere_points(n, radius, centre, seed):
    """n points uniform in a ball, rejection-sampled from the bounding cube."""
    rng = np.random.default_rng(seed)
    out = np.empty((0, 3))
    while out.shape[0] < n:
        c = rng.uniform(-radius, radius, size=(2 * n + 64, 3))
        c = c[(c * c).sum(1) < radius * radius]
        out = np.concatenate([out, c])
    return (out[:n] + np.asarray(centre)).astype(np.float32)


def snowball(n=10_000, radius=0.1, centre=(0.0, 0.3, 0.0), velocity=(0.0, -2.0, 0.0), h=0.01, dt=5e-4,
             steps=100, seed=1, friction=0.5):
    """C1 (CPU-runnable): a snowball dropped on the ground plane y = 0."""
    x = sphere_points(n, radius, centre, seed)
    mp = DENSITY * (4.0 / 3.0) * math.pi * radius ** 3 / n
    return {"name": f"snowball_{n}", "x": x, "v": np.tile(np.float32(velocity), (n, 1)),
            "m": np.full(n, mp, dtype=np.float32), "h": h, "dt": dt, "steps": steps, "snow": SNOW,
            "colliders": [plane((0.0, 1.0, 0.0, 0.0), friction)], "gravity": [GRAVITY]}


def two_snowballs(n_each=500_000, radius=0.15, h=0.005, dt=2.5e-4, steps=200, speed=3.0):
    """C2: two snowballs 0.6 m apart closing at 2 x 3 m/s, ground and gravity as C1."""
    a = sphere_points(n_each, radius, (-0.3, 0.3, 0.0), 2)
    b = sphere_points(n_each, radius, (0.3, 0.3, 0.0), 3)
    x = np.concatenate([a, b])
    v = np.concatenate([np.tile(np.float32((speed, 0, 0)), (n_each, 1)),
                        np.tile(np.float32((-speed, 0, 0)), (n_each, 1))])
    mp = DENSITY * (4.0 / 3.0) * math.pi * radius ** 3 / n_each
    return {"name": f"two_snowballs_{2 * n_each}", "x": x, "v": v, "m": np.full(2 * n_each, mp, dtype=np.float32),
            "h": h, "dt": dt, "steps": steps, "snow": SNOW, "colliders": [plane((0.0, 1.0, 0.0, 0.0), 0.5)],
            "gravity": [GRAVITY]}


def _slope_frame(angle_deg):
    """In-plane tangent (pointing up-slope) and normal of the plane phi = -sin(a) x + cos(a) y."""
    a = math.radians(angle_deg)
    t = np.array([math.cos(a), math.sin(a), 0.0])
    nrm = np.array([-math.sin(a), math.cos(a), 0.0])
    return t, nrm


def slab(cells=(171, 34, 86), h=None, angle_deg=30.0, seed_jitter=4, seed_e0=5, e0_range=(1e5, 2e5), dt=2.5e-4,
         steps=100, friction=0.5, per_particle_e0=True):
    """C3 (headline, 4,000,032 particles): a 1.0 x 0.2 x 0.5 m slab, 2x2x2 particles per lattice cell with
    U(+-0.25 cell) jitter, resting on a plane tilted by ``angle_deg`` about z, E0 log-uniform per particle."""
    nx, ny, nz = cells
    if h is None:
        h = 1.0 / nx
    # lattice of particle sites, 2 per cell per axis
    ix = (np.arange(2 * nx) + 0.5) * 0.5 * h
    iy = (np.arange(2 * ny) + 0.5) * 0.5 * h
    iz = (np.arange(2 * nz) + 0.5) * 0.5 * h
    U, W, Z = np.meshgrid(ix, iy, iz, indexing="ij")
    rng = np.random.default_rng(seed_jitter)
    n = U.size
    jit = rng.uniform(-0.25 * h, 0.25 * h, size=(n, 3))
    u = U.reshape(-1) + jit[:, 0]
    w = W.reshape(-1) + jit[:, 1] + 0.5 * h   # half a cell of clearance above the plane
    z = Z.reshape(-1) + jit[:, 2]
    t, nrm = _slope_frame(angle_deg)
    x = (u[:, None] * t[None, :] + w[:, None] * nrm[None, :]).astype(np.float64)
    x[:, 2] = z
    mp = DENSITY * h ** 3 / 8.0
    a = math.radians(angle_deg)
    scene = {"name": f"slab_{n}", "x": x.astype(np.float32), "v": np.zeros((n, 3), dtype=np.float32),
             "m": np.full(n, mp, dtype=np.float32), "h": float(h), "dt": dt, "steps": steps, "snow": SNOW,
             "colliders": [plane((-math.sin(a), math.cos(a), 0.0, 0.0), friction)], "gravity": [GRAVITY]}
    if per_particle_e0:
        rng2 = np.random.default_rng(seed_e0)
        e0 = np.exp(rng2.uniform(math.log(e0_range[0]), math.log(e0_range[1]), size=n))
        nu = SNOW[1]
        scene["mu0"] = (e0 / (2 * (1 + nu))).astype(np.float32)
        scene["lambda0"] = (e0 * nu / ((1 + nu) * (1 - 2 * nu))).astype(np.float32)
    return scene


def avalanche(size=(2.0, 0.5, 1.0), n_target=16_000_000, h=0.005, angle_deg=35.0, dt=2e-4, steps=100, seed=6,
              cyl=(0.5, 0.5, 0.1), spacing=None):
    """C5: a 2.0 x 0.5 x 1.0 m block on a 35 degree slope with a vertical cylinder collider (r = 0.1 m).

    The cylinder stands in the snowpack like a tree trunk. ``cyl = (u, z, radius)``: its axis is vertical through
    the point of the slope at along-slope distance u and depth z.  The particles within the cylinder (plus a
    quarter cell) are left out, so the snow around it is in contact from the first step."""
    L, H, D = size
    if spacing is None:
        spacing = (L * H * D / n_target) ** (1.0 / 3.0)
    nx, ny, nz = int(round(L / spacing)), int(round(H / spacing)), int(round(D / spacing))
    ix = (np.arange(nx) + 0.5) * spacing
    iy = (np.arange(ny) + 0.5) * spacing
    iz = (np.arange(nz) + 0.5) * spacing
    U, W, Z = np.meshgrid(ix, iy, iz, indexing="ij")
    rng = np.random.default_rng(seed)
    n = U.size
    jit = rng.uniform(-0.25 * spacing, 0.25 * spacing, size=(n, 3))
    t, nrm = _slope_frame(angle_deg)
    u = U.reshape(-1) + jit[:, 0]
    w = W.reshape(-1) + jit[:, 1] + 0.5 * h
    x = (u[:, None] * t[None, :] + w[:, None] * nrm[None, :])
    x[:, 2] = Z.reshape(-1) + jit[:, 2]
    mp = DENSITY * L * H * D / n
    a = math.radians(angle_deg)
    cx, cz, r = cyl[0] * t[0], cyl[1], cyl[2]
    keep = (x[:, 0] - cx) ** 2 + (x[:, 2] - cz) ** 2 >= (r + 0.25 * h) ** 2
    x = x[keep]
    n = x.shape[0]
    return {"name": f"avalanche_{n}", "x": x.astype(np.float32), "v": np.zeros((n, 3), dtype=np.float32),
            "m": np.full(n, mp, dtype=np.float32), "h": h, "dt": dt, "steps": steps, "snow": SNOW,
            "colliders": [plane((-math.sin(a), math.cos(a), 0.0, 0.0), 0.5), cylinder(cx, cz, r, 0.5)],
            "gravity": [GRAVITY]}


def avalanche_section(size=(0.4, 0.2, 0.3), cyl=(0.2, 0.15, 0.1)):
    """A section of C5 for the FP64 oracle: the avalanche's particle spacing, grid, slope, time step and cylinder
    (r = 0.1 m) standing in the snow, over a 0.4 x 0.2 x 0.3 m block (263,765 particles)."""
    spacing = (2.0 * 0.5 * 1.0 / 16_000_000) ** (1.0 / 3.0)
    return avalanche(size=size, spacing=spacing, cyl=cyl, seed=7)


def disc_2d(centre=(0.0, 0.0), radius=0.2, h=0.025, dt=2.5e-3, ground=-0.5, steps=100):
    """The reference's 2-D demo (main.cpp:71-105): a disc of snow on a 40 x 40 lattice at half a cell spacing in
    the z = 0 plane, density 400, over a sticky ground plane (friction 0.7) with gravity -9.8; dimension 2."""
    sp = 0.5 * h
    i, j = np.meshgrid(np.arange(40), np.arange(40), indexing="ij")
    xr = sp * (i.reshape(-1) - 20 + 0.5)
    yr = sp * (j.reshape(-1) - 20 + 0.5)
    keep = xr * xr + yr * yr < radius * radius
    x = np.stack([xr[keep] + centre[0], yr[keep] + centre[1], np.zeros(int(keep.sum()))], 1).astype(np.float32)
    n = x.shape[0]
    return {"name": f"disc_2d_{n}", "x": x, "v": np.zeros((n, 3), dtype=np.float32),
            "m": np.full(n, DENSITY * sp ** 3, dtype=np.float32), "h": h, "dt": dt, "steps": steps, "snow": SNOW,
            "colliders": [plane((0.0, 1.0, 0.0, -ground), 0.7, sticky=True)], "gravity": [(0.0, -9.8, 0.0)],
            "dimension": 2}


def lattice_block(n=4, spacing=0.05, origin=(0.0, 0.0, 0.0)):
    """n^3 lattice points at half-cell offsets (the TestSimClass.cpp:53-69 construction)."""
    g = (np.arange(n) + 0.5) * spacing
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    return (np.stack([X.reshape(-1), Y.reshape(-1), Z.reshape(-1)], 1) + np.asarray(origin)).astype(np.float32)
