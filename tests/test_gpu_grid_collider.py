"""The sampled signed-distance grid collider (the GPU form of the Houdini plugin's VDBCollisionObject,
houdiniPlugin/VDBCollisionObject.cpp:11-37) against the oracle's restatement — needs a B200.

Scene: a snowball dropped into a spinning spherical bowl given only as samples of phi and of the bowl's velocity
on a grid.  The collision flags are compared bit for bit with the FP32 oracle (the same separately rounded
trilinear arithmetic), the grid phases and trajectories with the FP64 oracle.
"""
import numpy as np
import pytest

from mpmsnow_b200 import scenes as S
from tests.gpu_helpers import gpu_sim, oracle_sim, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    from mpmsnow_b200 import build, sim
    build.build()
    return sim


def bowl_scene(spin=3.0):
    sc = S.snowball(n=3000, radius=0.06, centre=(0.05, 0.08, 0.0), velocity=(0.8, -1.0, 0.3), h=0.01)
    sc["colliders"] = [S.bowl_collider(spin=spin)]
    return sc


def _term(M):
    return M.SquareMagnitudeTermination(60, 1e-5)


def _into_contact(M, sc):
    """The GPU sim after 3 steps into the bowl's wall, and an FP32 oracle holding the same particle state."""
    g = gpu_sim(sc)
    for _ in range(3):
        g.advance(sc["dt"], _term(M))
    o32 = oracle_sim(sc, prec=32)
    for name in ("p", "v", "F", "Fp", "FinvTrans", "R", "Ginv", "J", "mu", "lambda", "volume"):
        vals = g.particleData().variable(name).astype(np.float64)
        o32.set(name, vals.reshape(vals.shape[0], -1) if vals.ndim > 1 else vals)
    g.advance(sc["dt"], _term(M), stop_phase=1)
    o32.advance(sc["dt"], 60, 1e-5, stop_phase=1)
    return g, o32


def test_grid_collider_phases(M):
    """A bowl at rest, against the FP32 oracle from the same particle state: the collision flags, then the
    collision velocities, explicit momenta, rhs, preconditioner and guess.  phi and its gradient are sampled with
    the same separately rounded arithmetic on both sides (the seeding test checks that sampling bit for bit).
    Velocities and momenta are compared in the world frame (frame velocity added back: the reference sums the
    body's centre-of-mass velocity in FP32 particle by particle, Sim.cpp:84-93, the GPU in FP64, so the comoving
    frames differ by that sum's rounding).  Where the snow slides along the curved wall, two thresholds of the
    explicit update's collide() are met within round-off: the normal velocity's sign (the node's flag) and the
    friction cone (vt against -friction vn: the node sticks or slides).  The splats' summation order decides those
    nodes: at most 1 % of the nodes flag differently, and of the collided nodes both flag alike at most 2 % take
    the other friction branch.  Nodes that neither side collided match to 2e-5 of the largest value."""
    g, o32 = _into_contact(M, bowl_scene(spin=0.0))
    fg, fo = g.grid_get(0, "nodeCollided"), o32.grid_get(0, "nodeCollided")
    assert (fg == 0).sum() > 20 and np.mean(fg != fo) < 0.01
    free = (fg == -1) & (fo == -1)
    hit = (fg == 0) & (fo == 0)
    fvg = g.grid_info(0)["frame_velocity"].astype(np.float64)
    fvo = o32.grid_info(0)["frame_velocity"].astype(np.float64)
    mg = g.grid_get(0, "masses").astype(np.float64)
    mo = o32.grid_get(0, "masses").astype(np.float64)
    for name in ("vc", "explicitMomenta", "rhs", "diag", "x0"):
        a = g.grid_get(0, name).astype(np.float64).reshape(-1, 3)
        b = o32.grid_get(0, name).astype(np.float64).reshape(-1, 3)
        if name in ("explicitMomenta", "rhs"):      # momenta: m (v - v_frame) + ...
            a, b = a + mg[:, None] * fvg[None, :], b + mo[:, None] * fvo[None, :]
        elif name == "vc":                          # the object's velocity relative to the frame, where collided
            a, b = a + (fg >= 0)[:, None] * fvg[None, :], b + (fo >= 0)[:, None] * fvo[None, :]
        elif name == "x0":                          # the uniform guess relative to the frame, on every node
            a, b = a + fvg[None, :], b + fvo[None, :]
        # velocities in the world frame of a bowl at rest are near 0: their scale is the frame's speed
        scale = max(np.abs(b).max(), np.abs(fvo).max() if name in ("vc", "x0") else 0.0)
        assert scale > 0, name
        d = np.abs(a - b).max(1)
        off = d[hit] >= 2e-5 * scale
        print(f"{name}: free nodes {d[free].max() / scale:.2e}, collided nodes off by more than 2e-5: "
              f"{off.sum()} of {hit.sum()}")
        assert d[free].max() < 2e-5 * scale, name
        assert off.mean() <= 0.02, name


def test_grid_collider_sampled_velocity(M):
    """A spinning bowl: the velocity a collided node takes from the bowl is its sampled (trilinear) velocity
    there; compared as vc + v_frame (the object's own velocity) on the nodes both sides flag, against the FP32
    oracle from the same particle state (flag differences as above)."""
    g, o32 = _into_contact(M, bowl_scene(spin=3.0))
    fg, fo = g.grid_get(0, "nodeCollided"), o32.grid_get(0, "nodeCollided")
    both = (fg == 0) & (fo == 0)
    assert both.sum() > 20 and np.mean(fg != fo) < 0.02
    vcg = g.grid_get(0, "vc").reshape(-1, 3)[both] + g.grid_info(0)["frame_velocity"].astype(np.float64)
    vco = o32.grid_get(0, "vc").reshape(-1, 3)[both] + o32.grid_info(0)["frame_velocity"]
    assert np.abs(vcg - vco).max() < 1e-6 * np.abs(vco).max()
    assert np.abs(vco).max() > 0.1   # the spin is in it


def test_grid_collider_steps_track_fp64(M):
    """10 steps in the spinning bowl: positions within 1e-4 of the FP64 oracle's and no particle left outside
    the bowl's surface by more than half a cell."""
    sc = bowl_scene()
    g = gpu_sim(sc)
    o = oracle_sim(sc, prec=64)
    for _ in range(10):
        gs = g.advance(sc["dt"], _term(M))
        os_ = o.advance(sc["dt"], 60, 1e-5)
        assert gs["n_bodies"] == os_["n_bodies"]
    p = g.particleData().variable("p").astype(np.float64)
    po = o.get("p")
    assert np.abs(p - po).max() / np.abs(po).max() < 1e-4
    r = np.linalg.norm(p - np.array([0.0, 0.25, 0.0]), axis=1)
    assert r.max() < 0.25 + 0.5 * sc["h"]


def test_set_collision_object_between_steps(M):
    """Sim.setCollisionObject (mpm_set_collider) replaces a collider: a sim built with the bowl and switched to a
    plane before its first step builds the same collision flags as the oracle built with that plane."""
    sc = bowl_scene()
    g = gpu_sim(sc)
    plane = S.plane((0.0, 1.0, 0.0, -0.05), 0.5)
    g.setCollisionObject(0, M.CollisionPlane(plane["c"], plane["friction"], plane["sticky"]))
    sc2 = dict(sc, colliders=[plane])
    o32 = oracle_sim(sc2, prec=32)
    g.advance(sc["dt"], _term(M), stop_phase=1)
    o32.advance(sc["dt"], 60, 1e-5, stop_phase=1)
    flags = g.grid_get(0, "nodeCollided")
    assert np.array_equal(flags, o32.grid_get(0, "nodeCollided")) and (flags == 0).sum() > 20
    with pytest.raises(M.MpmError):
        g.setCollisionObject(3, M.CollisionPlane(plane["c"]))
