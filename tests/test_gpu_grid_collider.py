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


def bowl_scene():
    sc = S.snowball(n=3000, radius=0.06, centre=(0.05, 0.08, 0.0), velocity=(0.8, -1.0, 0.3), h=0.01)
    sc["colliders"] = [S.bowl_collider(spin=3.0)]
    return sc


def _term(M):
    return M.SquareMagnitudeTermination(60, 1e-5)


def test_grid_collider_phases(M):
    sc = bowl_scene()
    g = gpu_sim(sc)
    o32 = oracle_sim(sc, prec=32)
    o = oracle_sim(sc, prec=64)
    for _ in range(3):  # into contact with the bowl's wall
        g.advance(sc["dt"], _term(M))
        o.advance(sc["dt"], 60, 1e-5)
    # the three sims now hold slightly different states; restart the FP32 oracle from the GPU's
    for name in ("p", "v", "F", "Fp", "FinvTrans", "R", "Ginv", "J", "mu", "lambda", "volume"):
        vals = g.particleData().variable(name).astype(np.float64)
        o32.set(name, vals.reshape(vals.shape[0], -1) if vals.ndim > 1 else vals)
    g.advance(sc["dt"], _term(M), stop_phase=1)
    o32.advance(sc["dt"], 60, 1e-5, stop_phase=1)
    flags = g.grid_get(0, "nodeCollided")
    assert np.array_equal(flags, o32.grid_get(0, "nodeCollided"))
    assert (flags == 0).sum() > 20
    # the bowl's sampled spin at the collided nodes, relative to the body's frame
    assert rel_err(g.grid_get(0, "vc"), o32.grid_get(0, "vc")) < 1e-6
    for name in ("explicitMomenta", "rhs", "diag", "x0"):
        assert rel_err(g.grid_get(0, name), o32.grid_get(0, name)) < 2e-5, name


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
