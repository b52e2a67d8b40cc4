"""Lower-dimensional simulations on the GPU (Sim's ``dimension`` = 2, Grid.cpp:180-207, 1112, 1144-1158) against
the FP64 oracle — needs a B200.  The scene is the reference's 2-D demo disc (main.cpp:71-105), started just above
its sticky ground plane."""
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


def _scene():
    return S.disc_2d(centre=(0.02, -0.285))


def test_2d_grid_and_cells(M):
    """The 2-D grid spans one node in z at 0; stencil cells in x and y equal the oracle's bit for bit; masses,
    velocities, forces, explicit momenta, collision flags (exact), collision velocities, rhs, preconditioner and
    guess against the FP64 oracle."""
    sc = _scene()
    g = gpu_sim(sc)
    o = oracle_sim(sc)
    o32 = oracle_sim(sc, prec=32)   # the reference's own arithmetic: grid geometry and cells bit for bit
    g.advance(sc["dt"], M.SquareMagnitudeTermination(60, 1e-5), stop_phase=1)
    o.advance(sc["dt"], 60, 1e-5, stop_phase=1)
    o32.advance(sc["dt"], 60, 1e-5, stop_phase=1)
    gi, oi = g.grid_info(0), o32.grid_info(0)
    assert np.array_equal(gi["n"], oi["n"]) and gi["n"][2] == 1
    assert np.array_equal(gi["min"].astype(np.float64), oi["min"])
    body, cell, _ = g.particle_cells()
    inds, base, _, _ = o32.grid_particles(0)
    assert np.array_equal(cell[inds, :2], base[:, :2] + 1) and np.all(cell[:, 2] == 0)
    flags = g.grid_get(0, "nodeCollided")
    assert np.array_equal(flags, o.grid_get(0, "nodeCollided")) and (flags == 0).sum() > 5
    assert rel_err(g.grid_get(0, "masses"), o.grid_get(0, "masses")) < 2e-6
    for name in ("forces", "explicitMomenta", "rhs", "diag", "x0"):
        assert rel_err(g.grid_get(0, name), o.grid_get(0, name)) < 2e-5, name
    assert rel_err(g.grid_get(0, "vc"), o.grid_get(0, "vc")) < 1e-6


def test_2d_steps_track_the_oracle(M):
    """40 full 2-D steps onto the sticky plane: positions within 1e-4 of the FP64 oracle (relative to the largest
    coordinate) and as close as the FP32 restatement's own deviation allows; z stays exactly 0."""
    sc = _scene()
    g = gpu_sim(sc)
    o = oracle_sim(sc, prec=64)
    o32 = oracle_sim(sc, prec=32)
    term = M.SquareMagnitudeTermination(60, 1e-5)
    for _ in range(40):
        gs = g.advance(sc["dt"], term)
        os_ = o.advance(sc["dt"], 60, 1e-5)
        o32.advance(sc["dt"], 60, 1e-5)
        assert gs["n_bodies"] == os_["n_bodies"]
    p = g.particleData().variable("p").astype(np.float64)
    po = o.get("p")
    scale = np.abs(po).max()
    e_gpu = np.abs(p - po).max() / scale
    e_32 = np.abs(o32.get("p") - po).max() / scale
    print(f"2-D disc after 40 steps: GPU {e_gpu:.3g}, FP32 restatement {e_32:.3g}")
    assert e_gpu < 1e-4 and e_gpu <= 10 * e_32 + 1e-6, (e_gpu, e_32)
    assert np.all(p[:, 2] == 0.0)
    assert np.abs(p - sc["x"]).max() > 10 * sc["h"] * 1e-3  # the disc moved


def test_2d_rejects_the_learned_warm_start(M):
    from mpmsnow_b200 import capi
    sc = _scene()
    g = gpu_sim(sc)
    ws = capi.MpmWarmStart()
    ws.density = 400.0
    assert capi.load().mpm_set_warm_start(g._h, ws) == 13  # MPM_ERR_UNSUPPORTED: the network is 3-D
