"""The oracle's lower-dimensional grids (Sim's ``dimension``, Grid.cpp:180-207, 1112, 1144-1158) on the CPU.

The reference exercises dimension 2 only through its GL demo (main.cpp:71-105), so the 2-D mode is pinned against
the 3-D machinery the reference's own tests pin: for particles in the z = 0 plane, a 2-D grid node holds exactly
what the 3-D grid's column of nodes above it holds in sum (the B-spline weights along z sum to one), for masses
and momenta; the 2-D grid spans one node in z at 0; and a free-falling 2-D body follows gravity exactly.
"""
import numpy as np
import pytest

from mpmsnow_b200 import scenes as S


@pytest.fixture(scope="module")
def O():
    from oracle import oracle as O
    O.build()
    return O


def _sims(O, sc):
    args = (sc["x"], sc["m"], sc["h"], sc["snow"], sc["colliders"], sc["gravity"])
    return O.OracleSim(*args, prec=64, dimension=2), O.OracleSim(*args, prec=64, dimension=3)


def test_2d_grid_is_the_3d_grid_summed_over_z(O):
    sc = S.disc_2d()
    sc["v"] = np.random.default_rng(3).normal(size=sc["x"].shape).astype(np.float32)
    sc["v"][:, 2] = 0.0
    o2, o3 = _sims(O, sc)
    o2.set("v", sc["v"])
    o3.set("v", sc["v"])
    o2.advance(sc["dt"], 60, 1e-5, stop_phase=1)
    o3.advance(sc["dt"], 60, 1e-5, stop_phase=1)
    g2, g3 = o2.grid_info(0), o3.grid_info(0)
    n2, n3 = g2["n"], g3["n"]
    assert n2[2] == 1 and g2["min"][2] == 0.0
    assert np.array_equal(n2[:2], n3[:2]) and np.array_equal(g2["min"][:2], g3["min"][:2])
    m2 = o2.grid_get(0, "masses").reshape(n2[1], n2[0])
    m3 = o3.grid_get(0, "masses").reshape(n3[2], n3[1], n3[0])
    assert np.abs(m2 - m3.sum(0)).max() <= 1e-12 * m2.max()
    assert abs(m2.sum() - sc["m"].astype(np.float64).sum()) <= 1e-12 * m2.sum()
    # momenta about each grid's own frame velocity (the same centre-of-mass velocity)
    v2 = o2.grid_get(0, "prevVelocities").reshape(n2[1], n2[0], 3)
    v3 = o3.grid_get(0, "prevVelocities").reshape(n3[2], n3[1], n3[0], 3)
    p2 = m2[..., None] * v2
    p3 = (m3[..., None] * v3).sum(0)
    assert np.abs(p2 - p3).max() <= 1e-10 * np.abs(p2).max()
    assert np.all(v2[..., 2] == 0.0)


def test_2d_free_fall_follows_gravity(O):
    sc = S.disc_2d(centre=(0.0, 0.0))
    sc["colliders"] = []
    o2 = O.OracleSim(sc["x"], sc["m"], sc["h"], sc["snow"], sc["colliders"], sc["gravity"], prec=64, dimension=2)
    for _ in range(10):
        st = o2.advance(sc["dt"], 60, 1e-5)
        assert st["n_bodies"] == 1
    v = o2.get("v")
    assert np.abs(v[:, 1] + 9.8 * 10 * sc["dt"]).max() < 1e-9
    assert np.abs(v[:, 0]).max() < 1e-9 and np.all(v[:, 2] == 0.0)
    assert np.all(o2.get("p")[:, 2] == 0.0)


def test_dimension_out_of_range_is_rejected(O):
    sc = S.disc_2d()
    with pytest.raises(O.OracleError):
        O.OracleSim(sc["x"], sc["m"], sc["h"], sc["snow"], [], [], prec=64, dimension=4)
