"""The iterate trace writer (mpmsnow_b200/trace.py) on the CPU, with a stand-in for the simulator's grid
accessors: the byte layout the reference's viewer reads (src/viewer.cpp:54-78), the body filter and the
size check."""
import struct

import numpy as np
import pytest

from mpmsnow_b200.trace import IterateTraceWriter, read_trace


class _Grid:
    """The three accessors the writer uses, over a 3 x 2 x 2 grid."""

    def __init__(self):
        rng = np.random.default_rng(0)
        self.gridSize = 0.01
        self.n = np.array([3, 2, 2], dtype=np.int32)
        self.count = 12
        self.arrays = {"masses": np.where(rng.uniform(size=12) > 0.3, rng.uniform(0.1, 1.0, 12), 0.0).astype(np.float32),
                       "explicitMomenta": rng.normal(size=36).astype(np.float32),
                       "vc": rng.normal(size=36).astype(np.float32)}

    def grid_info(self, body):
        return {"min": np.array([-0.02, 0.0, 0.03], dtype=np.float32), "n": self.n,
                "frame_velocity": np.zeros(3, dtype=np.float32), "n_particles": 10}

    def grid_get(self, body, name):
        return self.arrays[name]


def test_layout_round_trip(tmp_path):
    g = _Grid()
    w = IterateTraceWriter(body=1)
    its = [np.random.default_rng(k).normal(size=36).astype(np.float32) for k in range(3)]
    w.on_iterate(0, 0, np.zeros(36 * 2, dtype=np.float32))     # another body's grid: ignored
    for k, x in enumerate(its):
        w.on_iterate(1, k, x)
    path = str(tmp_path / "debug.dat")
    assert w.write(path, g) == 3
    raw = open(path, "rb").read()
    head = struct.pack("=f3f3i", 0.01, -0.02, 0.0, 0.03, 3, 2, 2)
    assert raw[:len(head)] == head
    assert len(raw) == len(head) + 4 * 12 + 12 * 12 * (1 + 3)
    t = read_trace(path)
    assert t["h"] == np.float32(0.01) and list(t["n"]) == [3, 2, 2]
    m = g.arrays["masses"]
    assert np.array_equal(t["masses"], m)
    vel = np.zeros((12, 3), dtype=np.float32)
    nz = m != 0
    vel[nz] = g.arrays["explicitMomenta"].reshape(12, 3)[nz] / m[nz, None]
    assert np.array_equal(t["explicit"], vel.reshape(-1) + g.arrays["vc"])
    assert len(t["iterates"]) == 3
    for got, x in zip(t["iterates"], its):
        assert np.array_equal(got, x + g.arrays["vc"])


def test_plain_debug_call_and_size_check(tmp_path):
    g = _Grid()
    w = IterateTraceWriter()
    w(np.ones(36, dtype=np.float32))
    assert w.write(str(tmp_path / "a.dat"), g) == 1
    w.reset()
    w(np.ones(35, dtype=np.float32))
    with pytest.raises(ValueError):
        w.write(str(tmp_path / "b.dat"), g)
