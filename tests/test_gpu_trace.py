"""The iterate trace of a solve on the GPU (the reference's debug.dat, src/tests/TestGrid.cpp:398-447) — needs a
B200: the header is the body's grid, there is one iterate per solver iteration plus the first, and the last
iterate is the solved grid velocity v = x + vc (Grid.cpp:1014)."""
import numpy as np
import pytest

from tests.gpu_helpers import gpu_sim, impact_scene

pytestmark = pytest.mark.gpu


def test_iterate_trace_of_a_solve(tmp_path):
    from mpmsnow_b200 import build
    from mpmsnow_b200 import sim as M
    from mpmsnow_b200.trace import IterateTraceWriter, read_trace
    build.build()
    sc = impact_scene(n=1500)
    g = gpu_sim(sc)
    w = IterateTraceWriter(body=0)
    st = g.advance(sc["dt"], M.SquareMagnitudeTermination(60, 1e-5), w, stop_phase=2)
    path = str(tmp_path / "debug.dat")
    assert w.write(path, g) == st["iterations"][0] + 1
    t = read_trace(path)
    info = g.grid_info(0)
    assert t["h"] == np.float32(sc["h"])
    assert np.array_equal(t["n"], info["n"]) and np.array_equal(t["min"], info["min"])
    assert np.array_equal(t["masses"], g.grid_get(0, "masses"))
    assert len(t["iterates"]) == st["iterations"][0] + 1
    v = g.grid_get(0, "velocities").astype(np.float64)
    assert np.abs(t["iterates"][-1] - v).max() <= 1e-6 * max(1.0, np.abs(v).max())
