"""Iterate trace in the reference's ``debug.dat`` format: one body's grid and every conjugate-residual iterate of
its solve, for offline inspection.  The reference writes it from a test-side ``LinearSolver::Debug``
(src/tests/TestGrid.cpp:398-447) and its viewer reads it (src/viewer.cpp:54-78); the viewer itself is an OpenGL
program and is not part of this package.

Layout, native byte order, 4-byte fields:

    float h                grid spacing
    float min[3]           grid origin
    int   n[3]             nodes per axis; N = n0 n1 n2 nodes in the order i + n0 (j + n1 k)
    float masses[N]
    float explicit[3N]     explicit momenta / mass (0 on massless nodes) + collision velocities vc
    float iterate[3N]      x + vc after each solver iteration, one block per iteration to the end of the file

Usage::

    w = IterateTraceWriter(body=0)
    sim.advance(dt, termination, w)
    w.write("debug.dat", sim)
"""
from __future__ import annotations

import struct

import numpy as np

from .sim import LinearSolverDebug


class IterateTraceWriter(LinearSolverDebug):
    """Records the iterates of one body's solve during ``Sim.advance`` and writes them with the body's grid."""

    def __init__(self, body: int = 0):
        self.body = int(body)
        self.iterates = []

    def __call__(self, x):
        """LinearSolver::Debug::operator() (LinearSolver.h:17-21), for callers that pass iterates without a body."""
        self.iterates.append(np.array(x, dtype=np.float32))

    def on_iterate(self, body, iteration, x):
        """Called by ``Sim.advance`` with every body's iterate; keeps this writer's body."""
        if int(body) == self.body:
            self.iterates.append(np.array(x, dtype=np.float32))

    def reset(self):
        self.iterates = []

    def write(self, path, sim):
        """Write the trace of the last ``advance``: the header from the body's grid (still held by ``sim`` until
        its next step) and the recorded iterates.  Returns the number of iterates written."""
        info = sim.grid_info(self.body)
        n = [int(v) for v in info["n"]]
        count = n[0] * n[1] * n[2]
        masses = np.asarray(sim.grid_get(self.body, "masses"), dtype=np.float32).reshape(count)
        momenta = np.asarray(sim.grid_get(self.body, "explicitMomenta"), dtype=np.float32).reshape(count, 3)
        vc = np.asarray(sim.grid_get(self.body, "vc"), dtype=np.float32).reshape(3 * count)
        with np.errstate(divide="ignore", invalid="ignore"):
            vel = np.where(masses[:, None] != 0, momenta / masses[:, None], np.float32(0)).astype(np.float32)
        explicit = (vel.reshape(-1) + vc).astype(np.float32)
        with open(path, "wb") as f:
            f.write(struct.pack("=f3f3i", float(sim.gridSize), *[float(v) for v in info["min"]], *n))
            f.write(masses.tobytes())
            f.write(explicit.tobytes())
            for x in self.iterates:
                if x.size != 3 * count:
                    raise ValueError(f"iterate of {x.size} floats for a grid of {count} nodes")
                f.write((x + vc).astype(np.float32).tobytes())
        return len(self.iterates)


def read_trace(path):
    """Parse a trace the way the reference's viewer does (header, masses, explicit velocities, then iterate
    blocks to the end of the file); only complete blocks are returned."""
    with open(path, "rb") as f:
        data = f.read()
    h, mx, my, mz, nx, ny, nz = struct.unpack_from("=f3f3i", data, 0)
    count = nx * ny * nz
    off = struct.calcsize("=f3f3i")
    masses = np.frombuffer(data, dtype=np.float32, count=count, offset=off)
    off += 4 * count
    explicit = np.frombuffer(data, dtype=np.float32, count=3 * count, offset=off)
    off += 12 * count
    block = 12 * count
    iterates = [np.frombuffer(data, dtype=np.float32, count=3 * count, offset=off + k * block)
                for k in range((len(data) - off) // block)] if block else []
    return {"h": h, "min": np.array([mx, my, mz], dtype=np.float32), "n": np.array([nx, ny, nz]),
            "masses": masses, "explicit": explicit, "iterates": iterates}
