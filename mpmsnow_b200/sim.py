"""Python mirror of the reference's ``MpmSim`` API over the CUDA C-ABI.

Same class names, constructor arguments and error behaviour as the reference's C++ classes (include/MpmSim/*.h),
so scripts and tests read like the reference's own.  Errors the reference throws as ``std::runtime_error``
raise :class:`mpmsnow_b200.capi.MpmError` carrying the same message.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional

import numpy as np

from . import capi
from .capi import MpmError


class CubicBsplineShapeFunction:
    """CubicBsplineShapeFunction (CubicBsplineShapeFunction.h:9-24); the only shape function of the path."""

    def supportRadius(self) -> int:
        return 2


class SnowConstitutiveModel:
    """SnowConstitutiveModel(youngsModulus, poissonRatio, hardening, compressiveStrength, tensileStrength)
    (SnowConstitutiveModel.h:13-18)."""

    def __init__(self, youngsModulus, poissonRatio, hardening, compressiveStrength, tensileStrength):
        self.youngsModulus = float(youngsModulus)
        self.poissonRatio = float(poissonRatio)
        self.hardening = float(hardening)
        self.compressiveStrength = float(compressiveStrength)
        self.tensileStrength = float(tensileStrength)


class CollisionObject:
    kind = 0

    def __init__(self, coeffs, coulombFriction=0.5, sticky=False):
        self.coeffs = [float(c) for c in coeffs]
        self.v = [0.0, 0.0, 0.0]
        self._friction = float(coulombFriction)
        self._sticky = bool(sticky)

    def coulombFriction(self):
        return self._friction

    def sticky(self):
        return self._sticky

    def setV(self, v):
        """CollisionPlane::setV (CollisionPlane.cpp:46-49)."""
        self.v = [float(a) for a in v]

    def as_struct(self) -> capi.MpmCollider:
        s = capi.MpmCollider()
        s.kind = self.kind
        for i in range(4):
            s.coeffs[i] = self.coeffs[i]
        for i in range(3):
            s.velocity[i] = self.v[i]
        s.friction = self._friction
        s.sticky = int(self._sticky)
        return s


class CollisionPlane(CollisionObject):
    """CollisionPlane(c, coulombFriction=0.5, sticky=False) (CollisionPlane.h:16): phi = c.xyz . x + c3."""
    kind = 0

    def setCoeffs(self, c):
        self.coeffs = [float(a) for a in c]


class CollisionCylinder(CollisionObject):
    """Solid vertical cylinder collider (no reference counterpart): axis along y through (cx, cz)."""
    kind = 1

    def __init__(self, cx, cz, radius, coulombFriction=0.5, sticky=False):
        super().__init__((cx, cz, radius, 0.0), coulombFriction, sticky)


class GridCollisionObject(CollisionObject):
    """A collider sampled on a dense grid, in place of the Houdini plugin's VDBCollisionObject (VDBCollisionObject.h:
    14-31; friction 0.5, not sticky by default as there): ``phi`` of shape (nz, ny, nx) sampled at
    ``origin + spacing * (i, j, k)``, and optionally a sampled velocity of shape (nz, ny, nx, 3).  phi and the
    velocity are trilinear between samples; outside the sampled box there is no collider."""
    kind = 2

    def __init__(self, phi, origin, spacing, velocity=None, coulombFriction=0.5, sticky=False):
        self.phi = np.ascontiguousarray(np.asarray(phi, dtype=np.float32))
        if self.phi.ndim != 3 or min(self.phi.shape) < 2:
            raise ValueError("phi must be a 3-D array with at least 2 samples per axis")
        self.velocity = None
        if velocity is not None:
            self.velocity = np.ascontiguousarray(np.asarray(velocity, dtype=np.float32).reshape(self.phi.shape + (3,)))
        super().__init__(tuple(float(o) for o in origin) + (float(spacing),), coulombFriction, sticky)

    def as_struct(self) -> capi.MpmCollider:
        s = super().as_struct()
        nz, ny, nx = self.phi.shape
        s.grid_dims[0], s.grid_dims[1], s.grid_dims[2] = nx, ny, nz
        s.grid_phi = self.phi.ctypes.data_as(C.POINTER(C.c_float))
        if self.velocity is not None:
            s.grid_velocity = self.velocity.ctypes.data_as(C.POINTER(C.c_float))
        return s


class CollisionObjectSet:
    """CollisionObject::CollisionObjectSet (CollisionObject.h:33-45): owns its objects."""

    def __init__(self):
        self._objects: List[CollisionObject] = []

    def add(self, o: CollisionObject):
        self._objects.append(o)

    def object(self, i):
        return self._objects[i]

    def numObjects(self):
        return len(self._objects)


class GravityField:
    """GravityField(gravity) (GravityField.h:13): force = gravity * m."""

    def __init__(self, gravity):
        self.gravity = [float(g) for g in gravity]


class ForceFieldSet:
    """ForceField::ForceFieldSet (ForceField.h:21-35)."""

    def __init__(self):
        self._fields: List[GravityField] = []

    def add(self, f: GravityField):
        self._fields.append(f)


class TerminationCriterion:
    def cancelled(self) -> bool:
        return False


class SquareMagnitudeTermination(TerminationCriterion):
    """SquareMagnitudeTermination(maxIters, tolError) (SquareMagnitudeTermination.h:14): stop when
    |r|^2 < tol^2 |b|^2 or after maxIters iterations."""

    def __init__(self, maxIters, tolError):
        self.maxIters = int(maxIters)
        self.tolError = float(tolError)


class LinearSolverDebug:
    """LinearSolver::Debug (LinearSolver.h:17-21): called with each body's solver iterate."""

    def __call__(self, x: np.ndarray):  # pragma: no cover - interface
        raise NotImplementedError


VAR_COMPONENTS = {"p": 3, "v": 3, "F": 9, "Fp": 9, "FinvTrans": 9, "R": 9, "Ginv": 9, "m": 1, "volume": 1, "J": 1,
                  "mu": 1, "lambda": 1, "mu0": 1, "lambda0": 1}


class MaterialPointData:
    """Host view of the device particle state (MaterialPointData.h:14-34).

    ``variable(name)`` returns a numpy array the caller may modify in place, as the reference returns a
    ``std::vector<T>&``.  As in the reference, the array lives as long as the Sim: ``Sim.advance`` refreshes every
    fetched array in place with the step's values, and before the step uploads those whose contents the caller
    changed (an array that was only read is not written back).  Matrices are (n, 3, 3).
    """

    def __init__(self, sim: "Sim"):
        self._sim = sim
        self._cache: Dict[str, np.ndarray] = {}
        self._shadow: Dict[str, np.ndarray] = {}

    def _download(self, name: str, out: np.ndarray) -> None:
        flat = out.reshape(-1)
        self._sim._check(capi.load().mpm_get_variable(self._sim._h, name.encode(), flat.ctypes.data, flat.size))
        self._shadow[name] = flat.view(np.uint32).copy()

    def variable(self, name: str) -> np.ndarray:
        if name in self._cache:
            return self._cache[name]
        k = VAR_COMPONENTS.get(name)
        n = self._sim.n
        if k is None:
            raise MpmError(11, f"Material point data has no variable named '{name}'")
        out = np.empty(n * k, dtype=np.float32)
        self._download(name, out)
        shaped = out.reshape(n, 3, 3) if k == 9 else (out.reshape(n, 3) if k == 3 else out)
        self._cache[name] = shaped
        return shaped

    def setVariable(self, name: str, values) -> None:
        k = VAR_COMPONENTS.get(name)
        if k is None:
            raise MpmError(11, f"Material point data has no variable named '{name}'")
        arr = np.ascontiguousarray(np.asarray(values, dtype=np.float32).reshape(-1))
        self._sim._check(capi.load().mpm_set_variable(self._sim._h, name.encode(), arr.ctypes.data, arr.size))
        if name in self._cache:
            self._cache[name].reshape(-1)[:] = arr
            self._shadow[name] = arr.view(np.uint32).copy()

    def variableNames(self):
        return [n for n in VAR_COMPONENTS if capi.load().mpm_variable_info(self._sim._h, n.encode(), None) == 0]

    def numVariables(self):
        return len(self.variableNames())

    def _flush(self):
        """Uploads the arrays whose contents differ (bit for bit) from the values last exchanged."""
        for name, arr in self._cache.items():
            flat = arr.reshape(-1)
            if np.array_equal(flat.view(np.uint32), self._shadow[name]):
                continue
            a = np.ascontiguousarray(flat, dtype=np.float32)
            self._sim._check(capi.load().mpm_set_variable(self._sim._h, name.encode(), a.ctypes.data, a.size))
            self._shadow[name] = a.view(np.uint32).copy()

    def _refresh(self):
        """The device state moved on: every fetched array is overwritten in place with the new values."""
        for name, arr in self._cache.items():
            self._download(name, arr)


class Sim:
    """Sim(x, masses, gridSize, shapeFunction, model, collisionObjects, forceFields, dimension=3)
    (Sim.h:32-41), stepped on CUDA device ``device``."""

    def __init__(self, x, masses, gridSize, shapeFunction, model: SnowConstitutiveModel,
                 collisionObjects: CollisionObjectSet, forceFields: ForceFieldSet, dimension: int = 3, device: int = 0):
        L = capi.load()
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float32).reshape(-1, 3))
        m = np.ascontiguousarray(np.asarray(masses, dtype=np.float32).reshape(-1))
        self.n = x.shape[0]
        self.gridSize = float(gridSize)
        colls = [o.as_struct() for o in collisionObjects._objects]
        self._coll_arr = (capi.MpmCollider * max(1, len(colls)))(*colls)
        grav = [g for f in forceFields._fields for g in f.gravity]
        self._grav_arr = (C.c_float * max(1, len(grav)))(*grav)
        d = capi.MpmSceneDesc()
        d.grid_size = float(gridSize)
        d.dimension = int(dimension)
        d.shape_function = 0 if isinstance(shapeFunction, CubicBsplineShapeFunction) else 1
        d.youngs_modulus = model.youngsModulus
        d.poisson_ratio = model.poissonRatio
        d.hardening = model.hardening
        d.compressive_strength = model.compressiveStrength
        d.tensile_strength = model.tensileStrength
        d.num_colliders = len(colls)
        d.colliders = C.cast(self._coll_arr, C.POINTER(capi.MpmCollider))
        d.num_gravity_fields = len(forceFields._fields)
        d.gravity = C.cast(self._grav_arr, C.POINTER(C.c_float))
        d.device = int(device)
        h = C.c_void_p()
        st = L.mpm_create(C.byref(d), self.n, x, m, C.byref(h))
        if st != 0:
            raise MpmError(st, L.mpm_status_string(st).decode())
        self._h = h
        self._data = MaterialPointData(self)
        self.last_stats: Optional[dict] = None

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            capi.load().mpm_destroy(h)
            self._h = None

    def _check(self, st):
        if st != 0:
            L = capi.load()
            msg = L.mpm_last_error(self._h).decode() if self._h else ""
            raise MpmError(st, msg or L.mpm_status_string(st).decode())

    def particleData(self) -> MaterialPointData:
        return self._data

    def setCollisionObject(self, index: int, obj: CollisionObject) -> None:
        """Replaces collider ``index`` between steps (mpm_set_collider): a moved plane (CollisionPlane::setCoeffs,
        setV) or a newly sampled grid collider."""
        s = obj.as_struct()
        self._check(capi.load().mpm_set_collider(self._h, int(index), C.byref(s)))

    def advance(self, timeStep, terminationCriterion: SquareMagnitudeTermination, d: Optional[LinearSolverDebug] = None,
                stop_phase: int = 0):
        """Sim::advance (Sim.cpp:57-134).  ``terminationCriterion.cancelled()`` is polled after the solve."""
        self._data._flush()
        L = capi.load()
        sp = capi.MpmSolveParams(int(terminationCriterion.maxIters), float(terminationCriterion.tolError))
        st = capi.MpmStepStats()
        cancel_cb = capi.CANCEL_FN(0)
        iter_cb = capi.ITERATE_FN(0)
        if type(terminationCriterion).cancelled is not TerminationCriterion.cancelled:
            cancel_cb = capi.CANCEL_FN(lambda ctx: int(bool(terminationCriterion.cancelled())))
        if d is not None:
            # a debug object with on_iterate(body, iteration, x) also learns which body and iteration each
            # iterate belongs to; otherwise it is called with the iterate alone, as LinearSolver::Debug is
            per_body = getattr(d, "on_iterate", None)

            def _it(ctx, body, iteration, xptr, count):
                x = np.ctypeslib.as_array(xptr, shape=(count,)).copy()
                if per_body is not None:
                    per_body(body, iteration, x)
                else:
                    d(x)
            iter_cb = capi.ITERATE_FN(_it)
        rc = L.mpm_step_ex(self._h, float(timeStep), C.byref(sp), int(stop_phase), cancel_cb, None, iter_cb, None,
                           C.byref(st))
        nb = st.num_bodies
        self.last_stats = {"n_bodies": nb, "n_ballistic": st.num_ballistic,
                           "iterations": [st.iterations[i] for i in range(min(nb, 64))],
                           "bNorm2": [st.b_norm2[i] for i in range(min(nb, 64))],
                           "rNorm2": [st.r_norm2[i] for i in range(min(nb, 64))],
                           "exit": [st.exit_reason[i] for i in range(min(nb, 64))],
                           "max_iterations": st.max_iterations_used, "total_iterations": st.total_iterations,
                           "fp64_svd_particles": st.fp64_svd_particles, "kernel_launches": st.kernel_launches}
        if rc != 1:  # the step ran (it may have failed or been cancelled): the fetched arrays follow the device
            try:
                self._data._refresh()
            except MpmError:
                if rc == 0:
                    raise
        if rc == 14:  # cancelled: the reference recomputes bodies and returns (Sim.cpp:107-111)
            return self.last_stats
        self._check(rc)
        return self.last_stats

    # --- inspection (parity tests) -------------------------------------------------------------------------
    def bodies(self):
        L = capi.load()
        out = np.empty(self.n, dtype=np.int32)
        nb, nbal = C.c_int(0), C.c_int(0)
        self._check(L.mpm_get_bodies(self._h, out.ctypes.data, C.byref(nb), C.byref(nbal)))
        return out, nb.value, nbal.value

    def grid_info(self, body):
        mn, fv = np.zeros(3, dtype=np.float32), np.zeros(3, dtype=np.float32)
        n3 = np.zeros(3, dtype=np.int32)
        npart = C.c_int(0)
        self._check(capi.load().mpm_debug_grid_info(self._h, int(body), mn, n3, fv, C.byref(npart)))
        return {"min": mn, "n": n3, "frame_velocity": fv, "n_particles": npart.value}

    def grid_get(self, body, name):
        info = self.grid_info(body)
        G = int(np.prod(info["n"]))
        k = 1 if name in ("masses", "nodeCollided") else 3
        out = np.zeros(G * k, dtype=np.float32)
        self._check(capi.load().mpm_debug_grid_get(self._h, int(body), name.encode(), out, out.size))
        return out

    def grid_apply(self, body, op, vec, dt):
        v = np.ascontiguousarray(np.asarray(vec, dtype=np.float32).reshape(-1))
        out = np.zeros_like(v)
        self._check(capi.load().mpm_debug_apply(self._h, int(body), op.encode(), v, out, v.size, float(dt)))
        return out

    def particle_cells(self):
        n = self.n
        body = np.zeros(n, dtype=np.int32)
        cell = np.zeros(3 * n, dtype=np.int32)
        vox = np.zeros(3 * n, dtype=np.int32)
        self._check(capi.load().mpm_debug_particle_cells(self._h, body, cell, vox))
        return body, cell.reshape(n, 3), vox.reshape(n, 3)


def profile_enable(sim: Sim, on: bool = True):
    """Per-phase device timing with CUDA events on the handle's stream (mpm_profile_enable)."""
    sim._check(capi.load().mpm_profile_enable(sim._h, int(on)))


def profile_read(sim: Sim):
    arr = (capi.MpmPhaseProfile * 32)()
    n = capi.load().mpm_profile_read(sim._h, arr, 32)
    if n < 0:
        sim._check(2)
    return [{"name": arr[i].name.decode(), "launches": arr[i].launches, "ms": arr[i].total_ms,
             "particles": arr[i].particles, "nodes": arr[i].nodes} for i in range(n)]


def stream_ptr(sim: Sim) -> int:
    return capi.load().mpm_get_stream(sim._h) or 0


def from_scene(scene, device=0) -> Sim:
    """Build a Sim from a ``mpmsnow_b200.scenes`` dict (positions, masses, velocities, colliders, fields)."""
    colls = CollisionObjectSet()
    for c in scene["colliders"]:
        if c["kind"] == 0:
            o = CollisionPlane(c["c"], c.get("friction", 0.5), c.get("sticky", False))
        elif c["kind"] == 2:
            nx, ny, nz = c["dims"]
            vel = c.get("grid_velocity")
            o = GridCollisionObject(np.asarray(c["phi"]).reshape(nz, ny, nx), c["c"][:3], c["c"][3],
                                    None if vel is None else np.asarray(vel).reshape(nz, ny, nx, 3),
                                    c.get("friction", 0.5), c.get("sticky", False))
        else:
            o = CollisionCylinder(c["c"][0], c["c"][1], c["c"][2], c.get("friction", 0.5), c.get("sticky", False))
        o.setV(c.get("vel", (0.0, 0.0, 0.0)))
        colls.add(o)
    fields = ForceFieldSet()
    for g in scene["gravity"]:
        fields.add(GravityField(g))
    sim = Sim(scene["x"], scene["m"], scene["h"], CubicBsplineShapeFunction(), SnowConstitutiveModel(*scene["snow"]),
              colls, fields, dimension=scene.get("dimension", 3), device=device)
    if "v" in scene and np.any(scene["v"]):
        sim.particleData().setVariable("v", scene["v"])
    if "mu0" in scene:
        sim.particleData().setVariable("mu0", scene["mu0"])
        sim.particleData().setVariable("lambda0", scene["lambda0"])
    return sim
