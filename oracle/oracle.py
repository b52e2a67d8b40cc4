"""CPU ORACLE — test infrastructure only.

ctypes binding of ``oracle/libmpm_oracle.so`` (the FP32 / FP64 restatement of the reference step in
``mpm_oracle.hpp``).  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU arm import this module,
and only as the checker / the timed CPU baseline; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libmpm_oracle.so")
_lib = None


class OrcCollider(C.Structure):
    _fields_ = [("kind", C.c_int), ("c", C.c_double * 4), ("vel", C.c_double * 3), ("friction", C.c_double),
                ("sticky", C.c_int), ("dims", C.c_int * 3), ("phi", C.POINTER(C.c_double)),
                ("gvel", C.POINTER(C.c_double))]


class OrcStepStats(C.Structure):
    _fields_ = [("nBodies", C.c_int), ("nBallistic", C.c_int), ("iterations", C.c_int * 64),
                ("bNorm2", C.c_double * 64), ("rNorm2", C.c_double * 64), ("exitReason", C.c_int * 64)]


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++, no GPU needed)."""
    src = [os.path.join(_HERE, f) for f in ("oracle_capi.cpp", "mpm_oracle.hpp")]
    if force or not os.path.exists(_LIB_PATH) or any(os.path.getmtime(s) > os.path.getmtime(_LIB_PATH) for s in src):
        subprocess.run(["make", "-s", "-C", _HERE, "-B" if force else "libmpm_oracle.so"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_int, C.c_long, dp, dp, C.c_void_p, C.c_void_p, C.c_double, dp, C.c_int,
                                 C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_char_p]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_advance.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int,
                                  C.POINTER(OrcStepStats), C.c_char_p]
        L.orc_num_particles.restype = C.c_long
        L.orc_num_particles.argtypes = [C.c_void_p]
        L.orc_get.argtypes = [C.c_void_p, C.c_char_p, dp]
        L.orc_set.argtypes = [C.c_void_p, C.c_char_p, dp]
        L.orc_bodies.argtypes = [C.c_void_p, ip, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_num_grids.argtypes = [C.c_void_p]
        L.orc_grid_info.argtypes = [C.c_void_p, C.c_int, dp, ip, dp, C.POINTER(C.c_int)]
        L.orc_grid_get.argtypes = [C.c_void_p, C.c_int, C.c_char_p, dp]
        L.orc_grid_apply.argtypes = [C.c_void_p, C.c_int, C.c_char_p, dp, dp, C.c_double]
        L.orc_grid_particles.argtypes = [C.c_void_p, C.c_int, ip, ip, ip, ip]
        L.orc_bspline.argtypes = [C.c_int, C.c_long, dp, dp, dp]
        L.orc_collide.argtypes = [C.c_int, C.c_int, C.c_void_p, dp, dp, dp, C.c_int]
        L.orc_snow_update.argtypes = [C.c_int, dp, C.c_long, dp, dp, dp, dp, dp, dp, dp, dp]
        L.orc_snow_eval.argtypes = [C.c_int, dp, dp, dp, dp, dp, C.c_double, C.c_double, C.c_double, dp, dp, dp, dp]
        L.orc_cr_dense.argtypes = [C.c_int, C.c_int, dp, dp, dp, C.c_int, C.c_double, C.c_void_p, C.c_void_p,
                                   C.POINTER(C.c_int)]
        L.orc_wall_seconds.restype = C.c_double
        L.orc_grid_create.restype = C.c_void_p
        L.orc_grid_create.argtypes = [C.c_int, C.c_long, dp, dp, dp, dp, dp, dp, C.c_int, C.c_double, dp, ip,
                                      C.c_long, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_int)]
        L.orc_grid_destroy.argtypes = [C.c_void_p]
        L.orc_grid_call.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_void_p, C.c_double, C.c_int, C.c_double]
        L.orc_grid_sinfo.argtypes = [C.c_void_p, dp, ip]
        L.orc_grid_sget.argtypes = [C.c_void_p, C.c_char_p, dp]
        L.orc_grid_sset.argtypes = [C.c_void_p, C.c_char_p, dp]
        L.orc_grid_sstats.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_stencil.argtypes = [C.c_int, C.c_double, dp, dp, dp, ip, dp, dp]
        _lib = L
    return _lib


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def colliders_array(colliders):
    """colliders: list of dicts {kind, c, vel, friction, sticky} (same meaning as the C-ABI's mpm_collider); a
    grid collider (kind 2) also has dims, phi and optionally grid_velocity.  The sample arrays are kept alive
    on the returned array (``_keep``) for as long as it is referenced."""
    arr = (OrcCollider * max(1, len(colliders)))()
    keep = []
    for i, c in enumerate(colliders):
        arr[i].kind = int(c.get("kind", 0))
        for k, v in enumerate(c["c"]):
            arr[i].c[k] = float(v)
        for k, v in enumerate(c.get("vel", (0.0, 0.0, 0.0))):
            arr[i].vel[k] = float(v)
        arr[i].friction = float(c.get("friction", 0.5))
        arr[i].sticky = int(bool(c.get("sticky", False)))
        if arr[i].kind == 2:
            for k in range(3):
                arr[i].dims[k] = int(c["dims"][k])
            phi = _f64(c["phi"]).reshape(-1)
            keep.append(phi)
            arr[i].phi = phi.ctypes.data_as(C.POINTER(C.c_double))
            if c.get("grid_velocity") is not None:
                gv = _f64(c["grid_velocity"]).reshape(-1)
                keep.append(gv)
                arr[i].gvel = gv.ctypes.data_as(C.POINTER(C.c_double))
    arr._keep = keep
    return arr


class OracleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


VAR_SHAPES = {"p": 3, "v": 3, "F": 9, "Fp": 9, "FinvTrans": 9, "R": 9, "Ginv": 9, "m": 1, "volume": 1, "J": 1,
              "mu": 1, "lambda": 1}


class OracleSim:
    """The restated ``MpmSim::Sim`` (Sim.cpp:17-203) at FP32 (prec=32) or FP64 (prec=64)."""

    def __init__(self, x, m, h, snow, colliders=(), gravity=((0.0, -9.81, 0.0),), prec=64, threads=1,
                 mu0=None, lambda0=None, dimension=3):
        L = lib()
        x = _f64(x).reshape(-1, 3)
        m = _f64(m).reshape(-1)
        self.n = x.shape[0]
        self.prec = prec
        colls = colliders_array(list(colliders))
        grav = _f64(np.array(gravity, dtype=np.float64).reshape(-1, 3)) if len(gravity) else np.zeros(3)
        st = C.c_int(0)
        msg = C.create_string_buffer(256)
        mu0p = _f64(mu0) if mu0 is not None else None
        la0p = _f64(lambda0) if lambda0 is not None else None
        self._keep = (x, m, mu0p, la0p, colls, grav)
        self.h = L.orc_create(prec, self.n, x, m, mu0p.ctypes.data if mu0p is not None else None,
                              la0p.ctypes.data if la0p is not None else None, float(h), _f64(snow),
                              len(colliders), C.cast(colls, C.c_void_p), len(gravity),
                              grav.ctypes.data if len(gravity) else None, int(threads), int(dimension), C.byref(st),
                              msg)
        if not self.h:
            raise OracleError(st.value, msg.value.decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def advance(self, dt, max_iters=60, tol=1e-5, stop_phase=0, batched=False):
        st = OrcStepStats()
        msg = C.create_string_buffer(256)
        rc = lib().orc_advance(self.h, float(dt), int(max_iters), float(tol), int(stop_phase), int(batched),
                               C.byref(st), msg)
        if rc != 0:
            raise OracleError(rc, msg.value.decode())
        nb = st.nBodies
        return {"n_bodies": nb, "n_ballistic": st.nBallistic,
                "iterations": [st.iterations[i] for i in range(min(nb, 64))],
                "bNorm2": [st.bNorm2[i] for i in range(min(nb, 64))],
                "rNorm2": [st.rNorm2[i] for i in range(min(nb, 64))],
                "exit": [st.exitReason[i] for i in range(min(nb, 64))]}

    def get(self, name):
        k = VAR_SHAPES[name]
        out = np.empty(self.n * k, dtype=np.float64)
        if lib().orc_get(self.h, name.encode(), out) != 0:
            raise KeyError(name)
        return out.reshape(self.n, k) if k > 1 else out

    def set(self, name, values):
        if lib().orc_set(self.h, name.encode(), _f64(values).reshape(-1)) != 0:
            raise KeyError(name)

    def bodies(self):
        out = np.empty(self.n, dtype=np.int32)
        nb, nbal = C.c_int(0), C.c_int(0)
        lib().orc_bodies(self.h, out, C.byref(nb), C.byref(nbal))
        return out, nb.value, nbal.value

    def num_grids(self):
        return lib().orc_num_grids(self.h)

    def grid_info(self, g):
        mn, fv = np.zeros(3), np.zeros(3)
        n3 = np.zeros(3, dtype=np.int32)
        npart = C.c_int(0)
        if lib().orc_grid_info(self.h, g, mn, n3, fv, C.byref(npart)) != 0:
            raise IndexError(g)
        return {"min": mn, "n": n3.copy(), "frame_velocity": fv, "n_particles": npart.value}

    def grid_get(self, g, name):
        info = self.grid_info(g)
        G = int(np.prod(info["n"]))
        k = 1 if name in ("masses", "nodeCollided") else 3
        out = np.zeros(G * k, dtype=np.float64)
        rc = lib().orc_grid_get(self.h, g, name.encode(), out)
        if rc != 0:
            raise KeyError(name)
        return out

    def grid_apply(self, g, op, vec, dt=0.0):
        vec = _f64(vec).reshape(-1)
        out = np.zeros_like(vec)
        rc = lib().orc_grid_apply(self.h, g, op.encode(), vec, out, float(dt))
        if rc != 0:
            raise RuntimeError(f"orc_grid_apply rc={rc}")
        return out

    def grid_particles(self, g):
        info = self.grid_info(g)
        n = info["n_particles"]
        inds = np.zeros(n, dtype=np.int32)
        base = np.zeros(3 * n, dtype=np.int32)
        vox = np.zeros(3 * n, dtype=np.int32)
        col = np.zeros(n, dtype=np.int32)
        lib().orc_grid_particles(self.h, g, inds, base, vox, col)
        return inds, base.reshape(n, 3), vox.reshape(n, 3), col


def bspline(x, prec=64):
    x = _f64(x).reshape(-1)
    w, dw = np.zeros_like(x), np.zeros_like(x)
    lib().orc_bspline(prec, x.size, x, w, dw)
    return w, dw


def collide(colliders, v, x, frame_velocity=(0, 0, 0), add_collision_velocity=False, prec=64):
    v = _f64(v).copy()
    arr = colliders_array(list(colliders))
    r = lib().orc_collide(prec, len(colliders), C.cast(arr, C.c_void_p), v, _f64(x), _f64(frame_velocity),
                          int(add_collision_velocity))
    return r, v


def snow_update(snow, F, Fp, prec=64):
    """SnowConstitutiveModel::updateParticleData on arrays of row-major 3x3 F, Fp (n x 9)."""
    F = _f64(F).reshape(-1).copy()
    Fp = _f64(Fp).reshape(-1).copy()
    n = F.size // 9
    FiT, R, Gi = np.zeros(9 * n), np.zeros(9 * n), np.zeros(9 * n)
    J, mu, la = np.zeros(n), np.zeros(n), np.zeros(n)
    rc = lib().orc_snow_update(prec, _f64(snow), n, F, Fp, FiT, R, Gi, J, mu, la)
    if rc != 0:
        raise OracleError(rc, "snow update failed")
    return {"F": F.reshape(n, 3, 3), "Fp": Fp.reshape(n, 3, 3), "FinvTrans": FiT.reshape(n, 3, 3),
            "R": R.reshape(n, 3, 3), "Ginv": Gi.reshape(n, 3, 3), "J": J, "mu": mu, "lambda": la}


def snow_eval(snow, F, R, FinvTrans, Ginv, J, mu, lam, dF, prec=64):
    e = np.zeros(1)
    a, b = np.zeros(9), np.zeros(9)
    rc = lib().orc_snow_eval(prec, _f64(snow), _f64(F).reshape(-1), _f64(R).reshape(-1), _f64(FinvTrans).reshape(-1),
                             _f64(Ginv).reshape(-1), float(J), float(mu), float(lam), _f64(dF).reshape(-1), e, a, b)
    if rc != 0:
        raise OracleError(rc, "snow eval failed")
    return float(e[0]), a.reshape(3, 3), b.reshape(3, 3)


def cr_dense(A, b, max_iters, tol=0.0, prec=32):
    A = _f64(A)
    n = A.shape[0]
    x = np.zeros(n)
    res = np.zeros((max_iters + 2) * n)
    dirs = np.zeros((max_iters + 2) * n)
    nrec = C.c_int(0)
    lib().orc_cr_dense(prec, n, A.reshape(-1), _f64(b), x, int(max_iters), float(tol), res.ctypes.data,
                       dirs.ctypes.data, C.byref(nrec))
    k = nrec.value
    return x, res[: k * n].reshape(k, n), dirs[: k * n].reshape(k, n)


class OracleGrid:
    """A restated ``MpmSim::Grid`` over caller particles, driven like the reference's TestGrid (friend access)."""

    def __init__(self, x, v, m, volume, F, snow, h, inds=None, frame_velocity=(0, 0, 0), colliders=(),
                 gravity=(), update_model=False, prec=64):
        x = _f64(x).reshape(-1, 3)
        n = x.shape[0]
        self.n = n
        self.prec = prec
        inds = np.arange(n, dtype=np.int32) if inds is None else np.ascontiguousarray(inds, dtype=np.int32)
        colls = colliders_array(list(colliders))
        grav = _f64(np.array(gravity, dtype=np.float64).reshape(-1, 3)) if len(gravity) else np.zeros(3)
        F = _f64(F).reshape(n, 9)
        st = C.c_int(0)
        self._keep = (x, inds, colls, grav)
        self.h = lib().orc_grid_create(prec, n, x.reshape(-1), _f64(v).reshape(-1), _f64(m).reshape(-1),
                                       _f64(volume).reshape(-1), F.reshape(-1), _f64(snow), int(update_model),
                                       float(h), _f64(frame_velocity), inds, inds.size, len(colliders),
                                       C.cast(colls, C.c_void_p), len(gravity),
                                       grav.ctypes.data if len(gravity) else None, C.byref(st))
        if not self.h:
            raise OracleError(st.value, "grid construction failed")
        mn = np.zeros(3)
        n3 = np.zeros(3, dtype=np.int32)
        lib().orc_grid_sinfo(self.h, mn, n3)
        self.min = mn
        self.dims = n3
        self.G = int(np.prod(n3))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_grid_destroy(self.h)
            self.h = None

    def call(self, op, vec=None, dt=0.0, max_iters=0, tol=0.0, out_size=None):
        inp = _f64(vec).reshape(-1) if vec is not None else None
        out = np.zeros(out_size if out_size is not None else 3 * self.G)
        rc = lib().orc_grid_call(self.h, op.encode(), inp.ctypes.data if inp is not None else None, out.ctypes.data,
                                 float(dt), int(max_iters), float(tol))
        if rc != 0:
            raise OracleError(rc, f"grid op {op} failed")
        return out

    def get(self, name):
        k = {"masses": self.G, "nodeCollided": self.G, "inds": self.n}.get(name)
        if k is None:
            k = 3 * self.G if name in ("velocities", "prevVelocities", "rhs", "explicitMomenta", "diag", "vc") \
                else self.n * VAR_SHAPES[name]
        out = np.zeros(k)
        if lib().orc_grid_sget(self.h, name.encode(), out) != 0:
            raise KeyError(name)
        return out

    def set(self, name, vals):
        if lib().orc_grid_sset(self.h, name.encode(), _f64(vals).reshape(-1)) != 0:
            raise KeyError(name)

    def stats(self):
        it, b, r = C.c_int(0), C.c_double(0), C.c_double(0)
        lib().orc_grid_sstats(self.h, C.byref(it), C.byref(b), C.byref(r))
        return it.value, b.value, r.value


def stencil(h, origin, p, prec=64):
    mn = np.zeros(3)
    base = np.zeros(3, dtype=np.int32)
    w = np.zeros(64)
    g = np.zeros(192)
    lib().orc_stencil(prec, float(h), _f64(origin), _f64(p), mn, base, w, g)
    return mn, base, w, g.reshape(64, 3)
