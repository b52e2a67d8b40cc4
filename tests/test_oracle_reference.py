"""Pins the CPU oracle against the reference's own unit tests (src/tests/*.cpp) — no GPU.

Each test restates one of the reference's test functions with the same construction and the same tolerances,
reading the known-answer values from tests/golden/reference_kats.json.  The reference's tests draw from the
unseeded rand() / Eigen::Random; here every draw is seeded.
"""
import json
import math
import os

import numpy as np
import pytest

from mpmsnow_b200 import scenes as S

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))


def rot(ax, ay, az):
    """AngleAxis(ax, X) * AngleAxis(ay, Y) * AngleAxis(az, Z) as used in TestSnowConstitutiveModel.cpp:45-47."""
    def Rx(a):
        return np.array([[1, 0, 0], [0, math.cos(a), -math.sin(a)], [0, math.sin(a), math.cos(a)]])

    def Ry(a):
        return np.array([[math.cos(a), 0, math.sin(a)], [0, 1, 0], [-math.sin(a), 0, math.cos(a)]])

    def Rz(a):
        return np.array([[math.cos(a), -math.sin(a), 0], [math.sin(a), math.cos(a), 0], [0, 0, 1]])
    return Rx(ax) @ Ry(ay) @ Rz(az)


@pytest.mark.parametrize("prec", [32, 64])
def test_shape_function(oracle, prec):
    """TestShapeFunction.cpp:17-157."""
    k = KATS["shape_function"]
    w, dw = oracle.bspline([2.0, -2.0], prec)
    assert w[0] == 0 and w[1] == 0 and dw[0] == 0 and dw[1] == 0
    dx = k["fd_step"]
    for i in range(21):
        x = np.float32(0.1 * i)
        wp, dwp = oracle.bspline([x, -x], prec)
        assert wp[0] == wp[1] and dwp[0] == -dwp[1]
        ws, _ = oracle.bspline([x - 4, x - 3, x - 2, x - 1, x, x + 1, x + 2], prec)
        assert abs(ws.sum() - 1) < k["partition_of_unity_tol"]
        # The finite-difference check (TestShapeFunction.cpp:40-41) runs on the FP64 instance: in FP32 the
        # cubic's Horner form cancels near |x| = 2 (w(1.9)), which puts the float quotient ~2.5e-4 off on SSE
        # hardware; the float instance is instead held to the FP64 derivative.
        wf, _ = oracle.bspline([float(x) + dx, float(x) - dx], 64)
        _, dw64 = oracle.bspline([x], 64)
        assert abs((wf[0] - wf[1]) / (2 * dx) - dw64[0]) < k["fd_derivative_tol"]
        assert abs(dwp[0] - dw64[0]) < 1e-6
    h = k["h"]
    mn, base, wts, grads = oracle.stencil(h, k["grid_origin"], k["particle"], prec)
    assert wts.size == k["nodes_visited"]
    assert abs(wts.sum() - 1) < (1e-6 if prec == 64 else 1e-6 * 4)
    rel = (np.asarray(k["particle"]) - mn) / h
    assert (base == np.floor(rel).astype(int) - 1).all()

    def ev(node):
        r = (node - np.asarray(k["particle"])) / h
        a, _ = oracle.bspline(r, 64)
        return a.prod()
    q = 0
    for kk in range(4):
        for j in range(4):
            for i in range(4):
                node = (base + np.array([i, j, kk])) * h + mn
                assert abs(ev(node) - wts[q]) < 1e-4
                for a in range(3):
                    e = np.zeros(3)
                    e[a] = dx
                    fd = -(ev(node + e) - ev(node - e)) / (2 * dx)
                    assert abs(grads[q, a] - fd) < 1e-3
                q += 1


def test_conjugate_residuals_dense(oracle):
    """TestConjugateResiduals.cpp:43-102: a 6x6 symmetric indefinite system solved in 6 iterations."""
    k = KATS["cr_dense"]
    n = k["n"]
    rng = np.random.default_rng(11)
    A = rng.uniform(-1, 1, (n, n))
    A = A + A.T
    b = rng.uniform(-1, 1, n)
    x, res, dirs = oracle.cr_dense(A, b, n, 0.0, prec=32)
    assert np.linalg.norm(A @ x - b) < k["residual_tol"]
    for i in range(1, n):
        assert (res[i] ** 2).sum() < (res[i - 1] ** 2).sum()
    for i in range(n):
        for j in range(n):
            if i != j:
                assert abs(res[i] @ (A @ res[j])) < k["orthogonality_tol"]
                assert abs((A @ dirs[i]) @ (A @ dirs[j])) < k["orthogonality_tol"]


@pytest.mark.parametrize("prec", [32, 64])
def test_snow_model(oracle, prec):
    """TestSnowConstitutiveModel.cpp:17-158."""
    kc = KATS["snow_clamp"]
    params = kc["params"]
    rng = np.random.default_rng(3)
    p = rng.uniform(-1, 1, (3, 3))
    p = p @ p
    m = rng.uniform(-1, 1, (3, 3))
    m = m @ m
    r = oracle.snow_update(params, m.reshape(1, 9), p.reshape(1, 9), prec)
    F, Fp = r["F"][0], r["Fp"][0]
    tol = 1e-4 if prec == 32 else 1e-10
    scale = max(1.0, np.abs(m @ p).max())
    assert np.linalg.norm(F @ Fp - m @ p) < tol * scale * 10
    assert np.linalg.norm(np.linalg.inv(F).T - r["FinvTrans"][0]) < 1e-4 * max(1, np.abs(r["FinvTrans"][0]).max())
    assert abs(r["J"][0] - abs(np.linalg.det(F))) < 1e-4 * max(1, abs(r["J"][0]))
    # stretch clamping
    Fc = np.diag(kc["F_diag_in"])
    r = oracle.snow_update(params, Fc.reshape(1, 9), np.eye(3).reshape(1, 9), prec)
    assert abs(r["F"][0][0, 0] - kc["F_diag_out"][0]) < kc["tol"]
    assert abs(r["F"][0][1, 1] - kc["F_diag_out"][1]) < kc["tol"]

    def state(Fm):
        s = oracle.snow_update(params, Fm.reshape(1, 9), np.eye(3).reshape(1, 9), prec)
        return s

    def ev(s, dF=np.zeros((3, 3))):
        return oracle.snow_eval(params, s["F"][0], s["R"][0], s["FinvTrans"][0], s["Ginv"][0], s["J"][0],
                                s["mu"][0], s["lambda"][0], dF, prec)
    # identity: zero energy and stress
    e, dEdF, _ = ev(state(np.eye(3)))
    assert e == 0 and (dEdF == 0).all()
    # pure rotation: zero energy and stress
    Rm = rot(0.25 * math.pi, 0.5 * math.pi, 0.33 * math.pi)
    e, dEdF, _ = ev(state(Rm))
    assert abs(e) < 1e-6 and np.linalg.norm(dEdF) < 1e-6
    # stress vs central finite differences of the energy
    F0 = np.diag([1.02, 0.95, 1.0]) @ Rm
    s0 = state(F0)
    _, dEdF, _ = ev(s0)
    delta = 0.01
    fd = np.zeros((3, 3))
    for i in range(3):
        for j in range(3):
            Fpl, Fmi = F0.copy(), F0.copy()
            Fpl[i, j] += delta
            Fmi[i, j] -= delta
            fd[i, j] = (ev(state(Fpl))[0] - ev(state(Fmi))[0]) / (2 * delta)
    assert np.abs(dEdF - fd).max() < 1e-5 * (1 if prec == 64 else 2)
    # dEdFDifferential vs forward finite differences of the stress
    dF = rng.uniform(-1, 1, (3, 3)) * 0.001
    _, _, diff = ev(s0, dF)
    _, dEdF1, _ = ev(state(F0 + dF))
    assert np.abs((dEdF1 - dEdF) - diff).max() < 1e-5


@pytest.mark.parametrize("prec", [32, 64])
def test_processing_partitions(oracle, prec):
    """TestGrid.cpp:21-122: lexicographic voxel order; every particle in one partition of the right colour."""
    h = 0.01
    x = S.lattice_block(16, 0.5 * h)
    n = x.shape[0]
    g = oracle.OracleGrid(x, np.zeros((n, 3)), np.ones(n), np.ones(n), np.tile(np.eye(3).reshape(1, 9), (n, 1)),
                          (1.4e5, 0.2, 0, 1e5, 1e5), h, prec=prec)
    sim = oracle.OracleSim(x, np.ones(n), h, (1.4e5, 0.2, 0, 1e5, 1e5), [], [], prec=prec)
    sim.advance(1e-4, 2, 0.0, stop_phase=1)
    inds, base, vox, col = sim.grid_particles(0)
    assert sorted(inds.tolist()) == list(range(n))
    for q in range(1, n):
        d = vox[q] - vox[q - 1]
        nz = np.nonzero(d)[0]
        if nz.size:
            assert d[nz[0]] > 0
    assert (col == (vox[:, 0] & 1) + 2 * (vox[:, 1] & 1) + 4 * (vox[:, 2] & 1)).all()
    expect = np.floor(x.astype(np.float64 if prec == 64 else np.float32) / np.float32(4 * h)).astype(int)
    assert (vox == expect[inds]).all()
    del g


@pytest.mark.parametrize("prec", [32, 64])
def test_splatting_conservation(oracle, prec):
    """TestGrid.cpp:124-213: mass and momentum are conserved by P2G."""
    rng = np.random.default_rng(5)
    x = np.concatenate([np.zeros((1, 3)), rng.uniform(0, 1, (500, 3))])
    v = np.array([1.0, 0, 0]) + rng.uniform(-1, 1, (501, 3))
    n = x.shape[0]
    m = np.ones(n)
    g = oracle.OracleGrid(x, v, m, np.ones(n), np.tile(np.eye(3).reshape(1, 9), (n, 1)), (1.4e5, 0.2, 0, 1e5, 1e5),
                          0.01, prec=prec)
    gm = g.get("masses")
    gv = g.get("velocities").reshape(-1, 3)
    assert abs(m.sum() - gm.sum()) / m.sum() < 1e-4
    pm = (m[:, None] * v).sum(0)
    gmom = (gm[:, None] * gv).sum(0)
    assert np.linalg.norm(pm - gmom) / np.linalg.norm(pm) < 1e-4


@pytest.mark.parametrize("prec", [32, 64])
def test_deformation_gradient_update(oracle, prec):
    """TestGrid.cpp:216-278: a linear velocity field gives F = diag(1 + i dt, 1 - i dt, 1 + i dt/2)."""
    k = KATS["deformation_gradient"]
    g1 = np.arange(10) / 9.0 - 0.5
    X, Y, Z = np.meshgrid(g1, g1, g1, indexing="ij")
    pts = np.stack([X.reshape(-1), Y.reshape(-1), Z.reshape(-1)], 1)
    x = np.concatenate([np.zeros((1, 3)), pts]).astype(np.float32).astype(np.float64)
    v = np.stack([x[:, 0], -x[:, 1], 0.5 * x[:, 2]], 1)
    v[0] = 0
    n = x.shape[0]
    F = np.tile(np.eye(3).reshape(1, 9), (n, 1))
    for i in range(1, k["steps"] + 1):
        g = oracle.OracleGrid(x, v, np.ones(n), np.ones(n), F, (1.4e5, 0.2, 0, 1e5, 1e5), k["h"], prec=prec)
        g.call("updateF", dt=k["dt"], out_size=1)
        F = g.get("F").reshape(n, 9)
        x = x + v * k["dt"]
        assert abs(F[0, 0] - (1 + 0.01 * i)) < k["tol"]
        assert abs(F[0, 4] - (1 - 0.01 * i)) < k["tol"]
        assert abs(F[0, 8] - (1 + 0.005 * i)) < k["tol"]


def test_forces_and_differentials(oracle):
    """TestGrid.cpp:281-396: zero force at equilibrium; node force = -dE/dx; force differential vs FD.

    The reference's force differential (Grid.cpp:594-607) differentiates P(F) but not the F^T factor of the
    force -vol P F^T grad(w), so its agreement with finite differences is O(|P| / E): 1-3 % over random
    0.01 perturbations of F (the reference's own comment, TestGrid.cpp:388-389, reports ~2.5 %).  The draw
    here is seeded.
    """
    k = KATS["forces"]
    prec = 64
    Rm = rot(0.25 * math.pi, 0.5 * math.pi, 0.33 * math.pi)
    params = (1.4e3, 0.2, 0.0, 1e5, 1e5)
    x = np.zeros((1, 3))
    mk = lambda F: oracle.OracleGrid(x, np.zeros((1, 3)), np.ones(1), [0.5], F.reshape(1, 9), params, 1.0,
                                     update_model=True, prec=prec)
    g = mk(Rm)
    f = g.call("forces")
    assert np.abs(f).max() < k["equilibrium_tol"]
    rng = np.random.default_rng(1)
    Forig = Rm + 0.01 * rng.uniform(-1, 1, (3, 3))
    g = mk(Forig)
    f = g.call("forces")
    dx = 0.01
    checked = 0
    for i in range(f.size):
        if f[i] == 0:
            continue
        vel = np.zeros(f.size)
        vel[i] = dx
        df = g.call("DF", vel)
        res = []
        for sgn in (1, -1):
            g2 = mk(Forig)
            v2 = np.zeros(f.size)
            v2[i] = sgn * dx
            g2.call("setVelocities", v2)
            g2.call("updateF", dt=1.0)
            g2.call("model", out_size=1)
            e = g2.call("energy", out_size=1)[0] * 0.5
            fp = g2.call("forces")
            res.append((e, fp))
        (ep, fpl), (em, fmi) = res
        assert abs((f[i] + (ep - em) / (2 * dx)) / f[i]) < k["force_fd_rel"]
        assert np.linalg.norm(0.5 * (fpl - fmi) - df) / np.linalg.norm(df) < k["differential_fd_rel"]
        checked += 1
    assert checked >= 64


@pytest.mark.parametrize("prec", [32, 64])
def test_dfidxi_is_operator_diagonal(oracle, prec):
    """TestGrid.cpp:806-852: dForceidXi equals the diagonal of calculateForceDifferentials."""
    rng = np.random.default_rng(13)
    F = np.eye(3) + 0.1 * rng.uniform(-1, 1, (3, 3))
    g = oracle.OracleGrid(np.zeros((1, 3)), np.zeros((1, 3)), np.ones(1), [0.5], F.reshape(1, 9),
                          (1.4e5, 0.2, 0.0, 1e5, 1e5), 1.0, update_model=True, prec=prec)
    diag = g.call("dFidXi")
    for i in range(diag.size):
        e = np.zeros(diag.size)
        e[i] = 1
        assert abs(g.call("DF", e)[i] - diag[i]) < KATS["dfidxi"]["tol"]


@pytest.mark.parametrize("prec", [32, 64])
def test_implicit_update(oracle, prec):
    """TestGrid.cpp:456-708: no velocity into the colliders; the solve satisfies
    P(M(v - vc) - dt^2 DF v) = p* (the explicit momenta plus the collider term)."""
    k = KATS["implicit_update"]
    h = k["h"]
    rng = np.random.default_rng(17)
    distortion = rng.uniform(-1, 1, (3, 3)) * 0.001
    pts = []
    for i in range(4):
        for j in range(4):
            for kk in range(4):
                pts.append(((i - 0.5) * h, (j - 0.5) * h, (kk - 0.5) * h))
    x = np.array(pts, dtype=np.float32).astype(np.float64)
    n = x.shape[0]
    v = 0.1 + 0.01 * np.sin(2 * x)
    F = np.stack([(np.eye(3) + distortion * math.cos(2 * p[0])).reshape(9) for p in x])
    colls = [S.plane((-1, -1, -1, 1), vel=(-0.1, -0.2, -0.3)), S.plane((-1, 0, 0, 1.5), vel=(-0.2, -0.1, -0.4))]
    params = (1.4e5, 0.2, 0.0, 1e5, 1e5)
    g = oracle.OracleGrid(x, v, np.ones(n), np.ones(n), F, params, h, colliders=colls, prec=prec)
    g.call("volumes", out_size=1)
    dt = k["dt"]
    g.call("solve", dt=dt, max_iters=k["iters"], tol=0.0, out_size=1)
    vel = g.get("velocities").reshape(-1, 3)
    flags = g.get("nodeCollided").astype(int)
    vc = g.get("vc").reshape(-1, 3)
    nx, ny, nz = g.dims
    assert (flags >= 0).any() and (flags == -1).any()
    for idx in np.nonzero(flags >= 0)[0]:
        c = np.array(colls[flags[idx]]["c"][:3], dtype=np.float64)
        nrm = c / np.linalg.norm(c)
        assert np.allclose(vc[idx], colls[flags[idx]]["vel"], atol=1e-6)
        assert abs(nrm @ (vel[idx] - vc[idx])) < k["normal_velocity_tol"]
    for idx in np.nonzero(flags == -2)[0]:
        assert np.linalg.norm(vel[idx]) == 0 and np.linalg.norm(vc[idx]) == 0
    df = g.call("DF", vel.reshape(-1)).reshape(-1, 3)
    masses = g.get("masses")
    lhs = masses[:, None] * (vel - vc) - df * dt * dt
    for idx in range(lhs.shape[0]):
        if flags[idx] >= 0:
            c = np.array(colls[flags[idx]]["c"][:3], dtype=np.float64)
            nrm = c / np.linalg.norm(c)
            lhs[idx] -= (nrm @ lhs[idx]) * nrm
        elif flags[idx] == -2:
            lhs[idx] = 0
    pstar = g.get("explicitMomenta").reshape(-1, 3)
    err = np.linalg.norm(lhs - pstar, axis=1).max()
    assert err < (k["equation_max_norm_tol"] if prec == 64 else 2e-5)


def test_sim_initialization(oracle):
    """TestSimClass.cpp:45-118: two 4096-particle bodies and 4096 ballistic particles."""
    k = KATS["sim_init"]
    h = k["h"]
    a = S.lattice_block(16, 0.5 * h)
    b = a + np.float32([6, 0, 0])
    g = np.arange(16) * 1.1 * h
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    c = np.stack([X.reshape(-1) + 20, Y.reshape(-1), Z.reshape(-1)], 1).astype(np.float32)
    x = np.empty((2 * a.shape[0], 3), dtype=np.float32)
    x[0::2], x[1::2] = a, b
    x = np.concatenate([x, c])
    sim = oracle.OracleSim(x, np.ones(x.shape[0]), h, (1.4e5, 0.2, 0.0, 1e5, 1e5), [], [], prec=32)
    body, nb, nbal = sim.bodies()
    assert nb == k["n_bodies"] and nbal == k["n_ballistic"]
    assert [(body == i).sum() for i in range(nb)] == k["body_sizes"]
    with pytest.raises(KeyError):
        sim.get("Fiddlesticks")


@pytest.mark.parametrize("prec", [32, 64])
def test_sim_advance_gravity(oracle, prec):
    """TestSimClass.cpp:120-190: gravity +1 for 3 x 0.01 s gives a mean velocity of 0.03."""
    k = KATS["sim_advance"]
    h = k["h"]
    a = S.lattice_block(4, 0.5 * h)
    b = a + np.float32([6, 0, 0])
    g = np.arange(4) * 1.1 * h
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    c = np.stack([X.reshape(-1) + 20, Y.reshape(-1), Z.reshape(-1)], 1).astype(np.float32)
    x = np.empty((2 * a.shape[0], 3), dtype=np.float32)
    x[0::2], x[1::2] = a, b
    x = np.concatenate([x, c])
    sim = oracle.OracleSim(x, np.ones(x.shape[0]), h, k["params"], [], [k["gravity"]], prec=prec)
    for _ in range(k["steps"]):
        sim.advance(k["dt"], k["max_iters"], k["tol"])
    v = sim.get("v").mean(0)
    assert abs(v[0]) < k["vxz_tol"] and abs(v[2]) < k["vxz_tol"]
    assert abs(v[1] - k["mean_vy"]) < k["vy_tol"]


def test_batched_schedule_matches_reference_schedule(oracle):
    """The CUDA path builds and solves every body's grid before any G2P and runs plasticity once per step;
    on a two-body scene that schedule agrees with the reference's body-by-body schedule to round-off."""
    k = 2500
    a = S.sphere_points(k, 0.05, (-0.12, 0.08, 0.0), 21)
    b = S.sphere_points(k, 0.05, (0.12, 0.07, 0.0), 22)
    x = np.concatenate([a, b])
    n = x.shape[0]
    v = np.concatenate([np.tile([1.0, -1.0, 0.0], (k, 1)), np.tile([-1.0, -0.5, 0.0], (k, 1))])
    m = np.full(n, 400 * 4 / 3 * math.pi * 0.05 ** 3 / k)
    out = []
    for batched in (False, True):
        sim = oracle.OracleSim(x, m, 0.01, S.SNOW, [S.plane((0, 1, 0, 0))], [S.GRAVITY], prec=64)
        sim.set("v", v)
        for _ in range(4):
            st = sim.advance(5e-4, 60, 1e-5, batched=batched)
        body, nb, _ = sim.bodies()
        assert nb >= 2 and sorted(np.bincount(body[body >= 0]))[-2] > 0.95 * k
        out.append(sim.get("p"))
    assert np.abs(out[0] - out[1]).max() < 1e-9
