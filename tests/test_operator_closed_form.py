"""The closed form of the particle's linearised force map M that the force pass stores, against the oracle's
dEdFDifferential (SnowConstitutiveModel.cpp:218-287), in float64 on the CPU.

fm = vol dEdFDifferential(G F) F^T is linear in the gathered velocity gradient G, so fm = M vec(G) with
vec(G)[3a + d] = G[a][d].  The force pass writes M's upper triangle from

    M[(a,c),(b,d)] = vol [2 mu [a = b] (F F^T)_dc + lam J (2J - 1) C_ac C_bd - lam J (J - 1) C_ad C_bc
                          - 2 mu sum_kl (G^-1)_kl (Q_k)_ac (Q_l)_bd],

C = F^-T F^T and Q_k = R E_k F^T for E_0 = e0 e1^T - e1 e0^T, E_1 = e0 e2^T - e2 e0^T, E_2 = e1 e2^T - e2 e1^T.
Column (b, d) of M is the oracle's differential at G = e_b e_d^T; the states are the oracle's own plasticity
updates and states whose F was replaced afterwards (F set by a caller: R, F^-T, G^-1 and J from before).
"""
import numpy as np

from oracle import oracle

SNOW = (1.4e5, 0.2, 10.0, 2.5e-2, 7.5e-3)


def _closed_form(F, R, FiT, Gi, J, mu, lam, vol):
    """The force pass's formula, entry by entry, for every (row, column)."""
    B = F @ F.T
    C = FiT @ F.T
    q = []
    for i, j in ((0, 1), (0, 2), (1, 2)):
        E = np.zeros((3, 3))
        E[i, j], E[j, i] = 1.0, -1.0
        q.append(R @ E @ F.T)
    M = np.zeros((9, 9))
    for a in range(3):
        for c in range(3):
            for b in range(3):
                for d in range(3):
                    v = 2 * mu * B[d, c] if a == b else 0.0
                    v += lam * J * (2 * J - 1) * C[a, c] * C[b, d] - lam * J * (J - 1) * C[a, d] * C[b, c]
                    v -= 2 * mu * sum(Gi[k, l] * q[k][a, c] * q[l][b, d] for k in range(3) for l in range(3))
                    M[3 * a + c, 3 * b + d] = vol * v
    return M


def _columns(F, R, FiT, Gi, J, mu, lam, vol):
    """M column by column from the oracle's dEdFDifferential."""
    M = np.zeros((9, 9))
    for col in range(9):
        b, d = divmod(col, 3)
        G = np.zeros((3, 3))
        G[b, d] = 1.0
        _, _, dP = oracle.snow_eval(SNOW, F, R, FiT, Gi, J, mu, lam, G @ F, 64)
        M[:, col] = (vol * dP @ F.T).reshape(-1)
    return M


def test_closed_form_matches_the_oracle_differential():
    rng = np.random.default_rng(7)
    vol = 2.5e-8
    worst = 0.0
    for t in range(12):
        Fm = np.eye(3) + 0.15 * rng.normal(size=(3, 3))
        if np.linalg.det(Fm) <= 0.2:
            continue
        s = oracle.snow_update(SNOW, Fm.reshape(1, 9), np.eye(3).reshape(1, 9), 64)
        F, R, FiT, Gi = s["F"][0], s["R"][0], s["FinvTrans"][0], s["Ginv"][0]
        J, mu, lam = s["J"][0], s["mu"][0], s["lambda"][0]
        if t % 3 == 2:   # F replaced after the plasticity update: the rest of the state is stale
            F = np.eye(3) + 0.15 * rng.normal(size=(3, 3))
        ref = _columns(F, R, FiT, Gi, J, mu, lam, vol)
        got = _closed_form(F, R, FiT, Gi, J, mu, lam, vol)
        iu = np.triu_indices(9)      # the entries the force pass stores
        worst = max(worst, np.abs(got[iu] - ref[iu]).max() / np.abs(ref).max())
    assert worst < 1e-12, worst


def test_map_is_symmetric_on_consistent_states():
    """The records store only the upper triangle: on states the plasticity update produced, M is symmetric."""
    rng = np.random.default_rng(8)
    for _ in range(6):
        Fm = np.eye(3) + 0.2 * rng.normal(size=(3, 3))
        if np.linalg.det(Fm) <= 0.2:
            continue
        s = oracle.snow_update(SNOW, Fm.reshape(1, 9), np.eye(3).reshape(1, 9), 64)
        M = _columns(s["F"][0], s["R"][0], s["FinvTrans"][0], s["Ginv"][0], s["J"][0], s["mu"][0], s["lambda"][0], 1.0)
        assert np.abs(M - M.T).max() < 1e-9 * np.abs(M).max()
