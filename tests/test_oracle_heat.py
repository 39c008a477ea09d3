"""The oracle's implicit FLD step (P5) against the reference's heat tests
(crates/sr-physics/src/reference/heat.rs, crates/sr-engine/tests/gpu/heat.rs:10-22, 389-431, 713-787, 917-990)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle as O
from sandbox_reactions_b200.abi import Config


def test_lambda_is_levermore_pomraning():
    for r, want in ((0.0, 1 / 3), (1.0, 0.3), (2.0, 0.25), (3.0, 5 / 24), (10.0, 12 / 136)):
        assert abs(O.lam(r) - want) < 1e-15
    for r in (0.01, 1.0, 100.0, 1e6, 1e12):
        assert O.lam(r) * r < 1.0
    assert O.lam(1e12) * 1e12 > 1.0 - 1e-9
    vals = [O.lam(float(k)) for k in range(60)]
    assert all(b < a for a, b in zip(vals, vals[1:]))


def temperature_planes(T, sigma=1.0, gamma=2.0, mu=1.0):
    h, w = T.shape
    P = np.zeros((4, h, w))
    P[0] = sigma
    P[3] = sigma * T / (mu * (gamma - 1.0))
    return P


def temps(P, gamma=2.0, mu=1.0):
    return mu * (gamma - 1.0) * P[3] / P[0]


CHI, SIGMA0, PEAK, BG = 0.25, 3.0, 2.0, 0.05


def gaussian():
    w = h = 64
    j, i = np.mgrid[0:h, 0:w]
    r2 = (i - 31.5) ** 2 + (j - 31.5) ** 2
    T = BG + PEAK * np.exp(-r2 / (2 * SIGMA0 ** 2))
    cfg = Config(width=w, height=h, hydro=False, heat=True, chi=CHI, gamma=2.0, mu=1.0)
    return cfg, temperature_planes(T)


def moments(P):
    T = temps(P) - BG
    h, w = T.shape
    j, i = np.mgrid[0:h, 0:w]
    H = T.sum()
    cx, cy = (T * i).sum() / H, (T * j).sum() / H
    return H, (T * (i - cx) ** 2).sum() / H, (T * (j - cy) ** 2).sum() / H


def test_the_variance_grows_as_sigma0_squared_plus_two_chi_t_per_axis():
    cfg, P = gaussian()
    h0, vx0, vy0 = moments(P)
    for step in range(1, 25):
        P, rep, _, _ = O.heat_step(cfg, P, 1.0)
        assert rep.converged and rep.passes == 2 and rep.rounds > 0
        if step % 8 == 0:
            _, vx, vy = moments(P)
            want = vx0 + 2 * CHI * step
            assert max(abs(vx - want), abs(vy - want)) / want <= 0.01


def test_the_total_heat_is_constant():
    cfg, P = gaussian()
    h0, _, _ = moments(P)
    for _ in range(24):
        P, rep, _, _ = O.heat_step(cfg, P, 1.0)
        h, _, _ = moments(P)
        assert abs(h - h0) / h0 <= 1e-5


def test_the_flux_kept_is_chi_c_times_the_temperature_difference():
    cfg, P = gaussian()
    P, rep, fx, fy = O.heat_step(cfg, P, 1.0)
    T = temps(P)
    want = -CHI * 1.0 * (T[:, 1:] - T[:, :-1])
    assert np.abs(fx[:, 1:-1] - want).max() <= 1e-9 * np.abs(want).max()


def hot_field(w=48, h=40, seed=5):
    rng = np.random.default_rng(seed)
    T = 10.0 ** rng.uniform(0.0, 3.0, (h, w))
    return T


def test_the_fld_flux_is_bounded_by_free_streaming():
    """|F| ≤ c_sb a_r T⁴ of the hotter side (1 + 1e-6) at every face of the law (heat.rs:1-25)."""
    cfg = Config(width=48, height=40, hydro=False, heat=True)
    T = hot_field()
    P = temperature_planes(T, sigma=1e-3)
    fx, fy = O.heat_law(cfg, P)
    Tp = np.pad(T, 1, constant_values=cfg.t_floor)
    hot_x = np.maximum(Tp[1:-1, :-1], Tp[1:-1, 1:])
    hot_y = np.maximum(Tp[:-1, 1:-1], Tp[1:, 1:-1])
    assert np.all(np.abs(fx) <= cfg.c_sb * cfg.a_r * hot_x ** 4 * (1 + 1e-6))
    assert np.all(np.abs(fy) <= cfg.c_sb * cfg.a_r * hot_y ** 4 * (1 + 1e-6))


def test_thick_gas_has_the_radiative_conductivity():
    """F → -(4/3) a_r c_sb T³/(κΣ) ∇T in optically thick gas (tests/gpu/heat.rs:940-971)."""
    w, h = 64, 4
    cfg = Config(width=w, height=h, hydro=False, heat=True, kappa0=1e3)
    T = np.broadcast_to(100.0 + 0.01 * np.arange(w), (h, w)).copy()
    P = temperature_planes(T, sigma=1e3)
    fx, _ = O.heat_law(cfg, P)
    ks = 1e3 * 1e3
    mid = 0.5 * (T[:, :-1] + T[:, 1:])
    want = -(4.0 / 3.0) * cfg.a_r * cfg.c_sb * mid ** 3 / ks * (T[:, 1:] - T[:, :-1])
    assert np.abs((fx[:, 1:-1] - want) / want).max() <= 0.01


def test_a_one_cell_pulse_stays_non_negative_and_the_heat_balance_closes():
    w = h = 32
    cfg = Config(width=w, height=h, hydro=False, heat=True)
    T = np.full((h, w), 1.0)
    T[16, 16] = 300.0
    P = temperature_planes(T)
    E0 = P[3].sum()
    Q, rep, fx, fy = O.heat_step(cfg, P, 0.05)
    assert rep.converged
    Tn = temps(Q)
    assert np.all(Tn > 0.0)
    assert Tn[16, 16] < 300.0 and Tn[16, 17] > 1.0
    # the grid loses exactly what it books as radiated (δ closes the balance)
    assert abs((Q[3].sum() - E0) + rep.radiated) <= 1e-10 * E0


def test_backward_euler_is_first_order():
    w = h = 32
    cfg = Config(width=w, height=h, hydro=False, heat=True)
    j, i = np.mgrid[0:h, 0:w]
    T = 20.0 + 80.0 * np.exp(-((i - 15.5) ** 2 + (j - 15.5) ** 2) / 18.0)
    P0 = temperature_planes(T)
    t_end = 0.02

    def run(n):
        P = P0.copy()
        for _ in range(n):
            P, rep, _, _ = O.heat_step(cfg, P, t_end / n)
            assert rep.converged
        return temps(P)

    ref = run(64)
    e1 = np.abs(run(2) - ref).sum()
    e2 = np.abs(run(4) - ref).sum()
    assert 1.6 <= e1 / e2 <= 2.6


def test_the_twins_solve_matches_a_direct_sparse_solve():
    w, h = 40, 32
    rng = np.random.default_rng(11)
    cfg = Config(width=w, height=h, hydro=False, heat=True, opacity_plane=True)
    T = 50.0 + 200.0 * rng.random((h, w))
    P = temperature_planes(T)
    P[0, :3, :] = 1e-9  # a vacuum band: its faces are the vacuum state's
    kappa = 10.0 ** rng.uniform(-2, 2, (h, w))
    diag, rhs, kx, ky, gas = O.heat_system(cfg, P, 0.01, kappa)
    n = w * h
    idx = np.arange(n).reshape(h, w)
    rows, cols, vals = [idx.ravel()], [idx.ravel()], [diag.ravel()]
    g = gas.astype(bool)
    m = g[:, :-1] & g[:, 1:]
    rows += [idx[:, :-1][m], idx[:, 1:][m]]
    cols += [idx[:, 1:][m], idx[:, :-1][m]]
    vals += [-kx[:, 1:-1][m], -kx[:, 1:-1][m]]
    m = g[:-1, :] & g[1:, :]
    rows += [idx[:-1, :][m], idx[1:, :][m]]
    cols += [idx[1:, :][m], idx[:-1, :][m]]
    vals += [-ky[1:-1, :][m], -ky[1:-1, :][m]]
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    x_direct = spla.spsolve(A.tocsc(), rhs.ravel())
    x, rounds = O.heat_pcg(diag, rhs, kx, ky, gas, rel=1e-13)
    assert rounds > 0
    assert np.abs(x.ravel() - x_direct).max() <= 1e-9 * np.abs(x_direct).max()
    # the matvec is the matrix
    v = rng.random((h, w))
    assert np.abs(O.heat_matvec(diag, kx, ky, gas, v).ravel() - (A @ v.ravel()) * g.ravel()).max() < 1e-9 * np.abs(
        A @ v.ravel()).max()
