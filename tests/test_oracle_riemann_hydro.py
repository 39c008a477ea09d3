"""The oracle's exact Riemann solution and its hydro (P4) against the reference's tests
(crates/sr-physics/src/reference/riemann.rs:217-455, crates/sr-engine/tests/gpu/sod.rs:1-263)."""
import numpy as np
import pytest

import oracle as O
from sandbox_reactions_b200.abi import Config

PROBLEMS = [
    ("sod", (1.0, 0.0, 1.0), (0.125, 0.0, 0.1)),
    ("two rarefactions", (1.0, -0.5, 1.0), (1.0, 0.5, 1.0)),
    ("two shocks", (1.0, 1.0, 1.0), (1.0, -1.0, 1.0)),
    ("strong shock right", (1.0, 0.0, 1000.0), (1.0, 0.0, 0.01)),
    ("shock left, rarefaction right", (0.125, 0.0, 0.1), (1.0, 0.0, 1.0)),
    ("moving contact", (1.0, 0.75, 1.0), (0.125, 0.75, 1.0)),
    ("slow collision", (5.99924, 19.5975, 460.894), (5.99242, -6.19633, 46.0950)),
]


def du_across(g, p, k, side):
    """An independent pressure function (riemann.rs:262-276): Rankine-Hugoniot by the mass flux, or the isentrope."""
    rho, u, pk = k
    if p > pk:
        mu = (g - 1.0) / (g + 1.0)
        rs = rho * (p / pk + mu) / (mu * p / pk + 1.0)
        m = np.sqrt((p - pk) / (1.0 / rho - 1.0 / rs))
        return side * (p - pk) / m
    c = np.sqrt(g * pk / rho)
    cs = c * (p / pk) ** ((g - 1.0) / (2.0 * g))
    return side * 2.0 / (g - 1.0) * (cs - c)


def bisect_star(g, l, r):
    f = lambda p: (l[1] + du_across(g, p, l, -1.0)) - (r[1] + du_across(g, p, r, 1.0))
    lo, hi = 1e-12, 1.0
    while f(hi) > 0:
        hi *= 2
    for _ in range(300):
        mid = 0.5 * (lo + hi)
        if f(mid) > 0:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


@pytest.mark.parametrize("gamma", [2.0, 1.4, 5.0 / 3.0])
def test_star_pressure_matches_an_independent_bisection(gamma):
    for name, l, r in PROBLEMS:
        s = O.Riemann(gamma, l, r)
        p = bisect_star(gamma, l, r)
        assert abs(s.p_star - p) / p < 1e-10, name
        fl = l[1] + du_across(gamma, p, l, -1.0)
        assert abs(s.u_star - fl) < 1e-9 * (1 + abs(fl)), name


@pytest.mark.parametrize("gamma", [2.0, 1.4])
def test_mirrored_states_give_the_mirrored_solution(gamma):
    for name, l, r in PROBLEMS:
        a = O.Riemann(gamma, l, r)
        b = O.Riemann(gamma, (r[0], -r[1], r[2]), (l[0], -l[1], l[2]))
        assert abs(a.p_star - b.p_star) / a.p_star < 1e-10
        for xi in np.linspace(-15, 15, 61):
            q, m = a.sample(xi), b.sample(-xi)
            assert abs(q[0] - m[0]) <= 1e-9 * q[0] and abs(q[2] - m[2]) <= 1e-9 * q[2], (name, xi)


def test_a_state_with_no_solution_is_refused():
    ok = (1.0, 0.0, 1.0)
    for bad in ((0.0, 0.0, 1.0), (1.0, 0.0, -1.0), (np.nan, 0.0, 1.0), (1.0, np.inf, 1.0)):
        with pytest.raises(ValueError, match="bad state"):
            O.Riemann(2.0, bad, ok)
    with pytest.raises(ValueError, match="vacuum"):
        O.Riemann(2.0, (1.0, -3.0, 1.0), (1.0, 3.0, 1.0))
    O.Riemann(2.0, (1.0, -2.0, 1.0), (1.0, 2.0, 1.0))


# ------------------------------------------------------------------ hydro: G-SOD on the oracle


def sod_planes(w, h, gamma, x0, axis=0):
    P = np.zeros((4, h, w))
    idx = np.arange(w)[None, :] if axis == 0 else np.arange(h)[:, None]
    left = np.broadcast_to(idx < x0, (h, w))
    P[0] = np.where(left, 1.0, 0.125)
    P[3] = np.where(left, 1.0, 0.1) / (gamma - 1.0)
    return P


def advance(cfg, P, t_end):
    t, steps = 0.0, 0
    while t < t_end:
        dt = min(O.hydro_dt(cfg, P), t_end - t)
        assert np.isfinite(dt) and dt > 1e-9
        P, _ = O.hydro_step(cfg, P, dt)
        t += dt
        steps += 1
    return P, steps


def exact_cell_density(R, i, x0, t, n=400):
    """The exact density averaged over cell i by n midpoints (tests/gpu/sod.rs:94-99)."""
    xs = i + (np.arange(n) + 0.5) / n
    return np.mean([R.sample((x - x0) / t)[0] for x in xs])


@pytest.fixture(scope="module")
def sod_strip():
    cfg = Config(width=400, height=4, edge="bounce", limiter="mc", gamma=2.0)
    P0 = sod_planes(400, 4, 2.0, 200)
    P, steps = advance(cfg, P0, 80.0)
    return cfg, P0, P


def test_sod_shock_is_within_one_cell_and_l1_within_two_percent(sod_strip):
    cfg, _, P = sod_strip
    R = O.Riemann(2.0, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    rho = P[0, 0]
    mid = 0.5 * (R.sol[3] + 0.125)
    i = max(k for k in range(400) if rho[k] >= mid)
    x_num = (i + 0.5) + (rho[i] - mid) / (rho[i] - rho[i + 1])
    x_exact = 200.0 + R.sol[8] * 80.0
    assert abs(x_num - x_exact) <= 1.0
    ex = np.array([exact_cell_density(R, k, 200.0, 80.0, 100) for k in range(400)])
    assert np.abs(rho - ex).sum() / ex.sum() <= 0.02


def test_sod_mass_energy_and_the_walls_momentum_are_exact(sod_strip):
    cfg, P0, P = sod_strip
    rel = lambda a, b: abs(a - b) / abs(b)
    assert rel(P[0].sum(), P0[0].sum()) < 1e-12
    assert rel(P[3].sum(), P0[3].sum()) < 1e-12
    pushed = (1.0 - 0.1) * 80.0 * 4.0
    assert rel(P[1].sum(), pushed) < 1e-10
    assert abs(P[2].sum()) < 1e-12
    # every row the same gas (Σv only to rounding: HLL of two equal states returns Π to an ulp)
    assert np.abs(P - P[:, :1, :]).max() < 1e-12


def test_the_tube_laid_along_y_runs_as_along_x():
    cfg = Config(width=64, height=16, edge="bounce", gamma=2.0)
    P = sod_planes(64, 16, 2.0, 32)
    cfgt = Config(width=16, height=64, edge="bounce", gamma=2.0)
    Pt = np.stack([P[0].T, P[2].T, P[1].T, P[3].T])
    for _ in range(20):
        dt = O.hydro_dt(cfg, P)
        assert dt == O.hydro_dt(cfgt, Pt)
        P, _ = O.hydro_step(cfg, P, dt)
        Pt, _ = O.hydro_step(cfgt, Pt, dt)
    assert np.array_equal(P[0], Pt[0].T) and np.array_equal(P[1], Pt[2].T) and np.array_equal(P[3], Pt[3].T)


def test_the_mirrored_tube_is_the_mirror():
    cfg = Config(width=64, height=8, edge="bounce", gamma=2.0)
    P = sod_planes(64, 8, 2.0, 32)
    M = P[:, :, ::-1].copy()
    M[1] = -M[1]
    for _ in range(20):
        dt = O.hydro_dt(cfg, P)
        P, _ = O.hydro_step(cfg, P, dt)
        M, _ = O.hydro_step(cfg, M, dt)
    assert np.abs(P[0] - M[0, :, ::-1]).max() < 1e-13
    assert np.abs(P[1] + M[1, :, ::-1]).max() < 1e-13


@pytest.mark.parametrize("limiter", ["minmod", "mc"])
def test_config_mode_sod_gamma_1_4_leave_against_the_exact_solution(limiter):
    """The C1 scheme (γ = 1.4, minmod, HLL, outflow = leave) on a 1D strip against the γ-general exact solution."""
    gamma = 1.4
    cfg = Config(width=256, height=8, edge="leave", limiter=limiter, gamma=gamma)
    P = sod_planes(256, 8, gamma, 128)
    t_end = 0.2 * 256 / 1.0  # the unit tube's t = 0.2 with cells of 1/256 and speeds scaled by the grid
    P, _ = advance(cfg, P, t_end * 0.25)
    R = O.Riemann(gamma, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    ex = np.array([exact_cell_density(R, k, 128.0, t_end * 0.25, 50) for k in range(256)])
    assert np.abs(P[0, 0] - ex).sum() / ex.sum() <= 0.02


def test_leave_edges_book_what_escapes():
    cfg = Config(width=64, height=8, edge="leave", limiter="minmod", gamma=1.4)
    P = sod_planes(64, 8, 1.4, 32)
    m0 = P[0].sum()
    out = 0.0
    for _ in range(200):
        dt = O.hydro_dt(cfg, P)
        P, rep = O.hydro_step(cfg, P, dt)
        out += rep.escaped[0]
        assert rep.escaped[0] >= 0.0  # inflow is exactly 0
    assert out > 0.0
    assert abs(P[0].sum() + out - m0) < 1e-12 * m0


def test_floors_reset_vacuum_and_raise_cold_gas():
    """P8 (reference/floors.rs:124-196): Σ < Σ_vac → the floor state; ε_th below T_floor/μ raised to it."""
    cfg = Config(gamma=1.4, mu=1.0)
    P = np.zeros((4, 2, 2))
    P[0] = [[1e-7, 1.0], [1.0, 1.0]]
    P[1] = [[5.0, 0.0], [0.0, 1.0]]
    P[3] = [[1.0, 1e-9], [10.0, 0.5]]
    Q = O.floors(cfg, P)
    floor_eps = 0.05 / 1.0 / 0.4
    assert Q[0, 0, 0] == np.float64(np.float32(1e-8)) and Q[1, 0, 0] == 0.0
    assert abs(Q[3, 0, 0] - Q[0, 0, 0] * floor_eps) < 1e-15 * Q[3, 0, 0]
    assert abs(Q[3, 0, 1] - floor_eps) < 1e-15  # raised to the floor
    assert Q[3, 1, 0] == 10.0  # above it: kept
    assert abs(Q[3, 1, 1] - (0.5 + floor_eps)) < 1e-15  # kinetic 0.5 left, thermal raised from 0
