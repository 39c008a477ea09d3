"""The oracle's reference mode (oracle/sr_oracle_ref.c: 14 channels, the reference's own EOS, species and hold) pinned
against the reference's known answers:

  - the cold pressure's two limits and its blend, the u(x) table against the closed-form integral at every node and
    between nodes, the energy's limits (crates/sr-physics/src/eos.rs tests: cold_pressure_limits,
    table_nodes_equal_the_closed_form_integral, energy_limits, interpolation_between_nodes);
  - the fully ionised composition of pure species (registry.rs:145-154);
  - scenes/thin_cell.bin (the fixture tests/golden/thin_cell.npz, made from it by tests/golden/make_ref_fixtures.py):
    one twin step of P4 alone, leave edges, the hold's rule on the cut, as crates/sr-engine/tests/gpu/sod.rs:672-686
    runs it: no free gas cell faster than 10x its free neighbours' largest, and without the thermal bracket the thin
    cell leaves at |v| ~ 2,100, 54.6x its neighbours' (the figures the reference test's comments give);
  - with the cold pairs off and one species, reference mode steps the same gas as the config-mode oracle at γ = 2 and
    that species' μ (two code paths, one answer);
  - P8's floors and the hold on hand-made cells (floors.rs:124-243);
  - reference-mode P5 on scenes/heat_ceiling.bin (tests/golden/heat_ceiling.npz): the twin's step reaches the ceiling
    in 11 passes and 4,096 rounds and commits by limited fluxes with δ = 0 within the bounds to 1e-9 (the known answer
    crates/sr-engine/tests/gpu/heat.rs:1486-1501 states); with one species and no cold pressure it is the config-mode
    step with that μ and κ₀(1 + X_H)."""
import math
import os

import numpy as np
import pytest

import oracle as O
from sandbox_reactions_b200.abi import Config

HERE = os.path.dirname(os.path.abspath(__file__))
SHIPPED_PAIRS = [(21.3, 134.0), (2.67, 58.2)]


def rel(a, b):
    return abs((a - b) / b)


def node_x(i):
    return math.exp(math.log(1e-8) + i / 511 * (math.log(1e8) - math.log(1e-8)))


def test_cold_pressure_limits_and_blend():
    for k1, k2 in SHIPPED_PAIRS:
        assert rel(O.cold_pressure(1e-12, k1, k2), k1 * 1e-24) < 1e-6
        assert rel(O.cold_pressure(1e16, k1, k2), k2 * 1e16 ** 1.5) < 1e-6
        for x in (1e-6, 1e-2, 1.0, 30.0, 1e4):
            assert rel(O.cold_pressure(x, k1, k2), k1 * x * x / (1.0 + k1 * math.sqrt(x) / k2)) < 1e-12
    assert O.cold_pressure(0.0, 21.3, 134.0) == 0.0 and O.cold_pressure(1.0, 0.0, 0.0) == 0.0


def test_table_nodes_equal_the_closed_form_integral():
    for k1, k2 in SHIPPED_PAIRS + [(1.0, 100.0), (100.0, 1.0), (7.0, 7.0)]:
        t = O.cold_table(k1, k2)
        worst = max(rel(math.exp(t[i]), O.cold_energy_exact(node_x(i), k1, k2)) for i in range(512))
        assert worst < 1e-9, (k1, k2, worst)


def test_energy_limits_and_low_end():
    ur = O.cold_table(100.0, 1.0)
    for x in (1e8, 1e7):
        assert rel(O.cold_table_u(ur, x), 2.0 * x ** 1.5) < 1e-4
    nr = O.cold_table(1.0, 100.0)
    for x in (1e-8, 1e-6):
        assert rel(O.cold_table_u(nr, x), x * x) < 1e-4
    for k1, k2 in SHIPPED_PAIRS:
        assert rel(O.cold_energy_exact(1e-12, k1, k2), k1 * 1e-24) < 1e-6
        assert rel(O.cold_energy_exact(1e20, k1, k2), 2.0 * k2 * 1e30) < 1e-6
        t = O.cold_table(k1, k2)
        assert rel(O.cold_table_u(t, 1e-8), k1 * 1e-16) < 1e-4
        assert O.cold_table_u(t, 0.0) == 0.0 and O.cold_table_u(t, -1.0) == 0.0


def test_interpolation_between_nodes():
    step = (math.log(1e8) - math.log(1e-8)) / 511
    for k1, k2 in SHIPPED_PAIRS + [(1.0, 1e-2), (1.0, 1.0), (1e3, 1.0)]:
        t = O.cold_table(k1, k2)
        worst = 0.0
        for i in range(0, 511, 3):
            for frac in (1.0 / 3.0, 0.5, 2.0 / 3.0):
                x = math.exp(math.log(node_x(i)) + frac * step)
                worst = max(worst, rel(O.cold_table_u(t, x), O.cold_energy_exact(x, k1, k2)))
        assert worst <= 1e-4, (k1, k2, worst)


def test_composition_of_pure_species():
    def pure(s):
        x = [0.0] * 10
        x[s] = 1.0
        return O.composition(x)
    assert pure(0)[:2] == (2.0, 1.0)                      # H: 1/μ = (Z+1)/A = 2, Y_e = 1
    assert pure(1)[:2] == (0.75, 0.5)                     # He
    assert pure(9)[:2] == (1.0, 0.0)                      # neutron matter
    assert abs(pure(8)[0] - 27.0 / 56.0) < 1e-15 and abs(pure(8)[1] - 26.0 / 56.0) < 1e-15  # iron
    assert pure(2)[2] == 1.0 and pure(0)[2] == 0.0        # Z_met


def thin_cell():
    f = np.load(os.path.join(HERE, "golden", "thin_cell.npz"))
    return f["planes"].astype(np.float64), f["held"]


def thin_config(**kw):
    # physics.json as shipped (the cold pairs on), leave edges, P4 alone (sod.rs:672-686)
    return Config(width=64, height=64, channels=14, edge="leave", gravity=False, hydro=True, **kw)


def worst_leap(st, held, sigma_vac=1e-6):
    """sod.rs:620-643: the worst free gas cell inside the edge ring, |v| over its eight free gas neighbours' largest."""
    s, mx, my = st[0], st[1], st[2]
    gas = (held == 0) & (s >= sigma_vac)
    speed = np.hypot(mx, my) / s
    worst = (0.0, None, 0.0)
    h, w = s.shape
    for y in range(1, h - 1):
        for x in range(1, w - 1):
            if not gas[y, x]:
                continue
            near = [(y + dy, x + dx) for dy in (-1, 0, 1) for dx in (-1, 0, 1) if (dy, dx) != (0, 0)]
            most = max([speed[q] for q in near if gas[q]] + [0.0])
            if most > 0.0 and speed[y, x] / most > worst[0]:
                worst = (speed[y, x] / most, (x, y), speed[y, x])
    return worst


def test_the_thin_cell_takes_no_leap_and_leaps_without_the_bracket():
    P, _ = thin_cell()
    twin = O.RefTwin(thin_config(), P)
    twin.step()
    st, held = twin.state()
    ratio, _, _ = worst_leap(st, held)
    assert ratio <= 10.0, ratio
    # the bracket out: the thin cell (32, 32) leaves at |v| ~ 2,100, 54.6x its neighbours' largest
    twin = O.RefTwin(thin_config(thermal_bracket=False), P)
    twin.step()
    st, held = twin.state()
    ratio, cell, v = worst_leap(st, held)
    assert cell == (32, 32)
    assert abs(v / 2100.0 - 1.0) < 0.05, v
    assert abs(ratio / 54.6 - 1.0) < 0.1, ratio


def test_reference_mode_with_one_species_and_no_cold_pressure_is_the_config_mode_gas():
    rng = np.random.default_rng(5)
    h, w = 40, 48
    s = 1.0 + 0.5 * rng.random((h, w))
    s[:, :6] = 1e-9  # a vacuum strip
    mx, my = 0.3 * rng.standard_normal((h, w)) * s, 0.3 * rng.standard_normal((h, w)) * s
    e = s * (0.5 + rng.random((h, w))) + 0.5 * (mx * mx + my * my) / s
    P14 = np.zeros((14, h, w))
    P14[:4] = s, mx, my, e
    P14[5] = 1.0  # helium: 1/μ = 0.75
    off = dict(k1e=0.0, k2e=0.0, k1n=0.0, k2n=0.0)
    for edge in ("bounce", "leave"):
        cfg = Config(width=w, height=h, channels=14, edge=edge, gravity=True, **off)
        g = O.grav_field(cfg, s)[1:]
        ref, _ = O.ref_hydro_step(cfg, P14, 0.01, g)
        c4 = cfg.replace(channels=4, gamma=2.0, mu=1.0 / 0.75)
        out, _ = O.hydro_step(c4, P14[:4], 0.01, g)
        for k in range(4):
            assert np.abs(ref[k] - out[k]).max() <= 1e-12 * max(1.0, np.abs(out[k]).max()), (edge, k)
        assert np.all(ref[5] == 1.0) and np.all(ref[4] == 0.0)


def test_floors_and_the_hold_on_hand_made_cells():
    cfg = Config(width=16, height=16, channels=14)
    P = np.zeros((14, 16, 16))
    P[0] = 1.0
    P[4] = 1.0  # hydrogen
    P[3] = 1.0
    # a vacuum cell resets to the floor state with its fractions renormalised; its E holds the cold energy
    P[0, 2, 3] = 1e-7
    P[4, 2, 3], P[5, 2, 3] = 2.0, 2.0
    # a cell below its thermal floor is raised to it
    P[3, 5, 5] = 1e-9
    out, (vac, added) = O.ref_floors(cfg, P)
    x = np.zeros(10)
    x[0] = x[1] = 0.5
    inv_mu, ye, _ = O.composition(x)
    sf = float(np.float32(1e-8))
    ln_e = O.cold_table(21.3, 134.0)
    ln_n = O.cold_table(2.67, 58.2)
    cold = (O.cold_table_u(ln_e, ye * sf) + O.cold_table_u(ln_n, 0.0)) / sf
    assert out[0, 2, 3] == sf and out[1, 2, 3] == 0.0
    assert abs(out[3, 2, 3] - sf * (0.05 * inv_mu + cold)) <= 1e-15
    assert out[4, 2, 3] == 0.5 and out[5, 2, 3] == 0.5
    assert abs(vac - (1e-7 - sf)) < 1e-20
    inv_h, ye_h, _ = O.composition([1.0] + [0.0] * 9)
    eps_floor = 0.05 * inv_h
    cold_h = O.cold_table_u(ln_e, ye_h * 1.0) / 1.0
    assert abs(out[3, 5, 5] - (eps_floor + cold_h)) < 1e-12
    # the hold: a dense cold hydrogen cell (Σ >= σ_hold, ε_th <= η_hold ε_cold) is held and its momentum taken;
    # the same cell hotter is not; a held cell stays held until ε_th passes 2 η_hold ε_cold
    Q = np.zeros((14, 16, 16))
    Q[0] = 1e-7
    Q[4] = 1.0
    sig = 12.0
    cold12 = O.cold_table_u(ln_e, ye_h * sig) / sig
    Q[0, 8, 8] = sig
    Q[1, 8, 8] = 0.3
    Q[3, 8, 8] = sig * (0.05 * cold12 + cold12) + 0.5 * 0.3 * 0.3 / sig
    Q[0, 3, 3] = sig
    Q[3, 3, 3] = sig * (0.5 * cold12 + cold12)
    q, m, taken = O.ref_hold(cfg, Q)
    assert m[8, 8] == 1 and m[3, 3] == 0 and m.sum() == 1
    assert q[1, 8, 8] == 0.0 and abs(taken[0] - 0.3) < 1e-15
    Q[3, 8, 8] = sig * (0.15 * cold12 + cold12)  # between η and 2η: held stays held, a free cell is not taken
    _, m2, _ = O.ref_hold(cfg, Q, held=m)
    assert m2[8, 8] == 1
    _, m3, _ = O.ref_hold(cfg, Q)
    assert m3[8, 8] == 0
    # the disk gate: the same cell inside a disk of more than m_tov is free
    _, m4, _ = O.ref_hold(cfg.replace(m_tov=10.0), Q, held=m)
    assert m4[8, 8] == 0


def heat_cut(name):
    f = np.load(os.path.join(HERE, "golden", name + ".npz"))
    # the cuts ran on a_r 4e-5 and c_sb 200 (crates/sr-engine/tests/gpu/heat.rs:1433-1437), every test flag off
    cfg = Config(width=64, height=64, channels=14, heat=True, hydro=False, gravity=False, a_r=4e-5, c_sb=200.0)
    return cfg, f["planes"].astype(np.float64), float(np.float32(f["dt_next"]))


def held_above_floor(cfg, P):
    """heat.rs tests' held_above_floor: C (T⁰ - T_floor) on the gas, 0 off it."""
    t0, _, inv_mu = O.ref_heat_sides(cfg, P)
    gas = P[0] >= cfg.sigma_vac
    return np.where(gas, P[0] * inv_mu * (t0 - cfg.t_floor), 0.0)


def test_the_ceiling_cut_reaches_the_ceiling_and_moves_no_more_heat_than_its_cells_hold():
    # heat.rs:1486-1501: the twin's step of scenes/heat_ceiling.bin reaches the ceiling in 11 passes and 4,096 rounds;
    # its commit by limited fluxes has δ = 0 and holds the bounds to 1e-9
    cfg, P, dt = heat_cut("heat_ceiling")
    out, rep, _, _ = O.ref_heat_step(cfg, P, dt)
    assert (rep.passes, rep.rounds, rep.converged, rep.delta) == (11, 4096, 0, 0.0)
    held = held_above_floor(cfg, P)
    lost = P[3] - out[3]
    gas = P[0] >= cfg.sigma_vac
    assert np.all(lost[gas] <= held[gas] * (1 + 1e-9) + 1e-12 * np.abs(P[3][gas]))
    assert abs(lost.sum() - rep.radiated) <= 1e-9 * held.sum()
    assert rep.radiated <= held.sum() * (1 + 1e-9)


def test_reference_mode_heat_with_one_species_is_the_config_mode_step():
    # C = Σ/μ, T = μ ε_th and κ = κ₀(1 + X_H) of one species and no cold pressure: the config-mode step at γ = 2 with
    # that μ and the κ plane κ₀(1 + X_H)
    rng = np.random.default_rng(11)
    h, w = 32, 40
    s = 0.5 + rng.random((h, w))
    s[:4, :] = 1e-9
    e = s * (1.0 + 4.0 * rng.random((h, w)))
    P = np.zeros((14, h, w))
    P[0], P[3] = s, e
    P[4], P[5] = 0.7, 0.3
    off = dict(k1e=0.0, k2e=0.0, k1n=0.0, k2n=0.0)
    cfg = Config(width=w, height=h, channels=14, heat=True, hydro=False, **off)
    out, rep, fx, fy = O.ref_heat_step(cfg, P, 0.05)
    inv_mu = O.composition([0.7, 0.3] + [0.0] * 8)[0]
    c4 = cfg.replace(channels=4, mu=1.0 / inv_mu, gamma=2.0, opacity_plane=True)
    kappa = np.full((h, w), cfg.kappa0 * 1.7)
    o4, r4, fx4, fy4 = O.heat_step(c4, P[:4], 0.05, kappa)
    assert rep.converged and r4.converged and rep.passes == r4.passes
    assert np.abs(out[3] - o4[3]).max() <= 1e-10 * np.abs(o4[3]).max()
    assert np.abs(fx - fx4).max() <= 1e-10 * np.abs(fx4).max()
