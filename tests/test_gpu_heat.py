"""The CUDA implicit FLD step (P5), called through the C ABI, against the oracle's f64 twin
(crates/sr-physics/src/reference/heat.rs, crates/sr-engine/tests/gpu/heat.rs).

Tolerances: one implicit step from a shared f32 start, rel L1 of E <= 1e-5 (the per-step bar); each Newton pass's
linear solve reaches an FP64 relative residual <= 1e-8 (cfg.solve_tol); the first system's solution within 1e-6 of a
direct f64 solve."""
import numpy as np
import pytest

import oracle as O
from sandbox_reactions_b200 import scenes
from sandbox_reactions_b200.abi import Config
from sandbox_reactions_b200.engine import Step

pytestmark = pytest.mark.gpu


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)


def temperature_planes(T, sigma=1.0, gamma=2.0, mu=1.0):
    h, w = T.shape
    P = np.zeros((4, h, w))
    P[0] = sigma
    P[3] = sigma * T / (mu * (gamma - 1.0))
    return P.astype(np.float32)


def heat_cfg(w, h, **kw):
    base = dict(width=w, height=h, hydro=False, heat=True, gamma=2.0, mu=1.0)
    base.update(kw)
    return Config(**base)


def gpu_heat_step(cfg, P, dt, kappa=None, precond="mg"):
    cfg = cfg.replace(dt_fixed=dt, precond=precond)
    with Step(cfg) as s:
        s.upload(P)
        if kappa is not None:
            s.upload_opacity(kappa)
        s.run(1)
        out = s.readback()
        rep = s.read_heat()
        fx, fy = s.read_heat_flux()
    return out, rep, fx, fy


def test_constant_diffusivity_gaussian_matches_the_twin():
    w = h = 64
    j, i = np.mgrid[0:h, 0:w]
    T = 0.05 + 2.0 * np.exp(-((i - 31.5) ** 2 + (j - 31.5) ** 2) / 18.0)
    cfg = heat_cfg(w, h, chi=0.25)
    P = temperature_planes(T)
    gpu, rep, fx, fy = gpu_heat_step(cfg, P, 1.0)
    ref, orep, ofx, ofy = O.heat_step(cfg, P.astype(np.float64), 1.0)
    assert rep.converged and rep.rel_residual <= 1e-8
    assert rel_l1(gpu[3], ref[3]) <= 1e-5
    assert rel_l1(fx, ofx) <= 1e-5 and rel_l1(fy, ofy) <= 1e-5


@pytest.mark.parametrize("precond", ["mg", "jacobi"])
def test_fld_step_with_an_opacity_field_matches_the_twin(precond):
    w, h = 96, 80
    rng = np.random.default_rng(4)
    T = 30.0 + 300.0 * np.exp(-((np.mgrid[0:h, 0:w][1] - 40) ** 2 + (np.mgrid[0:h, 0:w][0] - 30) ** 2) / 60.0)
    T += 5.0 * rng.random((h, w))
    kappa = (10.0 ** rng.uniform(-1.0, 1.0, (h, w))).astype(np.float32)
    cfg = heat_cfg(w, h, opacity_plane=True)
    P = temperature_planes(T)
    P[0, :4, :] = 1e-9  # a vacuum band along the top edge
    P[3, :4, :] = 1e-9
    dt = 2e-3
    gpu, rep, fx, fy = gpu_heat_step(cfg, P, dt, kappa, precond)
    ref, orep, ofx, ofy = O.heat_step(cfg, P.astype(np.float64), dt, kappa.astype(np.float64))
    assert orep.converged and rep.converged
    assert rep.rel_residual <= 1e-8
    assert rel_l1(gpu[3], ref[3]) <= 1e-5, rel_l1(gpu[3], ref[3])
    assert abs(rep.radiated - orep.radiated) <= 1e-5 * abs(orep.radiated)
    assert rel_l1(fx, ofx) <= 1e-5


def test_the_first_system_solves_to_1e_8_with_either_preconditioner():
    cfg, P, kappa = scenes.fld(128, scene=7)
    x_ref = None
    for precond in ("mg", "jacobi"):
        with Step(cfg) as s:
            s.upload(P)
            s.upload_opacity(kappa)
            ms, rounds, rel, x = s.heat_first_solve(cfg.dt_fixed, precond, want_x=True)
        assert rel <= 1e-8 and rounds > 0
        if x_ref is None:
            diag, rhs, kx, ky, gas = O.heat_system(cfg, P.astype(np.float64), cfg.dt_fixed, kappa.astype(np.float64))
            x_ref, r = O.heat_pcg(diag, rhs, kx, ky, gas, rel=1e-12, max_rounds=200000)
        assert np.abs(x - x_ref).max() <= 1e-6 * np.abs(x_ref).max()


def test_multigrid_needs_far_fewer_rounds_than_jacobi():
    cfg, P, kappa = scenes.fld(256, scene=8)
    rounds = {}
    with Step(cfg) as s:
        s.upload(P)
        s.upload_opacity(kappa)
        for precond in ("mg", "jacobi"):
            _, rounds[precond], rel, _ = s.heat_first_solve(cfg.dt_fixed, precond)
            assert rel <= 1e-8
    assert rounds["mg"] * 4 <= rounds["jacobi"], rounds


def test_past_the_ceiling_the_step_commits_by_limited_fluxes():
    w = h = 64
    T = np.full((h, w), 1.0)
    T[32, 32] = 3e4
    cfg = heat_cfg(w, h, max_rounds=2)
    P = temperature_planes(T)
    gpu, rep, fx, fy = gpu_heat_step(cfg, P, 1.0)
    assert not rep.converged
    # the grid loses exactly what it books as radiated, and no cell gives more than it holds above its floor
    e0 = P[3].astype(np.float64).sum()
    assert abs((gpu[3].astype(np.float64).sum() - e0) + rep.radiated) <= 1e-5 * e0
    assert np.all(gpu[3] >= 0.05 - 1e-6)


def test_one_full_step_with_every_pass_matches_the_twin():
    cfg, P, kappa = scenes.full_step(64)
    with Step(cfg) as s:
        s.upload(P)
        s.upload_opacity(kappa)
        s.run(1)
        gpu = s.readback()
        dt = s.read_dt().dt
        rep = s.read_heat()
    assert rep.converged
    twin = O.Twin(cfg.replace(dt_fixed=dt), P.astype(np.float64), kappa.astype(np.float64))
    twin.step(1)
    ref = twin.state()
    for k in range(4):
        assert rel_l1(gpu[k], ref[k]) <= 1e-5, (k, rel_l1(gpu[k], ref[k]))


@pytest.mark.parametrize("pre,post", [(1, 1), (2, 2), (3, 3), (4, 4), (2, 4), (4, 1)])
def test_every_v_cycle_solves_the_first_system(pre, post):
    # 1..4 red-black sweeps a side (the smoothers' 2..8 half-sweep instances): the same solution to 1e-8, the deeper
    # cycles in no more rounds than V(1,1)
    cfg, P, kappa = scenes.fld(128, scene=7)
    cfg = cfg.replace(mg_pre=pre, mg_post=post)
    diag, rhs, kx, ky, gas = O.heat_system(cfg, P.astype(np.float64), cfg.dt_fixed, kappa.astype(np.float64))
    x_ref, _ = O.heat_pcg(diag, rhs, kx, ky, gas, rel=1e-12, max_rounds=200000)
    with Step(cfg) as s:
        s.upload(P)
        s.upload_opacity(kappa)
        _, rounds, rel, x = s.heat_first_solve(cfg.dt_fixed, "mg", want_x=True)
        with Step(cfg.replace(mg_pre=1, mg_post=1)) as s1:
            s1.upload(P)
            s1.upload_opacity(kappa)
            _, rounds1, _, _ = s1.heat_first_solve(cfg.dt_fixed, "mg")
    assert rel <= 1e-8 and rounds <= rounds1, (rounds, rounds1)
    assert np.abs(x - x_ref).max() <= 1e-6 * np.abs(x_ref).max()


def test_v44_on_the_row_band_levels():
    # a 1024² world: its big levels take the row-band smoothers (V(4,4): the 8 half-sweep instances, halos 10 and 8)
    cfg, P, kappa = scenes.fld(1024, scene=9)
    got = {}
    for nu in (2, 4):
        with Step(cfg.replace(mg_pre=nu, mg_post=nu)) as s:
            s.upload(P)
            s.upload_opacity(kappa)
            _, rounds, rel, x = s.heat_first_solve(cfg.dt_fixed, "mg", want_x=True)
        assert rel <= 1e-8
        got[nu] = (rounds, x)
    assert got[4][0] <= got[2][0]
    assert np.abs(got[4][1] - got[2][1]).max() <= 1e-6 * np.abs(got[2][1]).max()
