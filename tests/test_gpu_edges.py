"""Edge cases of the GPU path: a ragged, non-square world with vacuum holes (tile edges, odd coarse levels, masked
cells, the autotuner's small smoother tiles, the scalar-load fallbacks), and the largest world the ABI accepts (4096²,
gravity padded to 8192²), checked through size-independent properties.

Tolerances: the first system's solution within 1e-6 (max norm, relative) of a direct f64 solve, every implicit solve
to an FP64 relative residual <= 1e-8; at 4096² the step converges, stays finite and keeps the mass to 1e-3 (the leave
edges and the floors move a little)."""
import numpy as np
import pytest

import oracle as O
from sandbox_reactions_b200 import scenes
from sandbox_reactions_b200.engine import Step

pytestmark = pytest.mark.gpu


def ragged_fld(w=200, h=136, scene=11):
    cfg, P, kappa = scenes.fld(256, scene=scene)
    P = P[:, :h, :w].copy()
    kappa = np.ascontiguousarray(kappa[:h, :w])
    j, i = np.mgrid[0:h, 0:w]
    hole = ((i - 60) ** 2 + (j - 70) ** 2 < 12 ** 2) | ((i > 170) & (j > 110))
    P[0][hole] = 1e-9
    P[1][hole] = 0.0
    P[2][hole] = 0.0
    P[3][hole] = 1e-9
    return cfg.replace(width=w, height=h), P, kappa, hole


@pytest.mark.parametrize("precond", ["mg", "jacobi"])
def test_a_ragged_world_with_vacuum_solves_to_1e_8(precond):
    cfg, P, kappa, hole = ragged_fld()
    with Step(cfg) as s:
        s.upload(P)
        s.upload_opacity(kappa)
        ms, rounds, rel, x = s.heat_first_solve(cfg.dt_fixed, precond, want_x=True)
    assert rel <= 1e-8 and rounds > 0
    diag, rhs, kx, ky, gas = O.heat_system(cfg, P.astype(np.float64), cfg.dt_fixed, kappa.astype(np.float64))
    assert not gas[hole].any() and gas.sum() > 0.8 * gas.size
    x_ref, _ = O.heat_pcg(diag, rhs, kx, ky, gas, rel=1e-12, max_rounds=200000)
    assert np.abs(x - x_ref)[gas].max() <= 1e-6 * np.abs(x_ref[gas]).max()


def test_a_ragged_world_steps_like_the_twin():
    cfg, P, kappa, _ = ragged_fld(w=136, h=72, scene=12)
    with Step(cfg) as s:
        s.upload(P)
        s.upload_opacity(kappa)
        s.run(1)
        gpu = s.readback()
        rep = s.read_heat()
    assert rep.converged and rep.rel_residual <= 1e-8
    ref, orep, _, _ = O.heat_step(cfg, P.astype(np.float64), cfg.dt_fixed, kappa.astype(np.float64))
    err = np.abs(gpu[3].astype(np.float64) - ref[3]).sum() / np.abs(ref[3]).sum()
    assert err <= 1e-5, err


def test_the_largest_world_takes_a_full_step():
    cfg, P, kappa = scenes.full_step(4096)
    with Step(cfg) as s:
        s.upload(P)
        s.upload_opacity(kappa)
        s.run(1)
        out = s.readback()
        rep = s.read_heat()
    assert np.isfinite(out).all()
    assert rep.converged and rep.rel_residual <= 1e-8
    m0, m1 = P[0].astype(np.float64).sum(), out[0].astype(np.float64).sum()
    assert abs(m1 - m0) <= 1e-3 * m0
