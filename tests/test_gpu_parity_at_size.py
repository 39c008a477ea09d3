"""Parity at the benchmark configurations' own sizes: the CUDA path through the C ABI against the oracle's f64 twin
(the reference's GPU-vs-twin tier, crates/sr-engine/tests/gpu/cpu_gpu.rs:37-42,67-182, in the twin's pass order,
crates/sr-physics/src/reference/mod.rs:264-297), run on the worlds the benchmark times rather than on small ones.

  - the headline world: one full hydro + gravity + FLD step of the seeded 2048² world (scenes.full_step) from the
    same f32 start as the twin: rel L1 <= 1e-5 per field, P2's potential of the start state within 1e-5 and its
    acceleration within the reference's field bar 1e-3, and the implicit solve at an FP64 relative residual <= 1e-8;
  - config 1, Sod 512² (γ = 1.4, minmod, leave edges): one step within 1e-5 per field; 200 steps within the reference's
    G-REF bands (Σ and E rel L1 <= 1e-3, clock within 5e-4) and the exact Riemann density within 2 % in L1
    (tests/gpu/sod.rs:158-173's bar);
  - config 2, the 1024² disk: φ of the zero-padded 2048² FFT convolution against an f64 direct sum on a 128² subsample
    of target cells (rel L1 <= 1e-5, worst cell <= 1e-4), and one hydro + gravity step within 1e-5 per field;
  - config 3, the 2048² implicit-diffusion world: the first system's solution within 1e-6 (max norm, relative) of the
    twin's f64 Jacobi-PCG solve to 1e-12, and one implicit step's E within 1e-5 of the twin's."""
import os

import numpy as np
import pytest

import oracle as O
from sandbox_reactions_b200 import scenes
from sandbox_reactions_b200.engine import Step

pytestmark = pytest.mark.gpu


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)


@pytest.fixture(scope="module", autouse=True)
def all_host_threads():
    O.set_threads(os.cpu_count() or 1)


def test_the_2048_full_step_matches_the_twin():
    cfg, P, kappa = scenes.full_step(2048)
    with Step(cfg) as s:
        s.upload(P)
        s.upload_opacity(kappa)
        phi, gx, gy = s.gravity_field()
        s.run(1)
        gpu = s.readback()
        rep = s.read_heat()
        clock = s.read_dt()
    assert rep.converged and rep.rel_residual <= 1e-8, (rep.converged, rep.rel_residual)
    twin = O.Twin(cfg, P.astype(np.float64), kappa.astype(np.float64))
    ophi, ogx, ogy = twin.field()
    # φ to 1e-5; g to the reference's own GPU-vs-twin bar for the field, 1e-3 (tests/gpu/grav.rs:1-15): g is the
    # central difference of an FP32 φ near -420 (one ulp 3e-5) and is itself ~0.2, so it carries ~5e-5 of rounding
    assert rel_l1(phi, ophi) <= 1e-5, rel_l1(phi, ophi)
    assert rel_l1(gx, ogx) <= 1e-3 and rel_l1(gy, ogy) <= 1e-3, (rel_l1(gx, ogx), rel_l1(gy, ogy))
    twin.step(1)
    ref = twin.state()
    errs = [rel_l1(gpu[k], ref[k]) for k in range(4)]
    assert max(errs) <= 1e-5, errs
    assert abs(clock.sim_time - twin.clock()["sim_time"]) <= 1e-5 * twin.clock()["sim_time"]


def test_sod_512_one_step_and_two_hundred_steps():
    cfg, P = scenes.sod(512)
    with Step(cfg) as s:
        s.upload(P)
        s.run(1)
        one = s.readback()
        dt = s.read_dt().dt
        s.run(199)
        gpu = s.readback()
        clock = s.read_dt()
    ref, _ = O.hydro_step(cfg, P.astype(np.float64), dt)
    ref = O.floors(cfg, ref)
    errs = [rel_l1(one[k], ref[k]) for k in range(4) if np.abs(ref[k]).sum() > 0]
    assert max(errs) <= 1e-5, errs
    twin = O.Twin(cfg, P.astype(np.float64))
    twin.step(200)
    tref, tclock = twin.state(), twin.clock()
    assert rel_l1(gpu[0], tref[0]) <= 1e-3 and rel_l1(gpu[3], tref[3]) <= 1e-3
    assert abs(clock.sim_time - tclock["sim_time"]) <= 5e-4 * tclock["sim_time"]
    # the exact solution of the tube (interface at x = 256) at the GPU's clock, averaged over the rows
    R = O.Riemann(cfg.gamma, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
    t = clock.sim_time
    rho = gpu[0].astype(np.float64).mean(axis=0)
    exact = np.array([np.mean([R.sample((x - 256.0) / t)[0] for x in i + (np.arange(8) + 0.5) / 8])
                      for i in range(512)])
    assert np.abs(rho - exact).sum() / exact.sum() <= 0.02


def test_the_1024_disk_potential_matches_the_direct_sum():
    cfg, P = scenes.disk(1024)
    with Step(cfg.replace(hydro=False)) as s:
        s.upload(P)
        phi, _, _ = s.gravity_field()
    # reference/grav.rs:37-47: vacuum is no source (the f32 state compared with Σ_vac in f32, as on the device)
    src = np.where(P[0] >= np.float32(cfg.sigma_vac), P[0], 0.0).astype(np.float64)
    ty, tx = np.mgrid[4:1024:8, 4:1024:8]
    direct = O.direct_potential(cfg, src, tx.ravel(), ty.ravel())
    got = phi[ty.ravel(), tx.ravel()].astype(np.float64)
    assert rel_l1(got, direct) <= 1e-5, rel_l1(got, direct)
    assert (np.abs(got - direct) / np.abs(direct)).max() <= 1e-4


def test_the_1024_disk_step_matches_the_oracle():
    cfg, P = scenes.disk(1024)
    with Step(cfg) as s:
        s.upload(P)
        s.run(1)
        gpu = s.readback()
        dt = s.read_dt().dt
    P64 = P.astype(np.float64)
    _, gx, gy = O.grav_field(cfg, P64[0])
    ref, _ = O.hydro_step(cfg, P64, dt, (gx, gy))
    ref = O.floors(cfg, ref)
    errs = [rel_l1(gpu[k], ref[k]) for k in range(4)]
    assert max(errs) <= 1e-5, errs


def test_the_2048_fld_world_solves_and_steps_like_the_twin():
    cfg, P, kappa = scenes.fld(2048)
    P64, k64 = P.astype(np.float64), kappa.astype(np.float64)
    with Step(cfg) as s:
        s.upload(P)
        s.upload_opacity(kappa)
        _, rounds, rel, x = s.heat_first_solve(cfg.dt_fixed, "mg", want_x=True)
        s.run(1)
        gpu = s.readback()
        rep = s.read_heat()
    assert rel <= 1e-8 and rep.converged and rep.rel_residual <= 1e-8
    diag, rhs, kx, ky, gas = O.heat_system(cfg, P64, cfg.dt_fixed, k64)
    x_ref, _ = O.heat_pcg(diag, rhs, kx, ky, gas, rel=1e-12, max_rounds=200000)
    assert np.abs(x - x_ref)[gas].max() <= 1e-6 * np.abs(x_ref[gas]).max()
    ref, _, _, _ = O.heat_step(cfg, P64, cfg.dt_fixed, k64)
    assert rel_l1(gpu[3], ref[3]) <= 1e-5, rel_l1(gpu[3], ref[3])
