"""The CUDA hydro (P4) and gravity (P2) passes, called through the C ABI, against the oracle from the same f32 start
(the reference's GPU-vs-twin tier: crates/sr-engine/tests/gpu/cpu_gpu.rs, grav.rs, sod.rs).

Tolerances: one step from a shared start, rel L1 <= 1e-5 per field (the per-step parity bar); gravity's φ and g rel L1
<= 1e-5 (an FP32 FFT against the f64 one); 200 steps of Sod within the reference's G-REF bands (rel L1 <= 1e-3)."""
import numpy as np
import pytest

import oracle as O
from sandbox_reactions_b200 import scenes
from sandbox_reactions_b200.abi import Config
from sandbox_reactions_b200.engine import SrError, Step

pytestmark = pytest.mark.gpu


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)


def smooth_state(w, h, seed=0, gamma=2.0, vacuum=False):
    rng = np.random.default_rng(seed)
    j, i = np.mgrid[0:h, 0:w].astype(np.float64)
    sigma = 1.0 + 0.5 * np.sin(2 * np.pi * i / w) * np.cos(2 * np.pi * j / h) + 0.1 * rng.random((h, w))
    u = 0.3 * np.cos(2 * np.pi * j / h) + 0.05 * rng.standard_normal((h, w))
    v = -0.2 * np.sin(2 * np.pi * i / w) + 0.05 * rng.standard_normal((h, w))
    p = 1.0 + 0.3 * rng.random((h, w))
    if vacuum:
        sigma[: h // 4, : w // 4] = 1e-9
        u[: h // 4, : w // 4] = 0.0
        v[: h // 4, : w // 4] = 0.0
    P = np.zeros((4, h, w))
    P[0], P[1], P[2] = sigma, sigma * u, sigma * v
    P[3] = p / (gamma - 1.0) + 0.5 * sigma * (u * u + v * v)
    return P.astype(np.float32)


def one_step_pair(cfg, P32):
    """One GPU step and one oracle step from the same f32 planes on the GPU's Δt."""
    with Step(cfg) as s:
        s.upload(P32)
        s.run(1)
        gpu = s.readback().astype(np.float64)
        dt = s.read_dt().dt
    P = P32.astype(np.float64)
    g = None
    if cfg.gravity:
        _, gx, gy = O.grav_field(cfg, P[0])
        g = (gx, gy)
    ref, _ = O.hydro_step(cfg, P, dt, g)
    ref = O.floors(cfg, ref)
    return gpu, ref, dt


@pytest.mark.parametrize("edge", ["bounce", "leave"])
@pytest.mark.parametrize("limiter", ["mc", "minmod"])
def test_one_hydro_step_matches_the_oracle(edge, limiter):
    cfg = Config(width=96, height=64, edge=edge, limiter=limiter, gamma=1.4)
    gpu, ref, _ = one_step_pair(cfg, smooth_state(96, 64, 1, 1.4))
    for k in range(4):
        assert rel_l1(gpu[k], ref[k]) <= 1e-5, (k, rel_l1(gpu[k], ref[k]))


def test_one_step_with_vacuum_and_a_ragged_tile_edge():
    # 400 x 40: neither axis a multiple of the 32 x 8 tile's width; a vacuum corner exercises the floor state
    cfg = Config(width=400, height=40, edge="bounce", gamma=2.0)
    gpu, ref, _ = one_step_pair(cfg, smooth_state(400, 40, 2, 2.0, vacuum=True))
    for k in range(4):
        assert rel_l1(gpu[k], ref[k]) <= 1e-5, (k, rel_l1(gpu[k], ref[k]))


def test_sod_two_hundred_steps_stays_on_the_twin():
    cfg, P = scenes.sod(64)
    with Step(cfg) as s:
        s.upload(P)
        s.run(200)
        gpu = s.readback()
        clock = s.read_dt()
    twin = O.Twin(cfg, P.astype(np.float64))
    twin.step(200)
    ref = twin.state()
    assert rel_l1(gpu[0], ref[0]) <= 1e-3 and rel_l1(gpu[3], ref[3]) <= 1e-3
    assert abs(clock.sim_time - twin.clock()["sim_time"]) <= 5e-4 * twin.clock()["sim_time"]
    assert clock.steps == 200


def test_the_strip_along_y_runs_as_along_x():
    cfg = Config(width=64, height=32, edge="bounce", gamma=2.0)
    P = smooth_state(64, 32, 3)
    Pt = np.stack([P[0].T, P[2].T, P[1].T, P[3].T]).copy()
    with Step(cfg) as a, Step(cfg.replace(width=32, height=64)) as b:
        a.upload(P)
        b.upload(Pt)
        a.run(10)
        b.run(10)
        A, B = a.readback(), b.readback()
    assert rel_l1(A[0], B[0].T) <= 1e-5 and rel_l1(A[3], B[3].T) <= 1e-5


def test_reruns_are_bit_identical():
    cfg, P = scenes.disk(64)
    out = []
    for _ in range(2):
        with Step(cfg) as s:
            s.upload(P)
            s.run(5)
            out.append(s.readback())
    assert np.array_equal(out[0], out[1])


def test_gravity_field_matches_the_oracle_for_both_kernels():
    for kernel in ("self_cell", "softened"):
        cfg, P = scenes.disk(128)
        cfg = cfg.replace(kernel=kernel, hydro=False)
        with Step(cfg) as s:
            s.upload(P)
            phi, gx, gy = s.gravity_field()
        ophi, ogx, ogy = O.grav_field(cfg, P[0].astype(np.float64))
        assert rel_l1(phi, ophi) <= 1e-5
        assert rel_l1(gx, ogx) <= 1e-5 and rel_l1(gy, ogy) <= 1e-5


def test_gravity_on_a_wide_and_a_tall_world():
    for w, h in ((256, 32), (32, 256)):
        rng = np.random.default_rng(w)
        P = smooth_state(w, h, 4)
        P[0] *= rng.random((h, w)) < 0.5
        cfg = Config(width=w, height=h, gravity=True, hydro=False)
        with Step(cfg) as s:
            s.upload(P)
            phi, gx, gy = s.gravity_field()
        ophi, ogx, ogy = O.grav_field(cfg, P[0].astype(np.float64))
        assert rel_l1(phi, ophi) <= 1e-5 and rel_l1(gx, ogx) <= 1e-5 and rel_l1(gy, ogy) <= 1e-5


def test_maclaurin_disk_force_on_the_gpu():
    a, side = 40.0, 128
    j, i = np.mgrid[0:side, 0:side]
    c = side // 2
    r2 = ((i - c) ** 2 + (j - c) ** 2) / a ** 2
    P = np.zeros((4, side, side), np.float32)
    P[0] = np.where(r2 < 1, np.sqrt(np.clip(1 - r2, 0, None)), 0.0)
    P[3] = 1.0
    cfg = Config(width=side, height=side, gravity=True, hydro=False, sigma_vac=1e-30)
    with Step(cfg) as s:
        s.upload(P)
        _, gx, gy = s.gravity_field()
    k = np.pi ** 2 / (2 * a)
    dx, dy = i - c, j - c
    r = np.hypot(dx, dy)
    m = (r > 0) & (r <= 0.75 * a)
    err = np.sqrt((gx + k * dx) ** 2 + (gy + k * dy) ** 2)[m] / (k * r[m])
    assert err.max() <= 0.02


def test_one_hydro_gravity_step_matches_the_oracle():
    cfg, P = scenes.disk(128)
    gpu, ref, _ = one_step_pair(cfg, P)
    for k in range(4):
        assert rel_l1(gpu[k], ref[k]) <= 1e-5, (k, rel_l1(gpu[k], ref[k]))


def test_refusals_are_errors_not_crashes():
    with pytest.raises(SrError, match="multiple of 8"):
        Step(Config(width=100, height=64))
    with pytest.raises(SrError, match="gamma"):
        Step(Config(gamma=1.0))
    with Step(Config()) as s:
        with pytest.raises(SrError, match="no state uploaded"):
            s.run(1)
        with pytest.raises(SrError, match="planes of shape"):
            s.upload(np.zeros((4, 8, 8), np.float32))


def test_a_non_finite_state_is_reported_with_its_cell_and_channel():
    cfg = Config(width=64, height=64)
    P = smooth_state(64, 64, 5)
    P[3, 10, 20] = np.nan
    with Step(cfg) as s:
        s.upload(P)
        with pytest.raises(SrError) as e:
            s.run(1)
        assert e.value.status == 2
        nf = s.read_dt().non_finite
    assert nf is not None
