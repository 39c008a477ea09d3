"""A run stopped and resumed through the records a dump carries beyond the cells — dump_state / load_dump
(crates/sr-engine/src/dump.rs:355-410): the clock (Step::restore, step/latch.rs:493-510), P5's rate (Step::heat_rate /
set_heat_rate, step/heat.rs:550-582), the side flux F the next P4 pushes with (step/heat.rs:584-589) and the hold's
mask — steps on as the run would have, through the C ABI:

  - a reference-mode run with P5 and the radiation force, dumped after 3 steps (through the SRDUMP01 bytes) and
    resumed in a new context, against the same run stepped on: rel L1 <= 1e-5 per field after 3 more steps (the dump
    holds Δt in f32 and the rate in f32, the run's own in f64), the same step index and sim time;
  - the same state uploaded without the records steps further from the run (its first step pushes with F = 0, its
    implicit step starts cold);
  - a boxed FLD world (4 channels, the active box) resumed from its state, rate and clock after 20 steps: within
    1e-5 after 16 more, the refit after step index 32 where the run refit, the rate read back as set;
  - the clock restored and stepped on; the calls refused where their pass does not run."""
import numpy as np
import pytest

from sandbox_reactions_b200 import dump as D
from sandbox_reactions_b200.abi import Config
from sandbox_reactions_b200.engine import SrError, Step
from sandbox_reactions_b200.scene import Scene

pytestmark = pytest.mark.gpu

HOT_DISK = """{"version": 1,
 "world": {"width": 96, "height": 96, "edge": "leave"},
 "slowdown": false,
 "switches": {"gravity": true, "hydro": true, "heat": true, "reactions": false, "neutrinos": false, "sinks": false},
 "objects": [
   {"kind": "rect", "x0": 0, "y0": 0, "w": 96, "h": 96, "sigma": 2e-3, "t": 1.0, "composition": {"H": 1.0},
    "v": [0, 0]},
   {"kind": "disk", "x": 48, "y": 48, "a": 30, "sigma_c": 1.0, "t": 40.0,
    "composition": {"H": 0.7346, "He": 0.2485, "C": 0.0092, "O": 0.0077}, "v": [0.05, 0.02]},
   {"kind": "disk", "x": 40, "y": 52, "a": 6, "sigma_c": 2.0, "t": 400.0, "composition": {"He": 1.0}, "v": [0, 0]}
 ]}"""


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.abs(b).sum()
    return np.abs(a - b).sum() / d if d > 0 else np.abs(a).sum()


def gap(got, want):
    """The worst of Σ, Σu, Σv, E by rel L1 and of the species by their mass Σ·X against the total mass."""
    worst = max(rel_l1(got[k], want[k]) for k in range(4))
    if got.shape[0] > 4:
        m = np.abs(want[0].astype(np.float64)).sum()
        for k in range(4, got.shape[0]):
            worst = max(worst, np.abs(got[0] * got[k] - want[0] * want[k]).sum() / m)
    return worst


def test_a_reference_run_resumed_from_its_dump_steps_on_as_it_would_have():
    sc = Scene.parse(HOT_DISK)
    P, _ = sc.planes()
    cfg = sc.ref_config(strict=False).replace(heat=True)
    with Step(cfg) as a:
        a.upload(P)
        a.run(3)
        d = D.from_bytes(D.save_from(a).to_bytes())
        a.run(3)
        want, wclock, wheat = a.readback(), a.read_dt(), a.read_heat()
    assert d.step == 3 and d.flux is not None and d.rate is not None
    assert np.abs(d.flux).max() > 0 and np.abs(d.rate).max() > 0
    with Step(cfg) as b:
        D.load_into(b, d)
        c0 = b.read_dt()
        assert c0.steps == 3 and c0.sim_time == d.sim_time and c0.dt_next == np.float32(d.dt_next)
        assert np.array_equal(b.read_heat_rate(), d.rate)
        fx, fy = b.read_side_flux()
        assert np.array_equal(fx, d.flux[0]) and np.array_equal(fy, d.flux[1])
        b.run(3)
        got, gclock, gheat = b.readback(), b.read_dt(), b.read_heat()
    resumed = gap(got, want)
    assert resumed <= 1e-5, resumed
    assert gclock.steps == wclock.steps == 6
    assert abs(gclock.sim_time - wclock.sim_time) <= 1e-6 * wclock.sim_time
    assert abs(gheat.passes - wheat.passes) <= 1, (gheat.passes, wheat.passes)
    # the cells alone: the first step pushes with F = 0 and its implicit step starts from a zero rate
    with Step(cfg) as c:
        c.upload(d.planes)
        c.run(3)
        cold = gap(c.readback(), want)
    assert cold > resumed, (cold, resumed)


def disk_world(n, r=36.0, vr=0.3, t=20.0):
    yy, xx = np.mgrid[0:n, 0:n] + 0.5
    dx, dy = xx - n / 2, yy - n / 2
    rr = np.hypot(dx, dy)
    inside = rr < r
    s = np.where(inside, np.sqrt(np.clip(1 - (rr / r) ** 2, 0, 1)) + 1e-3, 1e-8)
    ux = np.where(inside, vr * dx / r, 0.0)
    uy = np.where(inside, vr * dy / r, 0.0)
    e = np.where(inside, s * t + 0.5 * s * (ux * ux + uy * uy), 1e-8 * 0.05)
    P = np.stack([s, s * ux, s * uy, e]).astype(np.float32)
    cfg = Config(width=n, height=n, edge="leave", gravity=True, hydro=True, heat=True, opacity_plane=True, gamma=2.0,
                 mu=1.0, active_box=True)
    kappa = (1.0 + 0.5 * np.random.default_rng(5).random((n, n))).astype(np.float32)
    return cfg, P, kappa


def test_a_boxed_fld_run_resumed_from_its_state_rate_and_clock():
    cfg, P, kappa = disk_world(256)
    with Step(cfg) as a:
        a.upload(P)
        a.upload_opacity(kappa)
        a.run(20)
        state, rate, clock = a.readback(), a.read_heat_rate(), a.read_dt()
        a.run(16)
        want, wbox, wclock = a.readback(), a.read_box(), a.read_dt()
    assert np.abs(rate).max() > 0
    with Step(cfg) as b:
        b.upload(state)
        b.upload_opacity(kappa)
        b.set_heat_rate(rate)
        b.set_clock(clock.steps, clock.sim_time, clock.dt, clock.dt_next)
        assert np.array_equal(b.read_heat_rate(), rate)
        b.run(16)
        got, gbox, gclock = b.readback(), b.read_box(), b.read_dt()
    assert gap(got, want) <= 1e-5, gap(got, want)
    assert gclock.steps == wclock.steps == 36 and abs(gclock.sim_time - wclock.sim_time) <= 1e-6 * wclock.sim_time
    # both refit after the step of index 32 (the 33rd), to the same state's box; the resumed run fit once before
    assert (gbox.x0, gbox.y0, gbox.w, gbox.h) == (wbox.x0, wbox.y0, wbox.w, wbox.h)
    assert gbox.fits == 2 and wbox.fits == 4


def test_the_clock_restored_runs_on():
    cfg = Config(width=64, height=64, edge="leave", hydro=True, gamma=1.4, mu=1.0)
    P = np.zeros((4, 64, 64), np.float32)
    P[0] = 1.0
    P[3] = 2.5
    with Step(cfg) as s:
        s.upload(P)
        s.set_clock(7, 1.25, 0.01, 0.02)
        c = s.read_dt()
        assert (c.steps, c.sim_time, c.dt, c.dt_next) == (7, 1.25, 0.01, 0.02)
        s.run(1)
        c = s.read_dt()
        assert c.steps == 8 and c.dt == 0.02 and abs(c.sim_time - 1.27) <= 1e-15
        for bad in ((7, 1.25, 0.01, 0.0), (2 ** 32, 1.0, 0.01, 0.02), (7, float("nan"), 0.01, 0.02)):
            with pytest.raises(SrError):
                s.set_clock(*bad)


def test_the_rate_and_the_side_flux_need_their_passes():
    P = np.zeros((4, 64, 64), np.float32)
    P[0] = 1.0
    P[3] = 2.5
    with Step(Config(width=64, height=64, hydro=True, heat=False)) as s:
        s.upload(P)
        with pytest.raises(SrError, match="no heat pass"):
            s.read_heat_rate()
        with pytest.raises(SrError, match="no heat pass"):
            s.set_heat_rate(None)
    with Step(Config(width=64, height=64, hydro=True, heat=True)) as s:
        s.upload(P)
        with pytest.raises(SrError, match="reference mode"):
            s.read_side_flux()
        r = np.full((64, 64), 0.5, np.float32)
        s.set_heat_rate(r)
        assert np.array_equal(s.read_heat_rate(), r)
        s.set_heat_rate(None)
        assert not s.read_heat_rate().any()
