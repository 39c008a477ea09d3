"""The active box (crates/sr-engine/src/step/boxfit.rs, BoxMode::Fit) through the C ABI: a world whose gas fills a
small part of it steps only the box around the gas — the bounding box of Σ >= Σ_vac grown by 8 cells and rounded out to
multiples of 8, refit before step 0 and after every 16th step's P9, its FFT sized to the box — and gives the state the
whole world gives (BoxMode::WholeWorld; the reference's G-BOX compares the two), within the FP32 rounding of FFTs of
other sizes (rel L1 <= 1e-5 per field):

  - an expanding disk under gravity (leave edges) in a 384² world, 40 steps through three refits, the box growing with
    the gas; the first box and the refit cadence as boxfit.rs gives them;
  - the reference's cold disk in a 256² world: the box's steps against the twin's whole world;
  - the same disk under gravity and FLD (4 channels, κ plane), 20 steps;
  - the reference's cold disk in reference mode (14 channels) in a 256² world, 20 steps;
  - gas in a corner of the world (the box clamped at the edges) and a world of vacuum alone (no box: the whole world);
  - the box's step faster than the whole world's (4x at least) on a 2048² world whose gas fills a 144² box."""
import numpy as np
import pytest

import oracle as O
from sandbox_reactions_b200.abi import Config
from sandbox_reactions_b200.engine import Step
from sandbox_reactions_b200.scene import Scene

pytestmark = pytest.mark.gpu


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    d = np.abs(b).sum()
    return np.abs(a - b).sum() / d if d > 0 else np.abs(a).sum()


COLD_DISK_256 = """{"version": 1,
 "world": {"width": 256, "height": 256, "edge": "leave"},
 "slowdown": false,
 "switches": {"gravity": true, "hydro": true, "heat": false, "reactions": false, "neutrinos": false, "sinks": false},
 "objects": [
   {"kind": "disk", "x": 128, "y": 128, "a": 40, "sigma_c": 1.0, "t": 0.05, "composition": {"H": 1.0}, "v": [0, 0]}
 ],
 "overrides": {"k1e": 0, "k2e": 0, "k1n": 0, "k2n": 0}}"""


def disk_world(n, r=40.0, vr=0.6, cx=None, cy=None, sigma_c=1.0, t=0.5):
    """A disk of Σ_c sqrt(1 - r²/a²) expanding at vr (x r/a) in an n² world of vacuum at the floor state."""
    cx = n / 2 if cx is None else cx
    cy = n / 2 if cy is None else cy
    yy, xx = np.mgrid[0:n, 0:n] + 0.5
    dx, dy = xx - cx, yy - cy
    rr = np.hypot(dx, dy)
    inside = rr < r
    s = np.where(inside, sigma_c * np.sqrt(np.clip(1 - (rr / r) ** 2, 0, 1)) + 1e-3, 1e-8)
    ux = np.where(inside, vr * dx / r, 0.0)
    uy = np.where(inside, vr * dy / r, 0.0)
    e = np.where(inside, s * t + 0.5 * s * (ux * ux + uy * uy), 1e-8 * 0.05)
    P = np.stack([s, s * ux, s * uy, e]).astype(np.float32)
    cfg = Config(width=n, height=n, edge="leave", gravity=True, hydro=True, gamma=2.0, mu=1.0)
    return cfg, P


def run(cfg, P, steps, kappa=None, box=False, chunks=1, boxes=None):
    with Step(cfg.replace(active_box=box)) as s:
        s.upload(P)
        if kappa is not None:
            s.upload_opacity(kappa)
        if boxes is not None:
            boxes.append(s.read_box())
        for _ in range(chunks):
            s.run(steps // chunks)
            if boxes is not None:
                boxes.append(s.read_box())
        out = s.readback()
        clock = s.read_dt()
    return out, clock


def test_an_expanding_disk_steps_alike_in_its_box_and_in_the_whole_world():
    cfg, P = disk_world(384)
    whole, c0 = run(cfg, P, 40)
    boxes = []
    boxed, c1 = run(cfg, P, 40, box=True, chunks=4, boxes=boxes)  # 10 steps a call: refits fall inside calls too
    for k in range(4):
        assert rel_l1(boxed[k], whole[k]) <= 1e-5, (k, rel_l1(boxed[k], whole[k]))
    assert abs(c1.sim_time - c0.sim_time) <= 1e-6 * c0.sim_time
    # the first box: the disk's cells (|r| < 40 about 192) grown by 8 and rounded out to 8; the FFT sized to it
    b0 = boxes[0]
    assert (b0.x0, b0.y0, b0.w, b0.h) == (144, 144, 96, 96) and (b0.fft_w, b0.fft_h) == (256, 256)
    assert [b.fits for b in boxes] == [1, 2, 3, 3, 4]  # before step 0, after steps 0, 16 and 32
    assert boxes[-1].w >= b0.w and all(b.w % 8 == 0 and b.x0 % 8 == 0 for b in boxes)


def test_the_boxed_cold_disk_steps_like_the_twins_whole_world():
    # the reference's scenes/cold_disk.json laid down in a 256² world (4 channels, γ = 2, one μ): 3 steps of the box
    # against the twin's whole world from the same f32 start
    sc = Scene.parse(COLD_DISK_256)
    P, _ = sc.planes()
    cfg = sc.config()
    P4 = np.ascontiguousarray(P[:4])
    out, clock = run(cfg, P4, 3, box=True)
    twin = O.Twin(cfg, P4.astype(np.float64))
    twin.step(3)
    ref = twin.state()
    for k in range(4):
        assert rel_l1(out[k], ref[k]) <= 1e-5, (k, rel_l1(out[k], ref[k]))
    assert abs(clock.sim_time - twin.clock()["sim_time"]) <= 1e-5 * twin.clock()["sim_time"]


def test_the_box_with_fld_steps_like_the_whole_world():
    cfg, P = disk_world(256, r=36.0, vr=0.3, t=20.0)
    cfg = cfg.replace(heat=True, opacity_plane=True, mu=1.0)
    rng = np.random.default_rng(2)
    kappa = (1.0 + 0.5 * rng.random((256, 256))).astype(np.float32)
    whole, _ = run(cfg, P, 20, kappa)
    boxed, _ = run(cfg, P, 20, kappa, box=True)
    for k in range(4):
        assert rel_l1(boxed[k], whole[k]) <= 1e-5, (k, rel_l1(boxed[k], whole[k]))





def test_the_cold_disk_in_reference_mode_steps_alike_in_its_box():
    sc = Scene.parse(COLD_DISK_256)
    P, _ = sc.planes()
    cfg = sc.ref_config()
    whole, _ = run(cfg, P, 20)
    boxed, _ = run(cfg, P, 20, box=True)
    for k in range(14):
        assert rel_l1(boxed[k], whole[k]) <= 1e-5, (k, rel_l1(boxed[k], whole[k]))


def test_gas_in_a_corner_and_a_world_of_vacuum():
    cfg, P = disk_world(192, r=20.0, vr=0.2, cx=14.0, cy=170.0)
    whole, _ = run(cfg, P, 18)
    boxed, _ = run(cfg, P, 18, box=True)
    for k in range(4):
        assert rel_l1(boxed[k], whole[k]) <= 1e-5, (k, rel_l1(boxed[k], whole[k]))
    empty = np.zeros_like(P)
    empty[0] = 1e-8
    empty[3] = 1e-8 * 0.05
    out, clock = run(cfg.replace(gravity=False), empty, 3, box=True)
    assert np.allclose(out, empty, rtol=1e-6, atol=0.0) and clock.steps == 3


def test_the_box_steps_faster_than_the_whole_world():
    cfg, P = disk_world(2048, r=60.0, vr=0.1)
    cfg = cfg.replace(dt_fixed=0.05)
    ms = {}
    for box in (False, True):
        with Step(cfg.replace(active_box=box)) as s:
            s.upload(P)
            s.run(17)  # past the first refit, the graphs captured
            s.set_timing(1)
            s.run(16)
            ms[box] = s.read_cost().total_ms
    assert ms[True] * 4.0 < ms[False], ms


def test_the_boxed_world_answers_the_reads_of_the_whole_world():
    # heat on: the implicit step's report and face fluxes (the world's face planes, 0 outside the box), P2's field
    # inside the box, the clock; against the same world stepped whole
    cfg, P = disk_world(256, r=36.0, vr=0.3, t=20.0)
    cfg = cfg.replace(heat=True, opacity_plane=True, mu=1.0)
    rng = np.random.default_rng(4)
    kappa = (1.0 + 0.5 * rng.random((256, 256))).astype(np.float32)
    got = {}
    for box in (False, True):
        with Step(cfg.replace(active_box=box)) as s:
            s.upload(P)
            s.upload_opacity(kappa)
            s.run(5)
            got[box] = (s.read_heat(), s.read_heat_flux(), s.gravity_field(), s.read_dt(), s.read_box())
    (hw, fw, gw, dw, _), (hb, fb, gb, db, b) = got[False], got[True]
    assert hw.converged and hb.converged and hb.rel_residual <= 1e-8
    assert abs(db.sim_time - dw.sim_time) <= 1e-6 * dw.sim_time and db.steps == dw.steps == 5
    for k in range(2):
        assert rel_l1(fb[k], fw[k]) <= 1e-4, (k, rel_l1(fb[k], fw[k]))
    ys, xs = slice(b.y0, b.y0 + b.h), slice(b.x0, b.x0 + b.w)
    for k in range(3):
        assert rel_l1(gb[k][ys, xs], gw[k][ys, xs]) <= 1e-5, (k, rel_l1(gb[k][ys, xs], gw[k][ys, xs]))
        assert np.all(gb[k][:b.y0] == 0.0) and np.all(gb[k][b.y0 + b.h:] == 0.0)
