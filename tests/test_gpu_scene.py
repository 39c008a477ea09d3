"""Scenes loaded from scene-file text and stepped on the GPU against the oracle's twin on the same Config and planes:
a two-gas shock tube (hydro, bounce edges), a hot square in a helium sheet (the implicit FLD solve alone, the
reference's opacity kappa0 (1 + X_H) as a plane), and a cold Maclaurin disk (gravity + hydro, leave edges). Each
with the reference's cold pressure switched off, as its own test scenes do. Tolerance: rel L1 <= 1e-5 per field."""
import numpy as np
import pytest

import oracle as O
from sandbox_reactions_b200 import scene as S
from sandbox_reactions_b200.engine import Step

pytestmark = pytest.mark.gpu

COLD_OFF = '"overrides": {"k1e": 0, "k2e": 0, "k1n": 0, "k2n": 0}'
QUIET = '"reactions": false, "neutrinos": false, "sinks": false'

TUBE = ('{"version": 1, "world": {"width": 128, "height": 64, "edge": "bounce"},'
        f' "switches": {{"gravity": false, "hydro": true, "heat": false, {QUIET}}},'
        ' "objects": ['
        '  {"kind": "rect", "x0": 0, "y0": 0, "w": 64, "h": 64, "sigma": 1.0, "pressure": 1.0, "composition": {"H": 1}},'
        '  {"kind": "rect", "x0": 64, "y0": 0, "w": 64, "h": 64, "sigma": 0.125, "pressure": 0.1,'
        '   "composition": {"He": 1}, "v": [0, 0.25]}],'
        f' {COLD_OFF}}}')

HOT_SQUARE = ('{"version": 1, "world": {"width": 64, "height": 64, "edge": "leave"},'
              f' "switches": {{"gravity": false, "hydro": false, "heat": true, {QUIET}}},'
              ' "objects": ['
              '  {"kind": "rect", "x0": 0, "y0": 0, "w": 64, "h": 64, "sigma": 1e-4, "t": 0.05,'
              '   "composition": {"He": 1}},'
              '  {"kind": "disk", "x": 40.5, "y": 20, "a": 6, "sigma_c": 1e-4, "t": 2.0, "composition": {"He": 1}}],'
              f' {COLD_OFF}}}')

DISK = ('{"version": 1, "world": {"width": 128, "height": 128, "edge": "leave"},'
        f' "switches": {{"gravity": true, "hydro": true, "heat": false, {QUIET}}},'
        ' "objects": [{"kind": "disk", "x": 60, "y": 66, "a": 36, "sigma_c": 1.0, "t": 0.05,'
        '  "composition": {"H": 0.75, "He": 0.25}, "v": [0.01, 0]}],'
        f' {COLD_OFF}}}')


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300)


@pytest.mark.parametrize("name,text,steps", [("tube", TUBE, 3), ("hot_square", HOT_SQUARE, 1), ("disk", DISK, 2)])
def test_a_loaded_scene_steps_like_the_twin(name, text, steps):
    sc = S.parse(text)
    cfg = sc.config()
    with Step(cfg) as s:
        planes = S.load_into(s, sc)
        dts = []
        for _ in range(steps):
            s.run(1)
            dts.append(s.read_dt().dt)
        gpu = s.readback()
        if cfg.heat:
            rep = s.read_heat()
            assert rep.converged and rep.rel_residual <= 1e-8
    kappa = S.Scene.opacity(planes, sc.physics()).astype(np.float64) if cfg.heat else None
    twin = O.Twin(cfg, planes[:4].astype(np.float64), kappa)
    for dt in dts:
        twin.step(1)
        assert abs(twin.clock()["dt"] - dt) <= 1e-6 * dt, (name, twin.clock()["dt"], dt)
    P = twin.state()
    for k in range(4):
        if np.abs(P[k]).sum() == 0.0:
            assert np.abs(gpu[k]).max() == 0.0, (name, k)
            continue
        assert rel_l1(gpu[k], P[k]) <= 1e-5, (name, k, rel_l1(gpu[k], P[k]))
    if cfg.heat:  # the hot spot spread: the step did something
        assert rel_l1(gpu[3], planes[3]) > 1e-3
