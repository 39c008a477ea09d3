"""Scene files (crates/sr-engine/src/scene.rs; its tests in crates/sr-engine/tests/gpu/scene.rs): the refusals by path,
where objects land, the energy `t` and `pressure` give through the EOS, a disk's mass against the Maclaurin integral,
physics.json's bounds on overrides, the cold-energy table against its closed form, every file of the reference's
scenes/ folder (read from the reference tree when it is present), and the mapping onto this build's Config."""
import json
import math
import os

import numpy as np
import pytest

from sandbox_reactions_b200 import scene as S

# the reference project's scenes/ folder, when SR_REFERENCE_DIR names a checkout of it (else these tests skip)
REF_SCENES = os.path.join(os.environ.get("SR_REFERENCE_DIR", ""), "scenes") if os.environ.get("SR_REFERENCE_DIR") else ""
MIX = '"composition": {"H": 0.7346, "He": 0.2485, "O": 0.0077, "C": 0.0092}'


def base(marker="", extra=""):
    """A scene holding every level a key can sit at; `extra` is spliced into the level its marker names."""
    at = lambda m: extra if m == marker else ""
    return (f'{{{at("@top")} "version": 1,'
            f' "world": {{{at("@world")} "width": 64, "height": 64, "edge": "leave"}},'
            f' "slowdown": true,'
            f' "switches": {{{at("@switches")} "gravity": true, "hydro": true, "heat": true, "reactions": true,'
            f' "neutrinos": true, "sinks": true}},'
            f' "test": {{{at("@test")} "pin_temperature": false, "constant_diffusivity": null, "flux_limiter": true}},'
            f' "objects": ['
            f'  {{{at("@disk")} "kind": "disk", "x": 32, "y": 32, "a": 10, "sigma_c": 0.5, "t": 2.0,'
            f'   "composition": {{{at("@composition")} "H": 0.7346, "He": 0.2485, "O": 0.0077, "C": 0.0092}},'
            f'   "v": [0, 0]}},'
            f'  {{{at("@rect")} "kind": "rect", "x0": 0, "y0": 0, "w": 64, "h": 4, "sigma": 1.0, "pressure": 100.0,'
            f'   "composition": {{"H": 1.0}}, "v": [0, 0]}},'
            f'  {{{at("@preset")} "kind": "preset", "preset": "sun", "x": 32, "y": 32}}'
            f' ],'
            f' "overrides": {{{at("@overrides")} "cfl": 0.3}}}}')


def edit(change):
    """The base scene with `change` applied to its parsed JSON."""
    d = json.loads(base())
    change(d)
    return json.dumps(d)


def refused(text, words):
    with pytest.raises(S.SceneError) as e:
        S.parse(text)
    assert words in str(e.value), str(e.value)
    return str(e.value)


def one(obj, world=(64, 64), extra=""):
    return S.parse(f'{{"version": 1, "world": {{"width": {world[0]}, "height": {world[1]}}}{extra},'
                   f' "objects": [{obj}]}}')


def planes_of(sc, world=None):
    p, warnings = sc.planes(world)
    assert warnings == []
    return p


def test_unknown_keys_are_refused_at_every_level():
    sc = S.parse(base())
    assert len(sc.objects) == 3 and sc.overrides == [("cfl", 0.3)]
    for marker, extra, words in [
        ("@switches", '"hydor": false,', "switches.hydor: unknown key"),
        ("@top", '"colour": 1,', "colour: unknown key"),
        ("@world", '"depth": 8,', "world.depth: unknown key"),
        ("@test", '"pin_temp": true,', "test.pin_temp: unknown key"),
        ("@disk", '"radius": 3,', "objects[0].radius: unknown key"),
        ("@composition", '"Hx": 0.0,', "objects[0].composition.Hx: unknown key"),
        ("@rect", '"colour": 1,', "objects[1].colour: unknown key"),
        ("@preset", '"mass": 1,', "objects[2].mass: unknown key"),
    ]:
        refused(base(marker, extra), words)


def test_t_and_pressure_are_one_or_the_other():
    refused(base("@disk", '"pressure": 1.0,'), "objects[0]: takes t or pressure, not both")
    refused(base().replace('"pressure": 100.0,', ""), "objects[1]: needs t or pressure")
    refused(base("@rect", '"t": 1.0,'), "objects[1]: takes t or pressure, not both")


def test_every_other_departure_is_refused_by_path():
    refused("{", "not JSON")
    refused('{"version": 1, "world": {"width": 64, "height": 64}, "objects": [], "x": NaN}', "not JSON")
    refused("[1, 2]", "the scene: must be an object")
    refused(base().replace('"version": 1', '"version": 2'), "version: must be 1")
    refused(base().replace('"version": 1', '"version": 1.0'), "version: must be 1")
    refused(base().replace('"width": 64,', '"width": 60,'), "world: world 60 × 64: width and height must be")
    refused(base().replace('"width": 64,', '"width": 64.0,'), "world.width: must be a whole number")
    refused(base().replace('"width": 64,', '"width": -8,'), "world.width: out of range")
    refused(base().replace('"edge": "leave"', '"edge": "wrap"'), 'world.edge must be "leave" or "bounce", got "wrap"')
    refused(base().replace('"slowdown": true', '"slowdown": 1'), "slowdown: must be true or false")
    refused(base().replace('"hydro": true', '"hydro": "yes"'), "switches.hydro: must be true or false")
    refused(base().replace('"constant_diffusivity": null', '"constant_diffusivity": 0'),
            "test.constant_diffusivity: must be > 0, got 0")
    refused(edit(lambda d: d.update(objects={"a": 1})), "objects: must be a list")
    refused(base().replace('"kind": "disk"', '"kind": "ring"'), 'objects[0].kind: must be "preset", "disk" or "rect"')
    refused(base().replace('"preset": "sun"', '"preset": "moon"'),
            'objects[2].preset: unknown preset "moon" (known: sun, massive, giant)')
    refused(base().replace('"a": 10', '"a": -1'), "objects[0].a: must be > 0, got -1")
    refused(base().replace('"sigma_c": 0.5', '"sigma_c": "big"'), "objects[0].sigma_c: must be a finite number")
    refused(base().replace('"x": 32, "y": 32, "a"', '"y": 32, "a"'), "objects[0].x: missing")
    refused(base().replace('"w": 64, "h": 4', '"w": 0, "h": 4'), "objects[1]: w and h must be ≥ 1, got 0 × 4")
    refused(base().replace('"x0": 0, "y0": 0', '"x0": 0.5, "y0": 0'), "objects[1].x0: must be a whole number")
    refused(base().replace('"He": 0.2485', '"He": 0.3'), "objects[0].composition: the fractions sum to")
    refused(base().replace('"He": 0.2485', '"He": -0.2485'), "objects[0].composition.He: must be a number ≥ 0")
    refused(base().replace('"composition": {"H": 1.0}', '"composition": [1]'),
            "objects[1].composition: must be an object of mass fractions")
    refused(base().replace('"v": [0, 0]}', '"v": [0]}', 1), "objects[0].v: must be [vx, vy], two finite numbers")
    refused(base().replace('"cfl": 0.3', '"cfl": "fast"'), "overrides.cfl: must be a number")
    refused(edit(lambda d: d.update(overrides=["cfl"])), "overrides: must be an object of physics.json keys")


def test_overrides_are_physics_keys_within_their_bounds():
    refused(base("@overrides", '"gravity_const": 2.0,'), "overrides.gravity_const: unknown key (physics.json keys only)")
    msg = refused(base().replace('"cfl": 0.3', '"cfl": -1.0'), "overrides: physics.json: cfl: must be > 0, got -1")
    assert "overrides" in msg and "cfl" in msg
    refused(base().replace('"cfl": 0.3', '"k1e": 0'), "physics.json: k1e: must be > 0 while k2e is")
    refused(base().replace('"cfl": 0.3', '"t_he": 50'), "physics.json: t_he: must be > t_h = 56 (K6), got 50")
    refused(base().replace('"cfl": 0.3', '"block": 2.5'), "physics.json: block: must be a whole number ≥ 1, got 2.5")
    refused(base().replace('"cfl": 0.3', '"nu_c_burn": 3'), "physics.json: nu_c_burn: must be ≥ 4")
    refused(base().replace('"cfl": 0.3', '"m_nu": 40'), "physics.json: m_nu: must be < nu_c_burn = 30")
    refused(base().replace('"cfl": 0.3', '"kappa_dust": 1'), "physics.json: kappa_dust: must be 0 while S1 is off")
    refused(base().replace('"cfl": 0.3', '"k2n": 20'), "physics.json: k2n: m_tov / m_ch must be in [1.4, 2.0]")
    pair_off = S.parse(base().replace('"cfl": 0.3', '"k1e": 0, "k2e": 0'))
    assert not pair_off.writes_calibration() and pair_off.physics().get("k1e") == 0.0
    plain = S.parse(base().replace(', "overrides": { "cfl": 0.3}', ""))
    assert plain.overrides == [] and plain.writes_calibration()
    assert plain.physics() == S.Physics.shipped()
    S.Physics.shipped().validate()


def test_objects_land_where_the_reference_puts_them():
    floor = np.float32(S.Physics.shipped().get("sigma_floor"))
    rect = one('{"kind": "rect", "x0": 8, "y0": 16, "w": 3, "h": 2, "sigma": 0.25, "t": 1.0, "composition": {"H": 1}}')
    p = planes_of(rect)[0]
    lit = [(int(x), int(y)) for y, x in zip(*np.nonzero(p != floor))]
    assert lit == [(8, 16), (9, 16), (10, 16), (8, 17), (9, 17), (10, 17)]
    disk = one('{"kind": "disk", "x": 20, "y": 40, "a": 1, "sigma_c": 1, "t": 1, "composition": {"H": 1}}')
    p = planes_of(disk)[0]
    lit = [(int(x), int(y)) for y, x in zip(*np.nonzero(p != floor))]
    assert lit == [(19, 39), (20, 39), (19, 40), (20, 40)]
    assert abs(p[39, 19] - math.sqrt(0.5)) < 1e-6
    # a wider world keeps the objects where they stood relative to the centre: (+32, +8) for 128 x 80
    p = planes_of(rect, (128, 80))[0]
    assert p[24, 40] > 0 and p[25, 42] > floor and p[25, 43] == floor
    two = S.parse('{"version": 1, "world": {"width": 64, "height": 64}, "objects": ['
                  '{"kind": "rect", "x0": 0, "y0": 0, "w": 2, "h": 1, "sigma": 0.3, "t": 1, "composition": {"H": 1},'
                  ' "v": [1, 0]},'
                  '{"kind": "rect", "x0": 1, "y0": 0, "w": 2, "h": 1, "sigma": 0.1, "t": 1, "composition": {"He": 1},'
                  ' "v": [0, -2]}]}')
    p = planes_of(two).reshape(14, -1)
    assert abs(p[0, 1] - 0.4) < 1e-7 and abs(p[1, 1] - 0.3) < 1e-7 and abs(p[2, 1] + 0.2) < 1e-7
    assert abs(p[4, 1] - 0.75) < 1e-7 and abs(p[5, 1] - 0.25) < 1e-7
    assert (p[0, 5], p[1, 5], p[2, 5], p[4, 5], p[5, 5]) == (floor, 0.0, 0.0, 1.0, 0.0)
    # the floor's energy: Sigma_floor of hydrogen (mu = 1/2) at T_floor, and no cold energy with the pairs off
    off = S.parse(f'{{"version": 1, "world": {{"width": 64, "height": 64}}, "objects": [],'
                  f' "overrides": {{"k1e": 0, "k2e": 0, "k1n": 0, "k2n": 0}}}}')
    assert planes_of(off).reshape(14, -1)[3, 0] == np.float32(1e-8 * (0.05 / 0.5))
    gone = one('{"kind": "disk", "x": 500, "y": 500, "a": 5, "sigma_c": 1, "t": 1, "composition": {"H": 1}}')
    assert gone.planes()[1] == ["objects[0] covers no cell of the 64x64 world"]


def test_t_and_pressure_set_the_energy_through_the_eos():
    phys = S.Physics.shipped()
    eos = S.Eos(phys)
    inv_mu, y_e, _ = S.composition(S.SUN_MIX)
    mu = 1.0 / inv_mu
    assert abs(inv_mu - 1.66527292) < 1e-8 and abs(y_e - 0.8673) < 1e-12  # registry.rs's hand values
    hot = one(f'{{"kind": "rect", "x0": 0, "y0": 0, "w": 1, "h": 1, "sigma": 2.0, "t": 3.0, {MIX}, "v": [0.5, -1.5]}}')
    e = float(planes_of(hot).reshape(14, -1)[3, 0])
    want = 2.0 * (3.0 / mu + float(eos.eps_cold(2.0, y_e, 0.0))) + 0.5 * 2.0 * (0.25 + 2.25)
    assert abs(e - want) <= 1e-6 * want
    pressed = one(f'{{"kind": "rect", "x0": 0, "y0": 0, "w": 1, "h": 1, "sigma": 2.0, "pressure": 500.0, {MIX}}}')
    eps_th = float(planes_of(pressed).reshape(14, -1)[3, 0]) / 2.0 - float(eos.eps_cold(2.0, y_e, 0.0))
    pi = 2.0 * eps_th + float(eos.pi_e(2.0, y_e))
    assert abs(pi - 500.0) <= 1e-5 * 500.0
    low = one(f'{{"kind": "rect", "x0": 3, "y0": 5, "w": 1, "h": 1, "sigma": 2.0, "pressure": 1e-6, {MIX}}}')
    with pytest.raises(S.SceneError) as err:
        low.planes()
    assert "objects[0].pressure" in str(err.value) and "cell (3, 5)" in str(err.value)


def test_the_cold_energy_table_follows_its_closed_form():
    """u(x) = x 2 (K2^2 / K1) (y - ln(1 + y)), y = (K1 / K2) sqrt x (eos.rs:48-66), against the tabulated u."""
    for k1, k2 in ((21.3, 134.0), (2.67, 58.2)):
        t = S.ColdTable(k1, k2)
        for x in (1e-10, 1e-6, 1e-2, 1.0, 30.0, 1e4, 1e7):
            y = k1 / k2 * math.sqrt(x)
            exact = x * 2.0 * k2 * k2 / k1 * (y - math.log1p(y))
            assert abs(float(t.u(np.array([x]))[0]) / exact - 1.0) < 1e-4, (k1, x)
        lo, hi = 1e-12, 1e16
        assert abs(float(S.cold_pressure(lo, k1, k2)) / (k1 * lo * lo) - 1.0) < 1e-6
        assert abs(float(S.cold_pressure(hi, k1, k2)) / (k2 * hi ** 1.5) - 1.0) < 1e-6


@pytest.mark.parametrize("x,y,a,sc", [(300.0, 200.0, 40.0, 1.0), (100.3, 57.8, 12.0, 0.5), (420.0, 300.25, 25.5, 2.0),
                                      (300.5, 200.5, 150.0, 0.1)])
def test_a_disks_mass_is_the_maclaurin_integral_within_its_sampling_bound(x, y, a, sc):
    text = (f'{{"version": 1, "world": {{"width": 600, "height": 400}}, "objects": [{{"kind": "disk", "x": {x},'
            f' "y": {y}, "a": {a}, "sigma_c": {sc}, "t": 2.0, {MIX}}}]}}')
    p = planes_of(S.parse(text))
    mass = p[0].astype(np.float64).sum() - np.float32(1e-8) * np.count_nonzero(p[0] == np.float32(1e-8))
    exact = 2.0 * math.pi * sc * a * a / 3.0
    assert abs(mass - exact) / exact <= 2.0 * math.sqrt(2.0) * a ** -1.5
    assert abs(p[4:, int(y), int(x)].astype(np.float64).sum() - 1.0) < 1e-6


def test_a_preset_cloud_holds_its_mass_at_the_virial_temperature():
    sc = S.Scene.preset("sun", 256, 256)
    p, w = sc.planes()
    assert w == []
    gas = p[0] > 1e-8
    mass = p[0][gas].astype(np.float64).sum()
    assert abs(mass - S.UNIT_MASS) < 1e-4 * S.UNIT_MASS
    assert S.cloud_shape(S.UNIT_MASS) == (40.0, pytest.approx(1.0))
    assert S.thermal_over_w(S.UNIT_MASS) == 0.1 and S.thermal_over_w(10 * S.UNIT_MASS) == 0.5
    # U_th = 0.1 |W|: W of a Maclaurin disk is -(3 pi^2 / 16) ... on the grid; check U_th / |W| from the planes
    eps_th = p[3][gas].astype(np.float64) / p[0][gas].astype(np.float64)  # at rest: E = Sigma (eps_th + eps_cold)
    assert np.ptp(eps_th) > 0  # the cold energy varies with Sigma; the temperature is uniform
    assert S.Scene.preset("giant", 256, 256).warnings() and not sc.warnings()
    with pytest.raises(S.SceneError):
        S.Scene.preset("moon", 256, 256)


def test_the_config_maps_a_scene_and_refuses_what_this_build_cannot_run():
    text = ('{"version": 1, "world": {"width": 128, "height": 64, "edge": "bounce"},'
            ' "switches": {"gravity": false, "hydro": false, "heat": true, "reactions": false, "neutrinos": false,'
            ' "sinks": false},'
            ' "test": {"constant_diffusivity": 0.5, "pin_temperature": true, "flux_limiter": false},'
            ' "objects": [{"kind": "rect", "x0": 0, "y0": 0, "w": 128, "h": 64, "sigma": 1e-3, "t": 0.1,'
            ' "composition": {"He": 1}}],'
            ' "overrides": {"k1e": 0, "k2e": 0, "k1n": 0, "k2n": 0, "kappa0": 2, "cfl": 0.3}}')
    sc = S.parse(text)
    cfg = sc.config()
    assert (cfg.width, cfg.height, cfg.edge, cfg.gravity, cfg.hydro, cfg.heat) == (128, 64, "bounce", False, False, True)
    assert cfg.gamma == 2.0 and cfg.mu == pytest.approx(4.0 / 3.0) and cfg.chi == 0.5 and cfg.cfl == 0.3
    assert cfg.pin_temperature and not cfg.flux_limiter and cfg.opacity_plane and cfg.kappa0 == 2.0
    p, _ = sc.planes()
    assert np.allclose(S.Scene.opacity(p, sc.physics()), 2.0)  # kappa0 (1 + X_H), helium
    # T = mu eps_th: the planes' temperature is the one asked for
    assert np.allclose(cfg.mu * p[3] / p[0], 0.1, rtol=1e-6)
    with pytest.raises(S.SceneError, match="switches.reactions: on"):
        S.parse(text.replace('"reactions": false', '"reactions": true')).config()
    with pytest.raises(S.SceneError, match="k1e/k2e cold pressure is on"):
        S.parse(text.replace('"k1e": 0, "k2e": 0, ', "")).config()
    lax = S.parse(text.replace('"k1e": 0, "k2e": 0, ', "")).config(strict=False)
    assert lax.heat
    mixed = text.replace('"w": 128, "h": 64', '"w": 64, "h": 64').replace(
        ' "composition": {"He": 1}}]', ' "composition": {"He": 1}}, {"kind": "rect", "x0": 64, "y0": 0, "w": 64,'
        ' "h": 64, "sigma": 1e-3, "t": 0.1, "composition": {"H": 1}}]')
    with pytest.raises(S.SceneError, match="one mu per world"):
        S.parse(mixed).config()
    hydro_only = mixed.replace('"hydro": false, "heat": true', '"hydro": true, "heat": false')
    assert S.parse(hydro_only).config().hydro  # mu does not enter a step without heat


def test_numbers_print_as_the_reference_prints_them():
    assert [S._fmt(v) for v in (1.0, -1.0, 0.5, 1e-6, 2.5e20, 0.1 + 0.2, 3)] == \
        ["1", "-1", "0.5", "0.000001", "250000000000000000000", "0.30000000000000004", "3"]


@pytest.mark.skipif(not (REF_SCENES and os.path.isdir(REF_SCENES)), reason="SR_REFERENCE_DIR does not name the reference tree")
def test_every_reference_scene_file_parses_and_lays_down_without_warnings():
    runnable = []
    for name in sorted(os.listdir(REF_SCENES)):
        if not name.endswith(".json"):
            continue
        path = os.path.join(REF_SCENES, name)
        with open(path) as f:
            if isinstance(json.load(f), list):
                continue  # an edits file, not a scene
        sc = S.Scene.load(path)
        p, warnings = sc.planes()
        assert warnings == [], (name, warnings)
        assert p.shape == (14, sc.height, sc.width) and np.isfinite(p).all()
        assert np.abs(p[4:].astype(np.float64).sum(axis=0) - 1.0).max() < 1e-5, name
        try:
            sc.config(planes=p)
            runnable.append(name)
        except S.SceneError:
            pass
    # the scenes whose physics the field update runs as the reference does (cold pairs off, no reactions/sinks)
    assert {"sod.json", "ref_sod.json", "cold_disk.json", "heat_spot.json", "heat_pulse.json"} <= set(runnable)
    sun = S.Scene.load(os.path.join(REF_SCENES, "sun_disk.json"))
    assert np.array_equal(sun.planes()[0], S.Scene.preset("sun", sun.width, sun.height).planes()[0])
    fill = S.Scene.load(os.path.join(REF_SCENES, "fill_world.json"))
    for w, h in ((64, 64), (600, 400), (2048, 64), (64, 2048)):
        assert (fill.planes((w, h))[0][0] > np.float32(1e-8)).all()


def test_the_reference_mode_benchmark_world_lays_down_as_a_scene():
    # scenes.ref_disk (bench.py --case ref): 14 canonical planes, the mass fractions summing to 1 in every cell, the
    # helium core's mass mixed into the disk's solar mix (objects add their mass: He well above the disk's 0.2485),
    # reference mode with gravity, hydro and heat on
    from sandbox_reactions_b200 import scenes

    cfg, P = scenes.ref_disk(128)
    assert P.shape == (14, 128, 128) and P.dtype == np.float32 and np.isfinite(P).all()
    assert cfg.channels == 14 and cfg.heat and cfg.gravity and cfg.hydro
    assert np.abs(P[4:].sum(axis=0) - 1.0).max() < 1e-5
    assert P[5].max() > 0.5 and P[0].max() > 1.0 and P[0].min() >= 1e-3
