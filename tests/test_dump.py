"""SRDUMP01 state dumps (crates/sr-engine/src/dump.rs): round trips, every refusal of Dump::from_bytes, the reference's
own dump fixtures (read as bytes from the reference tree when it is present), and a dump's state stepped on the GPU."""
import json
import os
import struct

import numpy as np
import pytest

from sandbox_reactions_b200 import dump as D

# the reference project's scenes/ folder, when SR_REFERENCE_DIR names a checkout of it (else these tests skip)
REF_SCENES = os.path.join(os.environ.get("SR_REFERENCE_DIR", ""), "scenes") if os.environ.get("SR_REFERENCE_DIR") else ""


def sample(w=64, h=64, flux=True, rate=True, held=True, sinks=1, seed=0):
    rng = np.random.default_rng(seed)
    planes = rng.random((14, h, w)).astype(np.float32)
    return D.Dump(width=w, height=h, step=123, sim_time=0.1 + 1.0 / 3.0, planes=planes,
                  sinks=[{"x": 1.5, "y": 2.25, "vx": -0.5, "vy": 0.125, "m": 1.0 / 7.0}] * sinks,
                  dt=1e-3, dt_next=1.1e-3, latch_since=0.25, box=tuple(range(8)), box_args=tuple(range(6)),
                  mass_carry=2.5e-7,
                  flux=rng.random((2, h, w)).astype(np.float32) if flux else None,
                  rate=rng.random((h, w)).astype(np.float32) if rate else None,
                  held=(rng.random((h, w)) < 0.1).astype(np.uint8) if held else None)


def same(a: D.Dump, b: D.Dump):
    assert (a.width, a.height, a.step, a.sim_time) == (b.width, b.height, b.step, b.sim_time)
    assert a.sinks == b.sinks and a.box == b.box and a.box_args == b.box_args
    assert (a.dt, a.dt_next, a.latch_since, a.mass_carry) == (np.float32(b.dt), np.float32(b.dt_next),
                                                              np.float32(b.latch_since), np.float32(b.mass_carry))
    assert np.array_equal(a.planes, b.planes)
    for x, y in ((a.flux, b.flux), (a.rate, b.rate), (a.held, b.held)):
        assert (x is None) == (y is None) and (x is None or np.array_equal(x, y))


@pytest.mark.parametrize("flux,rate,held", [(False, False, False), (True, False, False), (True, True, False),
                                            (True, True, True), (False, False, True)])
def test_a_dump_survives_its_bytes(flux, rate, held):
    d = sample(flux=flux, rate=rate, held=held)
    same(D.from_bytes(d.to_bytes()), d)


def header_of(d: D.Dump):
    b = d.to_bytes()
    (n,) = struct.unpack("<I", b[8:12])
    return json.loads(b[12:12 + n]), b[12 + n:]


def rebuild(header, body):
    text = json.dumps(header).encode()
    return D.MAGIC + struct.pack("<I", len(text)) + text + body


def refused(data, words):
    with pytest.raises(D.DumpError) as e:
        D.from_bytes(data)
    assert words in str(e.value), str(e.value)


def test_every_departure_is_refused_by_name():
    d = sample(flux=True, rate=True, held=True)
    good = d.to_bytes()
    h, body = header_of(d)
    plane = d.width * d.height * 4
    refused(b"SRDUMP0", "truncated")
    refused(b"NOTADUMP" + good[8:], "not a state dump")
    refused(good[:10], "header length")
    refused(good[:20], "truncated in the header")
    refused(D.MAGIC + struct.pack("<I", 2) + b"\xff\xfe", "not UTF-8")
    refused(D.MAGIC + struct.pack("<I", 3) + b"{x}", "not JSON")
    refused(rebuild({**h, "extra": 1}, body), "header.extra: unknown key")
    refused(rebuild({k: v for k, v in h.items() if k != "step"}, body), "header.step: missing")
    refused(rebuild({**h, "version": 2}, body), "header.version: 2")
    refused(rebuild({**h, "width": 60}, body), "header: world 60 x 64")
    refused(rebuild({**h, "channels": list(reversed(D.CHANNELS))}, body), "header.channels")
    refused(rebuild({**h, "sinks": [h["sinks"][0]] * 17}, body), "17 sinks")
    refused(rebuild({**h, "sinks": [{"x": 1}]}, body), "header.sinks[0].y: missing")
    refused(rebuild({**h, "resume": {**h["resume"], "box": [1, 2]}}, body), "header.resume.box")
    refused(rebuild({**h, "resume": {**h["resume"], "dt": "fast"}}, body), "header.resume.dt: not a finite number")
    refused(rebuild({**h, "resume": {**h["resume"], "flux": False}}, body), "header.resume.rate: true without F")
    refused(rebuild({**h, "resume": {**h["resume"], "held": False}}, body), "held: not true, but a plane follows")
    refused(rebuild(h, body[:-plane]), "held: true, but no mask plane")
    refused(good + b"\0\0\0\0", "4 bytes past the last plane")
    refused(good[:-4], "truncated in the planes")
    mask_at = len(good) - plane
    refused(good[:mask_at] + struct.pack("<f", 0.5) + good[mask_at + 4:], "the mask's cell 0 is 0.5")
    nf = sample(flux=False, rate=False, held=False)
    h2, body2 = header_of(nf)
    refused(rebuild(h2, body2 + b"\0" * (2 * plane)), "flux: false, but F's 2 planes follow")
    f2 = sample(flux=True, rate=False, held=False)
    h3, body3 = header_of(f2)
    refused(rebuild(h3, body3[:-2 * plane]), "flux: true, but no F planes follow")


def test_the_mass_carry_and_optional_flags_default_when_absent():
    d = sample(flux=False, rate=False, held=False)
    h, body = header_of(d)
    r = {k: v for k, v in h["resume"].items() if k not in ("rate", "held", "mass_carry")}
    got = D.from_bytes(rebuild({**h, "resume": r}, body))
    assert got.mass_carry == 0.0 and got.rate is None and got.held is None


@pytest.mark.skipif(not (REF_SCENES and os.path.isdir(REF_SCENES)), reason="SR_REFERENCE_DIR does not name the reference tree")
def test_the_reference_fixtures_read_and_round_trip():
    names = sorted(f for f in os.listdir(REF_SCENES) if f.endswith(".bin"))
    assert names
    for name in names:
        d = D.read(os.path.join(REF_SCENES, name))
        assert d.planes.shape == (14, d.height, d.width)
        assert np.isfinite(d.planes).all() and (d.planes[0] >= 0).all()
        frac = d.planes[4:].sum(axis=0)  # the mass fractions sum to 1 where there is gas
        gas = d.planes[0] > 0
        assert np.abs(frac[gas] - 1.0).max() < 1e-3, name
        assert d.state4().shape == (4, d.height, d.width)
        same(D.from_bytes(d.to_bytes()), d)


class StubStep:
    """The calls load_into and save_from make, recorded (no GPU): a Step of `channels` planes with or without P5."""

    def __init__(self, w=64, h=64, channels=14, heat=True):
        from sandbox_reactions_b200.abi import Config

        self.shape = (channels, h, w)
        self.config = Config(width=w, height=h, channels=channels, heat=heat)
        self.calls = []

    def __getattr__(self, name):
        if name.startswith(("upload", "set_")):
            return lambda *a: self.calls.append((name, a))
        raise AttributeError(name)


def test_load_into_writes_in_load_dumps_order():
    # dump.rs:397-409: the state, the hold's mask, F, the rate, then the clock
    d = sample(sinks=0)
    st = StubStep()
    D.load_into(st, d)
    assert [c[0] for c in st.calls] == ["upload", "upload_held", "set_side_flux", "set_heat_rate", "set_clock"]
    assert np.array_equal(st.calls[0][1][0], d.planes) and np.array_equal(st.calls[1][1][0], d.held)
    assert np.array_equal(st.calls[2][1][0], d.flux[0]) and np.array_equal(st.calls[2][1][1], d.flux[1])
    assert np.array_equal(st.calls[3][1][0], d.rate)
    assert st.calls[4][1] == (d.step, d.sim_time, d.dt, d.dt_next)
    # none held: a mask of zeros; no rate: zeros (None); step 0: the upload's own reduction, no clock
    d2 = sample(sinks=0, rate=False, held=False)
    d2.step = 0
    st2 = StubStep()
    D.load_into(st2, d2)
    assert [c[0] for c in st2.calls] == ["upload", "upload_held", "set_side_flux", "set_heat_rate"]
    assert not st2.calls[1][1][0].any() and st2.calls[3][1] == (None,)
    # a 4-channel step: Σ, Σu, Σv, E, the rate, the clock; no mask, no F
    st4 = StubStep(channels=4)
    D.load_into(st4, sample(sinks=0))
    assert [c[0] for c in st4.calls] == ["upload", "set_heat_rate", "set_clock"]
    assert st4.calls[0][1][0].shape == (4, 64, 64)


@pytest.mark.parametrize("case,message", [
    ("world", "dump world 64 x 64, the step's 72 x 64"),
    ("step", "past the GPU's u32 step count"),
    ("sinks", "runs no P3"),
    ("flux_no_heat", "dump holds F, and this step runs no P5"),
    ("heat_no_flux", "its first step would push with F = 0"),
])
def test_load_into_refuses_what_load_dump_refuses(case, message):
    d = sample(sinks=1 if case == "sinks" else 0, flux=case != "heat_no_flux")
    st = StubStep(w=72 if case == "world" else 64, heat=case != "flux_no_heat")
    if case == "step":
        d.step = 2 ** 32
    with pytest.raises(D.DumpError, match=message):
        D.load_into(st, d)
    assert st.calls == []  # refused before anything was written


def test_save_from_refuses_a_step_without_species():
    with pytest.raises(D.DumpError, match="no species"):
        D.save_from(StubStep(channels=4))


@pytest.mark.gpu
def test_a_dumped_state_steps_as_the_state_itself():
    from sandbox_reactions_b200 import scenes
    from sandbox_reactions_b200.engine import Step

    cfg, P = scenes.disk(64)
    planes = np.zeros((14, 64, 64), np.float32)
    planes[:4] = P
    planes[4] = 1.0
    d = D.from_bytes(D.Dump(width=64, height=64, step=0, sim_time=0.0, planes=planes).to_bytes())
    with Step(cfg) as a, Step(cfg) as b:
        a.upload(P)
        D.load_into(b, d)
        a.run(3)
        b.run(3)
        assert np.array_equal(a.readback(), b.readback())
