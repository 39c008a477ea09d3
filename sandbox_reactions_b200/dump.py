"""SRDUMP01 state dumps: read, check and write the reference's dump format, and hand a dump's state to a Step.

The format (crates/sr-engine/src/dump.rs:1-32, to_bytes at dump.rs:120-147): the 8 bytes ``SRDUMP01``, a little-endian
u32 header length, a UTF-8 JSON header, then the 14 canonical channels (state.rs:29-31: sigma, mom_x, mom_y, energy and
the ten mass fractions) as little-endian f32 planes, row-major; then, when ``resume.flux`` is true, F's two planes
(F_x, F_y); when ``resume.rate`` is true, P5's rate plane; when ``resume.held`` is true, the hold's mask (0 or 1).
The header holds exactly ``version`` (1), ``width``, ``height``, ``step``, ``sim_time``, ``channels``, ``sinks`` (at
most 16 objects of x, y, vx, vy, m) and ``resume`` (dt, dt_next, latch_since, box [8 words], box_args [6 words], flux,
and optionally rate, held, mass_carry) (parse_header, dump.rs:292-360). Every departure is refused with a message naming
it, as Dump::from_bytes refuses (dump.rs:150-215).

``load_into`` hands a dump to a Step as load_dump does (state, hold's mask, F, P5's rate, clock); ``save_from`` takes
one from a reference-mode Step as dump_state does, so a run stopped and resumed steps on as it would have.
"""
from __future__ import annotations

import json
import math
import struct
from dataclasses import dataclass, field

import numpy as np

MAGIC = b"SRDUMP01"
VERSION = 1
CHANNELS = ("sigma", "mom_x", "mom_y", "energy", "x_H", "x_He", "x_C", "x_O", "x_Ne", "x_Mg", "x_Si", "x_S", "x_Fe",
            "x_n")
MAX_SINKS = 16
WORLD_MIN, WORLD_MAX, WORLD_MULTIPLE = 64, 2048, 8  # the reference's WorldConfig (state.rs:67-84)
_HEADER_KEYS = ("version", "width", "height", "step", "sim_time", "channels", "sinks", "resume")
_RESUME_KEYS = ("dt", "dt_next", "latch_since", "box", "box_args", "flux")
_RESUME_OPTIONAL = ("rate", "held", "mass_carry")
_SINK_KEYS = ("x", "y", "vx", "vy", "m")


class DumpError(ValueError):
    """A refused dump; the message names the cause."""


@dataclass
class Dump:
    width: int
    height: int
    step: int
    sim_time: float
    planes: np.ndarray                      # (14, H, W) f32
    sinks: list = field(default_factory=list)  # dicts x, y, vx, vy, m
    dt: float = 0.0
    dt_next: float = 0.0
    latch_since: float = 0.0
    box: tuple = (0,) * 8
    box_args: tuple = (0,) * 6
    mass_carry: float = 0.0
    flux: np.ndarray | None = None          # (2, H, W) f32: F_x, F_y
    rate: np.ndarray | None = None          # (H, W) f32
    held: np.ndarray | None = None          # (H, W) u8

    def state4(self) -> np.ndarray:
        """The 4 channels this build steps: Σ, Σu, Σv, E, as (4, H, W) f32 for Step.upload."""
        return np.ascontiguousarray(self.planes[:4], np.float32)

    def to_bytes(self) -> bytes:
        resume = {"dt": _f32(self.dt), "dt_next": _f32(self.dt_next), "latch_since": _f32(self.latch_since),
                  "box": [int(v) for v in self.box], "box_args": [int(v) for v in self.box_args],
                  "flux": self.flux is not None, "rate": self.rate is not None}
        if self.held is not None:
            resume["held"] = True
        if self.mass_carry != 0.0:
            resume["mass_carry"] = _f32(self.mass_carry)
        header = {"version": VERSION, "width": self.width, "height": self.height, "step": self.step,
                  "sim_time": self.sim_time, "channels": list(CHANNELS), "sinks": list(self.sinks), "resume": resume}
        text = json.dumps(header, separators=(",", ":")).encode("utf-8")
        parts = [MAGIC, struct.pack("<I", len(text)), text, _le32(self.planes)]
        if self.flux is not None:
            parts.append(_le32(self.flux))
        if self.rate is not None:
            parts.append(_le32(self.rate))
        if self.held is not None:
            parts.append(_le32(self.held.astype(np.float32)))
        return b"".join(parts)


def _f32(v: float) -> float:
    return float(np.float32(v))


def _le32(a: np.ndarray) -> bytes:
    return np.ascontiguousarray(a, dtype="<f4").tobytes()


def _whole(m: dict, at: str, k: str) -> int:
    v = m[k]
    if isinstance(v, bool) or not isinstance(v, int) or v < 0:
        raise DumpError(f"{at}.{k}: not a whole number: {v!r}")
    return v


def _number(m: dict, at: str, k: str) -> float:
    v = m[k]
    if isinstance(v, bool) or not isinstance(v, (int, float)) or not math.isfinite(v):
        raise DumpError(f"{at}.{k}: not a finite number: {v!r}")
    return float(v)


def _words(m: dict, at: str, k: str, n: int) -> tuple:
    v = m[k]
    if (not isinstance(v, list) or len(v) != n or
            any(isinstance(w, bool) or not isinstance(w, int) or not 0 <= w < 2 ** 32 for w in v)):
        raise DumpError(f"{at}.{k}: not {n} whole numbers below 2^32: {v!r}")
    return tuple(v)


def _object(v, at: str, keys, optional=()) -> dict:
    if not isinstance(v, dict):
        raise DumpError(f"{at}: not an object")
    for k in v:
        if k not in keys and k not in optional:
            raise DumpError(f"{at}.{k}: unknown key")
    for k in keys:
        if k not in v:
            raise DumpError(f"{at}.{k}: missing")
    return v


def _flag(r: dict, k: str) -> bool:
    if k not in r:
        return False  # a header written before the key existed reads false
    if not isinstance(r[k], bool):
        raise DumpError(f"header.resume.{k}: not true or false: {r[k]!r}")
    return r[k]


def from_bytes(data: bytes) -> Dump:
    """Reads and checks a dump (the refusals of the reference's Dump::from_bytes, dump.rs:150-215)."""
    if len(data) < 8:
        raise DumpError(f"truncated: {len(data)} bytes, the magic alone is 8")
    if data[:8] != MAGIC:
        raise DumpError(f"not a state dump: magic {data[:8]!r}, expected \"SRDUMP01\"")
    if len(data) < 12:
        raise DumpError("truncated in the header length")
    (hlen,) = struct.unpack("<I", data[8:12])
    if len(data) < 12 + hlen:
        raise DumpError(f"truncated in the header: {hlen} bytes announced, {len(data) - 12} present")
    try:
        text = data[12:12 + hlen].decode("utf-8")
    except UnicodeDecodeError as e:
        raise DumpError(f"header: not UTF-8: {e}") from None
    try:
        header = json.loads(text)
    except json.JSONDecodeError as e:
        raise DumpError(f"header: not JSON: {e}") from None
    m = _object(header, "header", _HEADER_KEYS)
    version = _whole(m, "header", "version")
    if version != VERSION:
        raise DumpError(f"header.version: {version}, this build reads {VERSION}")
    w, h = _whole(m, "header", "width"), _whole(m, "header", "height")
    for n in (w, h):
        if not (WORLD_MIN <= n <= WORLD_MAX and n % WORLD_MULTIPLE == 0):
            raise DumpError(f"header: world {w} x {h}: each side a multiple of {WORLD_MULTIPLE} in "
                            f"[{WORLD_MIN}, {WORLD_MAX}]")
    if m["channels"] != list(CHANNELS):
        raise DumpError(f"header.channels: {m['channels']!r}, expected {list(CHANNELS)!r} in that order")
    if not isinstance(m["sinks"], list):
        raise DumpError("header.sinks: not a list")
    if len(m["sinks"]) > MAX_SINKS:
        raise DumpError(f"header.sinks: {len(m['sinks'])} sinks, at most {MAX_SINKS}")
    sinks = []
    for i, sk in enumerate(m["sinks"]):
        at = f"header.sinks[{i}]"
        sk = _object(sk, at, _SINK_KEYS)
        sinks.append({k: _number(sk, at, k) for k in _SINK_KEYS})
    r = _object(m["resume"], "header.resume", _RESUME_KEYS, _RESUME_OPTIONAL)
    if not isinstance(r["flux"], bool):
        raise DumpError(f"header.resume.flux: not true or false: {r['flux']!r}")
    flux, rate, held = r["flux"], _flag(r, "rate"), _flag(r, "held")
    if rate and not flux:
        raise DumpError("header.resume.rate: true without F (flux false): the rate is P5's")
    at_r = "header.resume"
    dump = Dump(width=w, height=h, step=_whole(m, "header", "step"), sim_time=_number(m, "header", "sim_time"),
                planes=np.zeros((0,), np.float32), sinks=sinks, dt=_f32(_number(r, at_r, "dt")),
                dt_next=_f32(_number(r, at_r, "dt_next")), latch_since=_f32(_number(r, at_r, "latch_since")),
                box=_words(r, at_r, "box", 8), box_args=_words(r, at_r, "box_args", 6),
                mass_carry=_f32(_number(r, at_r, "mass_carry")) if "mass_carry" in r else 0.0)

    body = data[12 + hlen:]
    plane = w * h * 4
    channels = len(CHANNELS) * plane
    with_flux = channels + (2 * plane if flux else 0)
    with_rate = with_flux + (plane if rate else 0)
    want = with_rate + (plane if held else 0)
    n = len(body)
    # a body that another flag would fit is that flag's refusal (dump.rs:171-192)
    if flux and n == want - 2 * plane:
        raise DumpError("header.resume.flux: true, but no F planes follow the 14 channels")
    if not flux and n == want + 2 * plane:
        raise DumpError("header.resume.flux: false, but F's 2 planes follow the 14 channels")
    if held and n == want - plane:
        raise DumpError("header.resume.held: true, but no mask plane follows the last")
    if rate and n == want - plane:
        raise DumpError("header.resume.rate: true, but no rate plane follows F's 2")
    if flux and not rate and n == want + plane:
        raise DumpError("header.resume.rate: false, but a plane follows F's 2")
    if not held and n == want + plane:
        raise DumpError("header.resume.held: not true, but a plane follows the last")
    if n < want:
        raise DumpError(f"truncated in the planes: {n} of {want} bytes")
    if n > want:
        raise DumpError(f"{n - want} bytes past the last plane")
    values = np.frombuffer(body, dtype="<f4")
    dump.planes = values[:channels // 4].astype(np.float32).reshape(len(CHANNELS), h, w)
    if flux:
        dump.flux = values[channels // 4:with_flux // 4].astype(np.float32).reshape(2, h, w)
    if rate:
        dump.rate = values[with_flux // 4:with_rate // 4].astype(np.float32).reshape(h, w)
    if held:
        mask = values[with_rate // 4:].astype(np.float32)
        bad = np.nonzero((mask != 0.0) & (mask != 1.0))[0]
        if bad.size:
            raise DumpError(f"header.resume.held: the mask's cell {int(bad[0])} is {mask[bad[0]]}, not 0 or 1")
        dump.held = (mask == 1.0).astype(np.uint8).reshape(h, w)
    return dump


def read(path) -> Dump:
    with open(path, "rb") as f:
        return from_bytes(f.read())


def write(dump: Dump, path) -> None:
    with open(path, "wb") as f:
        f.write(dump.to_bytes())


def load_into(step, dump: Dump) -> None:
    """load_dump (crates/sr-engine/src/dump.rs:368-410) into `step` (a sandbox_reactions_b200.engine.Step of the same
    world): the state (State::upload), then in reference mode (14 channels) the hold's mask (the dump's, or none held)
    and F into the side flux the next P4 pushes with, then P5's rate (the dump's, or zeros) when the step runs P5, then
    the clock (Step::restore: the next step's index, the sim time, Δt_n and Δt_n+1) — a dump at step 0 keeps the
    upload's own initial reduction, as the reference's restore does. A 4-channel step takes Σ, Σu, Σv, E, the rate and
    the clock; F has no reader there (its P4 takes no radiation force).

    Refused as load_dump refuses: another world than the step's; a step index past the GPU's u32 count; sinks (this
    build runs no P3 to keep them); in reference mode F without P5 to read it, and P5 without F (its first step would
    push with F = 0)."""
    c, h, w = step.shape
    if (h, w) != (dump.height, dump.width):
        raise DumpError(f"dump world {dump.width} x {dump.height}, the step's {w} x {h}")
    if dump.step > 0xFFFFFFFF:
        raise DumpError(f"dump step {dump.step}: past the GPU's u32 step count")
    if dump.sinks:
        raise DumpError(f"dump holds {len(dump.sinks)} sink(s), and this step runs no P3 to keep them")
    heat = bool(step.config.heat)
    ref = c == len(CHANNELS)
    if ref and dump.flux is not None and not heat:
        raise DumpError("dump holds F, and this step runs no P5 to keep it (heat off)")
    if ref and dump.flux is None and heat:
        raise DumpError("dump holds no F, and this step runs P5: its first step would push with F = 0")
    if ref:
        step.upload(np.ascontiguousarray(dump.planes, np.float32))
        held = dump.held if dump.held is not None else np.zeros((h, w), np.uint32)
        step.upload_held(held)
        if dump.flux is not None:
            step.set_side_flux(dump.flux[0], dump.flux[1])
    else:
        step.upload(dump.state4())
    if heat:
        step.set_heat_rate(dump.rate)
    if dump.step > 0:
        step.set_clock(dump.step, dump.sim_time, dump.dt, dump.dt_next)


def save_from(step) -> Dump:
    """dump_state (crates/sr-engine/src/dump.rs:355-366) of a reference-mode step (14 channels): the state, the step
    index and sim time, Δt_n and Δt_n+1, and with P5 the side flux F and P5's rate; the hold's mask when any cell is
    held. A 4-channel step is refused: a dump holds the 14 canonical channels, and that step has no species."""
    c, h, w = step.shape
    if c != len(CHANNELS):
        raise DumpError(f"a dump holds the {len(CHANNELS)} canonical channels; this step carries {c} (no species)")
    planes = step.readback()
    clock = step.read_dt()
    held = step.read_held()
    flux = rate = None
    if step.config.heat:
        flux = np.stack(step.read_side_flux())
        rate = step.read_heat_rate()
    return Dump(width=w, height=h, step=int(clock.steps), sim_time=float(clock.sim_time), planes=planes,
                dt=float(clock.dt), dt_next=float(clock.dt_next), flux=flux, rate=rate,
                held=held.astype(np.uint8) if held.any() else None)
