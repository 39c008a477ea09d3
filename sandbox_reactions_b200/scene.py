"""Scene files: the reference's ``scenes/*.json`` read, checked and laid down as a world's planes, and handed to a Step.

Follows crates/sr-engine/src/scene.rs. ``parse`` refuses every departure scene.rs refuses, each message naming its
path (``switches.hydor: unknown key``; scene.rs:140-402): unknown keys at every level, ``t`` with ``pressure``, a
composition that does not sum to 1, a world outside 64-2048 in multiples of 8 (state.rs:67-111), overrides that are not
physics.json keys or break physics.json's bounds (registry.rs:234-444). ``Scene.planes`` lays the objects down as
scene.rs:427-509 does: a ``rect`` covers [x0, x0 + w) x [y0, y0 + h) clipped to the world, a ``disk`` samples
Sigma_c sqrt(1 - r^2/a^2) at cell centres, a ``preset`` is the Sun-like cloud of the nominal unit mass at the temperature
that makes U_th = thermal_over_w(M) |W| with W from one gravity solve over its cells (scene.rs:518-628); objects add
mass, momentum, energy and species mass where they overlap; cells no object covers hold the floor state (Sigma_floor of
hydrogen at T_floor, at rest). The energy is E = Sigma (eps_th + eps_cold) + 1/2 Sigma |v|^2 with eps_th = T / mu, or
(Pi - Pi_e - Pi_n) / Sigma from a pressure (the reference's EOS, eos.rs:1-263: gamma = 2, the cold pressure of the two
K pairs tabulated as u(x) on 512 log-spaced nodes).

This build steps the 4-channel field update with the gamma = 2 ideal gas (no cold pressure) and one mu per world:
``Scene.config`` maps a scene onto a ``Config`` and refuses, by name, what that field update cannot run as the
reference would -- a K pair that is on, reactions / neutrinos / sinks switched on, and with heat on, gas cells of more
than one composition. The opacity the reference's FLD uses, kappa0 (1 + X_H) (reference/heat.rs:210-219, dust off),
comes as a per-cell plane (``Scene.opacity``); ``load_into`` uploads the state and that plane.
"""
from __future__ import annotations

import functools
import json
import math
from dataclasses import dataclass, field
from decimal import Decimal

import numpy as np

from .abi import Config

# elements.json's species in id order: key, mass number A, charge Z (registry.rs:45-153)
SPECIES = (("H", 1, 1), ("He", 4, 2), ("C", 12, 6), ("O", 16, 8), ("Ne", 20, 10), ("Mg", 24, 12), ("Si", 28, 14),
           ("S", 32, 16), ("Fe", 56, 26), ("n", 1, 0))
N_SPECIES = len(SPECIES)
N_CHANNELS = 4 + N_SPECIES
ID_H, ID_HE, ID_N = 0, 1, 9
WORLD_MIN, WORLD_MAX, WORLD_MULTIPLE = 64, 2048, 8

PRESETS = ("sun", "massive", "giant")
SUN_MIX = (0.7346, 0.2485, 0.0092, 0.0077, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0)
SUN_SIGMA_C, SUN_RADIUS, MAX_RADIUS = 1.0, 40.0, 150.0
UNIT_MASS = 2.0 * math.pi * SUN_SIGMA_C * SUN_RADIUS * SUN_RADIUS / 3.0
THERMAL_OVER_W, THERMAL_OVER_W_MAX = 0.1, 0.5
COMPOSITION_TOLERANCE = 1e-6
SELF_CELL = 3.525494348078172  # 4 ln(1 + sqrt 2): the potential at a unit square's centre from its own unit mass

# physics.json as shipped, and each key's class (registry.rs:234-293): P > 0, N >= 0, W whole >= 1, U (nu) >= 4
_SHIPPED = (
    ("t_h", 56.0, "P"), ("t_he", 100.0, "P"), ("t_c", 109.8, "P"), ("t_ne", 118.0, "P"), ("t_o", 122.0, "P"),
    ("t_si", 135.0, "P"), ("q_h", 8700.0, "P"), ("a_h_burn", 5e-4, "P"), ("a_he_burn", 1e-3, "P"),
    ("a_c_alpha", 1e-3, "P"), ("a_c_burn", 1e-3, "P"), ("a_ne_burn", 1e-3, "P"), ("a_o_burn", 1e-3, "P"),
    ("a_mg_burn", 1e-3, "P"), ("a_si_burn", 1e-3, "P"), ("a_s_burn", 1e-3, "P"), ("a_n_fe", 100.0, "P"),
    ("nu_c_burn", 30.0, "U"), ("nu_ne_burn", 30.0, "U"), ("nu_o_burn", 30.0, "U"), ("nu_mg_burn", 30.0, "U"),
    ("nu_si_burn", 30.0, "U"), ("nu_s_burn", 30.0, "U"), ("sigma_n", 160.0, "P"), ("burn_dx", 0.1, "P"),
    ("burn_dt", 0.05, "P"), ("burn_k", 15.0, "N"), ("sigma_floor", 1e-8, "P"), ("sigma_vac", 1e-6, "P"),
    ("t_floor", 0.05, "P"), ("sigma_obj", 1e-3, "P"), ("paint_sigma", 0.02, "P"), ("paint_t", 2.0, "P"),
    ("heat_factor", 1.05, "P"), ("cool_factor", 0.95, "P"), ("k1e", 21.3, "N"), ("k2e", 134.0, "N"),
    ("k1n", 2.67, "N"), ("k2n", 58.2, "N"), ("a_r", 6.25e-7, "P"), ("c_sb", 12800.0, "P"), ("kappa0", 1.0, "N"),
    ("k_cond", 0.0, "N"), ("a_nu", 1e-3, "N"), ("t_nu", 93.0, "P"), ("m_nu", 8.0, "P"), ("f_dep", 0.05, "N"),
    ("sigma_bh", 6000.0, "P"), ("cfl", 0.4, "P"), ("eta_g", 0.3, "P"), ("kappa_dust", 0.0, "N"),
    ("t_dust", 0.0, "N"), ("block", 4.0, "W"), ("sigma_hold", 10.0, "P"), ("eta_hold", 0.1, "P"),
    ("r_hold", 24.0, "P"),
)
_CLASS = {k: c for k, _, c in _SHIPPED}
_NU_KEYS = ("nu_c_burn", "nu_ne_burn", "nu_o_burn", "nu_mg_burn", "nu_si_burn", "nu_s_burn")


class SceneError(ValueError):
    """A refused scene; the message names the path of the cause."""


def _fmt(x) -> str:
    """A number as the reference prints it: shortest round-trip digits, no exponent, no trailing '.0'."""
    if isinstance(x, int):
        return str(x)
    if not math.isfinite(x):
        return {math.inf: "inf", -math.inf: "-inf"}.get(x, "NaN")
    s = format(Decimal(repr(float(x))), "f")
    if "." in s:
        s = s.rstrip("0").rstrip(".")
    return s


def _debug_str(s: str) -> str:
    return json.dumps(s, ensure_ascii=False)


# ---- physics.json

class Physics:
    """physics.json's constants with a scene's overrides, validated as a whole (registry.rs:358-444)."""

    def __init__(self, values: dict):
        self.values = dict(values)

    @staticmethod
    def shipped() -> "Physics":
        return Physics({k: v for k, v, _ in _SHIPPED})

    @staticmethod
    def keys():
        return [k for k, _, _ in _SHIPPED]

    def get(self, key: str):
        return self.values.get(key)

    def with_(self, overrides) -> "Physics":
        nxt = Physics(self.values)
        for key, x in overrides:
            if key not in nxt.values:
                raise SceneError(f"physics.json: {key}: unknown key")
            nxt.values[key] = float(x)
        nxt.validate()
        return nxt

    def validate(self) -> None:
        def bad(key, why):
            raise SceneError(f"physics.json: {key}: {why}")

        for key, _, cls in _SHIPPED:
            x = self.values[key]
            if not math.isfinite(x):
                bad(key, f"must be a finite number, got {_fmt(x)}")
            if cls == "P" and x <= 0.0:
                bad(key, f"must be > 0, got {_fmt(x)}")
            if cls == "N" and x < 0.0:
                bad(key, f"must be ≥ 0, got {_fmt(x)}")
            if cls == "W" and (x < 1.0 or x != math.floor(x)):
                bad(key, f"must be a whole number ≥ 1, got {_fmt(x)}")
            if cls == "U" and x < 4.0:
                bad(key, f"must be ≥ 4 (K7: steep burning), got {_fmt(x)}")
        v = self.values
        ladder = (("t_he", "t_h", "must be > t_h = {} (K6), got {}", lambda a, b: a <= b),
                  ("t_c", "t_he", "must be > t_he = {} (K6), got {}", lambda a, b: a <= b),
                  ("t_ne", "t_c", "must be > t_c = {} (K6), got {}", lambda a, b: a <= b),
                  ("t_o", "t_ne", "must be ≥ t_ne = {} (K6; Ne and O may tie), got {}", lambda a, b: a < b),
                  ("t_si", "t_o", "must be > t_o = {} (K6), got {}", lambda a, b: a <= b))
        for key, below, text, fails in ladder:
            if fails(v[key], v[below]):
                bad(key, text.format(_fmt(v[below]), _fmt(v[key])))
        if v["t_si"] / v["t_h"] > 10.0:
            bad("t_si", f"t_si / t_h must be ≤ 10 (§1.6.3), got {_fmt(v['t_si'] / v['t_h'])}")
        for nu in _NU_KEYS:
            if v["m_nu"] >= v[nu]:
                bad("m_nu", f"must be < {nu} = {_fmt(v[nu])} (§2.5.3), got {_fmt(v['m_nu'])}")

        def pair(k1, k2):
            a, b = v[k1] > 0.0, v[k2] > 0.0
            if a and not b:
                bad(k2, f"must be > 0 while {k1} is (a pair is on or off)")
            if b and not a:
                bad(k1, f"must be > 0 while {k2} is (a pair is on or off)")
            return a and b

        electrons, neutrons = pair("k1e", "k2e"), pair("k1n", "k2n")
        if electrons:
            floor = 2.0 * (v["k2e"] / v["k1e"]) ** 2
            if v["sigma_n"] < floor:
                bad("sigma_n", f"must be ≥ 2 (k2e/k1e)² = {_fmt(floor)} (§2.5.1), got {_fmt(v['sigma_n'])}")
        if electrons and neutrons:
            ratio = 8.0 * (v["k2n"] / v["k2e"]) ** 2
            if not 1.4 <= ratio <= 2.0:
                bad("k2n", f"m_tov / m_ch must be in [1.4, 2.0] (§2.7, K9), got {_fmt(ratio)}")
        if v["f_dep"] > 0.1:  # the stand-ins ship off: f_dep's cap is 0.1, kappa_dust stays 0
            bad("f_dep", f"must be ≤ 0.1 while S2 is off (§2.5.4, §1.6.4), got {_fmt(v['f_dep'])}")
        if v["kappa_dust"] != 0.0:
            bad("kappa_dust", f"must be 0 while S1 is off (§1.6.4), got {_fmt(v['kappa_dust'])}")

    def __eq__(self, other):
        return isinstance(other, Physics) and self.values == other.values


# ---- the reference's EOS (eos.rs): gamma = 2, T = mu eps_th, the cold pressure of two K pairs

TABLE_POINTS, X_MIN, X_MAX, QUAD_STEPS = 512, 1e-8, 1e8, 64


def cold_pressure(x, k1: float, k2: float):
    """P(x; K1, K2) = 1 / (1 / (K1 x^2) + 1 / (K2 x^{3/2})), 0 for x <= 0 or a pair that is off (eos.rs:22-29)."""
    x = np.asarray(x, dtype=np.float64)
    if k1 <= 0.0 or k2 <= 0.0:
        return np.zeros_like(x)
    with np.errstate(divide="ignore", invalid="ignore"):
        p = 1.0 / (1.0 / (k1 * x * x) + 1.0 / (k2 * x ** 1.5))
    return np.where(x > 0.0, p, 0.0)


class ColdTable:
    """u(x) = x * integral_0^x P(s) / s^2 ds on 512 nodes log-spaced over [1e-8, 1e8], each segment integrated by
    Simpson's rule in t = sqrt(s), and read by linear interpolation in (ln x, ln u); below the first node u follows
    K1 x^2 (eos.rs:31-131)."""

    def __init__(self, k1: float, k2: float):
        assert k1 > 0.0 and k2 > 0.0
        self.k1, self.k2 = k1, k2

        def f(t):
            if t <= 0.0:
                return 0.0
            s = t * t
            return 1.0 / (1.0 / (k1 * s * s) + 1.0 / (k2 * s ** 1.5)) / (s * s) * 2.0 * t

        ln_u = []
        t_prev, j = 0.0, 0.0
        for i in range(TABLE_POINTS):
            t = math.sqrt(self.node_x(i))
            n = QUAD_STEPS * 8 if i == 0 else QUAD_STEPS
            h = (t - t_prev) / n
            acc = f(t_prev) + f(t)
            for q in range(1, n):
                acc += f(t_prev + h * q) * (4.0 if q % 2 == 1 else 2.0)
            j += acc * h / 3.0
            ln_u.append(math.log(self.node_x(i) * j))
            t_prev = t
        self.ln_u = np.array(ln_u)

    @staticmethod
    def node_x(i: int) -> float:
        frac = i / (TABLE_POINTS - 1)
        return math.exp(math.log(X_MIN) + frac * (math.log(X_MAX) - math.log(X_MIN)))

    @staticmethod
    def step() -> float:
        return (math.log(X_MAX) - math.log(X_MIN)) / (TABLE_POINTS - 1)

    def u(self, x):
        x = np.asarray(x, dtype=np.float64)
        out = np.zeros_like(x)
        pos_x = x > 0.0
        with np.errstate(divide="ignore", invalid="ignore"):
            pos = (np.log(np.where(pos_x, x, 1.0)) - math.log(X_MIN)) / self.step()
        below = pos_x & (pos < 0.0)
        out = np.where(below, math.exp(self.ln_u[0]) * (x / X_MIN) ** 2, out)
        i = np.clip(np.floor(np.maximum(pos, 0.0)).astype(np.int64), 0, TABLE_POINTS - 2)
        frac = pos - i
        interp = np.exp(self.ln_u[i] + frac * (self.ln_u[i + 1] - self.ln_u[i]))
        return np.where(pos_x & ~below, interp, out)


@functools.lru_cache(maxsize=8)
def _cold_table(k1: float, k2: float) -> ColdTable:
    return ColdTable(k1, k2)


class Eos:
    """The reference's EOS from physics.json's K pairs and T_floor (eos.rs:150-263)."""

    def __init__(self, physics: Physics):
        g = physics.get
        self.t_floor = g("t_floor")
        self.k1e, self.k2e, self.k1n, self.k2n = g("k1e"), g("k2e"), g("k1n"), g("k2n")
        self.electrons = _cold_table(self.k1e, self.k2e) if self.k1e > 0.0 and self.k2e > 0.0 else None
        self.neutrons = _cold_table(self.k1n, self.k2n) if self.k1n > 0.0 and self.k2n > 0.0 else None

    @staticmethod
    def eps_th_of_t(t, mu):
        return t / mu

    def pi_e(self, sigma, y_e):
        return cold_pressure(y_e * np.asarray(sigma, np.float64), self.k1e, self.k2e) if self.electrons else \
            np.zeros_like(np.asarray(sigma, np.float64))

    def pi_n(self, sigma, x_n):
        return cold_pressure(x_n * np.asarray(sigma, np.float64), self.k1n, self.k2n) if self.neutrons else \
            np.zeros_like(np.asarray(sigma, np.float64))

    def eps_cold(self, sigma, y_e, x_n):
        sigma = np.asarray(sigma, np.float64)
        u_e = self.electrons.u(y_e * sigma) if self.electrons else 0.0
        u_n = self.neutrons.u(x_n * sigma) if self.neutrons else 0.0
        return (u_e + u_n) / sigma

    @property
    def cold(self) -> bool:
        return self.electrons is not None or self.neutrons is not None


def composition(x) -> tuple[float, float, float]:
    """1/mu, Y_e and Z_met of mass fractions in species order, fully ionised (registry.rs:145-154)."""
    inv_mu, y_e = 0.0, 0.0
    for (_, a, z), xi in zip(SPECIES, x):
        inv_mu += xi * (z + 1.0) / a
        y_e += xi * z / a
    return inv_mu, y_e, 1.0 - x[ID_H] - x[ID_HE] - x[ID_N]


# ---- the scene

@dataclass(frozen=True)
class Gas:
    heat: tuple  # ("t", T) or ("pressure", Pi)
    composition: tuple
    v: tuple = (0.0, 0.0)


@dataclass(frozen=True)
class Obj:
    kind: str                 # "preset", "disk" or "rect"
    x: float = 0.0            # preset / disk centre (points in cell units)
    y: float = 0.0
    a: float = 0.0            # disk radius
    sigma_c: float = 0.0      # disk central Sigma
    x0: int = 0               # rect
    y0: int = 0
    w: int = 0
    h: int = 0
    sigma: float = 0.0
    gas: Gas | None = None    # disk / rect
    preset: str = ""
    mass: float = 0.0         # preset


@dataclass
class Switches:
    gravity: bool = True
    hydro: bool = True
    heat: bool = True
    reactions: bool = True
    neutrinos: bool = True
    sinks: bool = True


@dataclass
class TestSettings:
    pin_temperature: bool = False
    constant_diffusivity: float | None = None
    flux_limiter: bool = True


class _Fields:
    """One JSON object being read: its path for messages, its keys checked against the ones it may hold."""

    def __init__(self, value, at: str, known):
        name = at if at else "the scene"
        if not isinstance(value, dict):
            raise SceneError(f"{name}: must be an object")
        for k in sorted(value):  # the reference's JSON maps iterate in key order
            if k not in known:
                raise SceneError(f"{_join(at, k)}: unknown key")
        self.map, self.at = value, at

    def path(self, key):
        return _join(self.at, key)

    def get(self, key):
        return self.map.get(key)

    def number(self, key):
        if key not in self.map:
            return None
        v = self.map[key]
        if _is_number(v) and math.isfinite(v):
            return float(v)
        raise SceneError(f"{self.path(key)}: must be a finite number")

    def required(self, key):
        x = self.number(key)
        if x is None:
            raise SceneError(f"{self.path(key)}: missing")
        return x

    def positive(self, key):
        x = self.required(key)
        if x > 0.0:
            return x
        raise SceneError(f"{self.path(key)}: must be > 0, got {_fmt(x)}")

    def whole(self, key):
        v = self.map.get(key)
        if isinstance(v, int) and not isinstance(v, bool) and -2 ** 63 <= v < 2 ** 63:
            return v
        raise SceneError(f"{self.path(key)}: must be a whole number")

    def flag(self, key, default):
        if key not in self.map:
            return default
        v = self.map[key]
        if isinstance(v, bool):
            return v
        raise SceneError(f"{self.path(key)}: must be true or false")


def _join(at, key):
    return key if not at else f"{at}.{key}"


def _is_number(v):
    return isinstance(v, (int, float)) and not isinstance(v, bool)


def _parse_gas(f: _Fields) -> Gas:
    has_t, has_p = "t" in f.map, "pressure" in f.map
    if has_t and has_p:
        raise SceneError(f"{f.at}: takes t or pressure, not both")
    if not has_t and not has_p:
        raise SceneError(f"{f.at}: needs t or pressure")
    heat = ("t", f.positive("t")) if has_t else ("pressure", f.positive("pressure"))
    at = f.path("composition")
    if "composition" not in f.map:
        raise SceneError(f"{at}: missing")
    m = f.map["composition"]
    if not isinstance(m, dict):
        raise SceneError(f"{at}: must be an object of mass fractions")
    keys = [s[0] for s in SPECIES]
    comp = [0.0] * N_SPECIES
    for key in sorted(m):
        if key not in keys:
            raise SceneError(f"{_join(at, key)}: unknown key")
        v = m[key]
        if not (_is_number(v) and math.isfinite(v) and v >= 0.0):
            raise SceneError(f"{_join(at, key)}: must be a number ≥ 0")
        comp[keys.index(key)] = float(v)
    total = 0.0
    for c in comp:
        total += c
    if abs(total - 1.0) > COMPOSITION_TOLERANCE:
        raise SceneError(f"{at}: the fractions sum to {_fmt(total)}, not 1")
    v = f.map.get("v")
    if v is None and "v" not in f.map:
        vel = (0.0, 0.0)
    elif (isinstance(v, list) and len(v) == 2 and all(_is_number(q) and math.isfinite(q) for q in v)):
        vel = (float(v[0]), float(v[1]))
    else:
        raise SceneError(f"{f.path('v')}: must be [vx, vy], two finite numbers")
    return Gas(heat=heat, composition=tuple(comp), v=vel)


def _parse_object(value, at: str) -> Obj:
    kind = value.get("kind") if isinstance(value, dict) else None
    if kind == "preset":
        f = _Fields(value, at, ("kind", "preset", "x", "y"))
        name = f.get("preset")
        name = name if isinstance(name, str) else ""
        if name not in PRESETS:
            raise SceneError(f"{f.path('preset')}: unknown preset {_debug_str(name)} (known: {', '.join(PRESETS)})")
        return Obj(kind="preset", preset=name, x=f.required("x"), y=f.required("y"), mass=UNIT_MASS)
    if kind == "disk":
        f = _Fields(value, at, ("kind", "x", "y", "a", "sigma_c", "t", "pressure", "composition", "v"))
        x, y, a, sc = f.required("x"), f.required("y"), f.positive("a"), f.positive("sigma_c")
        return Obj(kind="disk", x=x, y=y, a=a, sigma_c=sc, gas=_parse_gas(f))
    if kind == "rect":
        f = _Fields(value, at, ("kind", "x0", "y0", "w", "h", "sigma", "t", "pressure", "composition", "v"))
        w, h = f.whole("w"), f.whole("h")
        if w < 1 or h < 1:
            raise SceneError(f"{at}: w and h must be ≥ 1, got {w} × {h}")
        x0, y0, sigma = f.whole("x0"), f.whole("y0"), f.positive("sigma")
        return Obj(kind="rect", x0=x0, y0=y0, w=w, h=h, sigma=sigma, gas=_parse_gas(f))
    raise SceneError(f"{at}.kind: must be \"preset\", \"disk\" or \"rect\"")


def _world_ok(w: int, h: int) -> None:
    ok = lambda n: WORLD_MIN <= n <= WORLD_MAX and n % WORLD_MULTIPLE == 0
    if not (ok(w) and ok(h)):
        raise SceneError(f"world {w} × {h}: width and height must be multiples of {WORLD_MULTIPLE} within "
                         f"[{WORLD_MIN}, {WORLD_MAX}]")


def _no_constants(name):
    raise ValueError(f"not JSON: {name} is not a JSON number")


@dataclass
class Scene:
    width: int
    height: int
    edge: str = "leave"
    slowdown: bool = True
    switches: Switches = field(default_factory=Switches)
    test: TestSettings = field(default_factory=TestSettings)
    objects: list = field(default_factory=list)
    overrides: list = field(default_factory=list)   # [(key, value)] in key order

    # -- reading

    @staticmethod
    def load(path) -> "Scene":
        try:
            with open(path, encoding="utf-8") as fh:
                text = fh.read()
        except OSError as e:
            raise SceneError(f"{path}: {e}") from None
        try:
            return Scene.parse(text)
        except SceneError as e:
            raise SceneError(f"{path}: {e}") from None

    @staticmethod
    def parse(text: str) -> "Scene":
        """Reads and checks a scene (scene.rs:335-402)."""
        try:
            root = json.loads(text, parse_constant=_no_constants)
        except (json.JSONDecodeError, ValueError) as e:
            raise SceneError(f"not JSON: {e}") from None
        top = _Fields(root, "", ("version", "world", "slowdown", "switches", "test", "objects", "overrides"))
        version = top.get("version")
        if not (isinstance(version, int) and not isinstance(version, bool) and version == 1):
            raise SceneError("version: must be 1")
        if "world" not in top.map:
            raise SceneError("world: missing")
        wf = _Fields(top.map["world"], "world", ("width", "height", "edge"))

        def size(key):
            n = wf.whole(key)
            if not 0 <= n < 2 ** 32:
                raise SceneError(f"{wf.path(key)}: out of range")
            return n

        width, height = size("width"), size("height")
        try:
            _world_ok(width, height)
        except SceneError as e:
            raise SceneError(f"world: {e}") from None
        edge = "leave"
        if "edge" in wf.map:
            text_edge = wf.map["edge"] if isinstance(wf.map["edge"], str) else ""
            if text_edge not in ("leave", "bounce"):
                raise SceneError(f"world.edge must be \"leave\" or \"bounce\", got {_debug_str(text_edge)}")
            edge = text_edge
        slowdown = top.flag("slowdown", True)
        switches = Switches()
        if "switches" in top.map:
            s = _Fields(top.map["switches"], "switches",
                        ("gravity", "hydro", "heat", "reactions", "neutrinos", "sinks"))
            switches = Switches(**{k: s.flag(k, True) for k in
                                   ("gravity", "hydro", "heat", "reactions", "neutrinos", "sinks")})
        test = TestSettings()
        if "test" in top.map:
            t = _Fields(top.map["test"], "test", ("pin_temperature", "constant_diffusivity", "flux_limiter"))
            cd = None if t.get("constant_diffusivity") is None else t.positive("constant_diffusivity")
            test = TestSettings(pin_temperature=t.flag("pin_temperature", False), constant_diffusivity=cd,
                                flux_limiter=t.flag("flux_limiter", True))
        objs = top.get("objects")
        if not isinstance(objs, list):
            raise SceneError("objects: must be a list")
        objects = [_parse_object(v, f"objects[{i}]") for i, v in enumerate(objs)]
        overrides = []
        if "overrides" in top.map:
            m = top.map["overrides"]
            if not isinstance(m, dict):
                raise SceneError("overrides: must be an object of physics.json keys")
            for key in sorted(m):
                if key not in _CLASS:
                    raise SceneError(f"overrides.{key}: unknown key (physics.json keys only)")
                if not _is_number(m[key]):
                    raise SceneError(f"overrides.{key}: must be a number")
                overrides.append((key, float(m[key])))
            try:
                Physics.shipped().with_(overrides)
            except SceneError as e:
                raise SceneError(f"overrides: {e}") from None
        return Scene(width=width, height=height, edge=edge, slowdown=slowdown, switches=switches, test=test,
                     objects=objects, overrides=overrides)

    @staticmethod
    def preset(name: str, width: int, height: int, mass: float = UNIT_MASS) -> "Scene":
        """One preset cloud at the world's centre, everything else as a new game (scene.rs:237-262)."""
        if not (math.isfinite(mass) and mass > 0.0):
            raise SceneError(f"preset {name}: the mass must be a finite number > 0, got {_fmt(mass)}")
        if name not in PRESETS:
            raise SceneError(f"unknown preset {_debug_str(name)} (known: {', '.join(PRESETS)})")
        _world_ok(width, height)
        return Scene(width=width, height=height, edge="leave", slowdown=True,
                     objects=[Obj(kind="preset", preset=name, x=width / 2.0, y=height / 2.0, mass=mass)])

    def writes_calibration(self) -> bool:
        return not self.overrides

    def physics(self) -> Physics:
        return Physics.shipped().with_(self.overrides)

    def warnings(self) -> list[str]:
        return [f"preset {o.preset}: the nominal Sun-like disk until calibration gives preset_mass_sb (§2.11)"
                for o in self.objects if o.kind == "preset" and o.preset != "sun" and o.mass == UNIT_MASS]

    # -- laying down

    def _world(self, world):
        w, h = (self.width, self.height) if world is None else world
        _world_ok(w, h)
        return w, h

    def planes(self, world=None, physics: Physics | None = None) -> tuple[np.ndarray, list[str]]:
        """The 14 canonical planes (sigma, mom_x, mom_y, energy, the ten mass fractions) as (14, H, W) f32 for `world`
        (the scene's own, or (W, H): a resized world keeps the objects where they stood relative to its centre), and a
        warning per object that covers no cell (scene.rs:427-471)."""
        w, h = self._world(world)
        physics = self.physics() if physics is None else physics
        eos = Eos(physics)
        shift = (_trunc_half(w - self.width), _trunc_half(h - self.height))
        n = w * h
        s_sigma = np.zeros(n)
        s_mom = np.zeros((2, n))
        s_energy = np.zeros(n)
        s_species = np.zeros((N_SPECIES, n))
        warnings = []
        for k, obj in enumerate(self.objects):
            xs, ys, sig = _cells_of(obj, shift, w, h)
            if xs.size == 0:
                warnings.append(f"objects[{k}] covers no cell of the {w}x{h} world")
                continue
            gas = _sun_gas(xs, ys, sig, obj.mass, physics) if obj.kind == "preset" else obj.gas
            inv_mu, y_e, _ = composition(gas.composition)
            mu, x_n = 1.0 / inv_mu, gas.composition[N_SPECIES - 1]
            if gas.heat[0] == "t":
                eps_th = np.full(sig.shape, Eos.eps_th_of_t(gas.heat[1], mu))
            else:
                p = gas.heat[1]
                thermal = p - eos.pi_e(sig, y_e) - eos.pi_n(sig, x_n)
                bad = np.nonzero(thermal <= 0.0)[0]
                if bad.size:
                    q = bad[0]
                    raise SceneError(f"objects[{k}].pressure: {_fmt(p)} is below the cold pressure at cell "
                                     f"({xs[q]}, {ys[q]})")
                eps_th = thermal / sig
            kinetic = 0.5 * (gas.v[0] * gas.v[0] + gas.v[1] * gas.v[1])
            eps = eps_th + eos.eps_cold(sig, y_e, x_n) + kinetic if eos.cold else eps_th + 0.0 + kinetic
            i = ys * w + xs
            s_sigma[i] += sig
            s_mom[0, i] += sig * gas.v[0]
            s_mom[1, i] += sig * gas.v[1]
            s_energy[i] += sig * eps
            for s in range(N_SPECIES):
                s_species[s, i] += sig * gas.composition[s]
        sigma_floor = physics.get("sigma_floor")
        h_inv_mu, h_y_e, _ = composition([1.0 if s == ID_H else 0.0 for s in range(N_SPECIES)])
        floor_cold = float(eos.eps_cold(np.array([sigma_floor]), h_y_e, 0.0)[0]) if eos.cold else 0.0
        floor_eps = Eos.eps_th_of_t(eos.t_floor, 1.0 / h_inv_mu) + floor_cold
        floor_energy = sigma_floor * floor_eps
        out = np.zeros((N_CHANNELS, n), np.float32)
        gas_cells = s_sigma > 0.0
        out[0] = np.where(gas_cells, s_sigma, sigma_floor)
        out[1] = np.where(gas_cells, s_mom[0], 0.0)
        out[2] = np.where(gas_cells, s_mom[1], 0.0)
        out[3] = np.where(gas_cells, s_energy, floor_energy)
        with np.errstate(divide="ignore", invalid="ignore"):
            for s in range(N_SPECIES):
                out[4 + s] = np.where(gas_cells, s_species[s] / np.where(gas_cells, s_sigma, 1.0),
                                      1.0 if s == ID_H else 0.0)
        return out.reshape(N_CHANNELS, h, w), warnings

    # -- this build's field update

    def config(self, world=None, strict: bool = True, planes: np.ndarray | None = None) -> Config:
        """The scene as this build's Config: world, edge, switches, the test settings and physics.json's constants,
        with gamma = 2 (Pi = Sigma eps_th) and, with heat on, the one mu of the gas. With `strict`, refuses by name
        what the 4-channel field update cannot run as the reference would; without it those parts are left out."""
        w, h = self._world(world)
        physics = self.physics()
        v = physics.values
        sw = self.switches
        if strict:
            for name in ("reactions", "neutrinos", "sinks"):
                if getattr(sw, name):
                    raise SceneError(f"switches.{name}: on, but this build runs the field update only (hydro, "
                                     f"gravity, FLD): switch it off in the scene or load with strict=False")
            for k1, k2 in (("k1e", "k2e"), ("k1n", "k2n")):
                if v[k1] > 0.0:
                    raise SceneError(f"physics: the {k1}/{k2} cold pressure is on, but this build's EOS is the "
                                     f"gamma = 2 ideal gas: override the pair to 0 or load with strict=False")
        mu = 1.0
        if sw.heat:
            mu = self._heat_mu(w, h, physics, planes)
        return Config(width=w, height=h, edge=self.edge, gravity=sw.gravity, hydro=sw.hydro, heat=sw.heat,
                      kernel="self_cell", limiter="mc", thermal_bracket=True, gamma=2.0, mu=mu,
                      t_floor=v["t_floor"], sigma_vac=v["sigma_vac"], sigma_floor=v["sigma_floor"], cfl=v["cfl"],
                      eta_g=v["eta_g"], G=1.0, a_r=v["a_r"], c_sb=v["c_sb"], kappa0=v["kappa0"],
                      k_cond=v["k_cond"], chi=self.test.constant_diffusivity or 0.0,
                      pin_temperature=self.test.pin_temperature, flux_limiter=self.test.flux_limiter,
                      opacity_plane=sw.heat)

    def ref_config(self, world=None, strict: bool = True, m_tov: float = 4853.169981814195) -> Config:
        """The scene as a reference-mode Config (14 channels: the reference's EOS with the cold pairs of its physics,
        the species, the hold), for the planes ``Scene.planes`` lays down. ``m_tov`` is m_tov_sb, the hold's gate
        (assets/calibration.json's value for the shipped physics). With `strict`, refuses by name the switches the
        reference-mode field update does not run (heat, reactions, neutrinos, sinks); without it they are left out."""
        w, h = self._world(world)
        v = self.physics().values
        sw = self.switches
        if strict:
            for name in ("heat", "reactions", "neutrinos", "sinks"):
                if getattr(sw, name):
                    raise SceneError(f"switches.{name}: on, but the reference-mode field update runs hydro and "
                                     f"gravity only: switch it off in the scene or load with strict=False")
        return Config(width=w, height=h, channels=N_CHANNELS, edge=self.edge, gravity=sw.gravity, hydro=sw.hydro,
                      heat=False, kernel="self_cell", limiter="mc", thermal_bracket=True, gamma=2.0, mu=1.0,
                      t_floor=v["t_floor"], sigma_vac=v["sigma_vac"], sigma_floor=v["sigma_floor"], cfl=v["cfl"],
                      eta_g=v["eta_g"], G=1.0, a_r=v["a_r"], c_sb=v["c_sb"], kappa0=v["kappa0"],
                      k_cond=v["k_cond"], k1e=v["k1e"], k2e=v["k2e"], k1n=v["k1n"], k2n=v["k2n"],
                      kappa_dust=v["kappa_dust"], t_dust=v["t_dust"], sigma_hold=v["sigma_hold"],
                      eta_hold=v["eta_hold"], r_hold=v["r_hold"], m_tov=m_tov)

    def _heat_mu(self, w, h, physics, planes):
        """The gas cells' mu (Sigma >= sigma_vac), which must be one: from the compositions of the objects that
        cover gas cells, and hydrogen where the floor state is gas."""
        shift = (_trunc_half(w - self.width), _trunc_half(h - self.height))
        sigma_vac = physics.get("sigma_vac")
        if planes is None:
            planes, _ = self.planes((w, h), physics)
        gas = planes[0].reshape(-1) >= sigma_vac
        covered = np.zeros(w * h, bool)
        comps = set()
        for obj in self.objects:
            xs, ys, _ = _cells_of(obj, shift, w, h)
            if xs.size == 0:
                continue
            i = ys * w + xs
            covered[i] = True
            if gas[i].any():
                comps.add(SUN_MIX if obj.kind == "preset" else obj.gas.composition)
        if (gas & ~covered).any():
            comps.add(tuple(1.0 if s == ID_H else 0.0 for s in range(N_SPECIES)))
        inv = {composition(c)[0] for c in comps}
        if len(comps) > 1 and len(inv) > 1:
            raise SceneError(f"heat: the gas holds {len(comps)} compositions of different mu, but this build's FLD "
                             f"takes one mu per world")
        return 1.0 / inv.pop() if inv else 1.0

    @staticmethod
    def opacity(planes: np.ndarray, physics: Physics) -> np.ndarray:
        """The reference FLD's opacity per cell, kappa0 (1 + X_H) with the dust stand-in off (reference/heat.rs:210-219),
        as an (H, W) f32 plane."""
        return (physics.get("kappa0") * (1.0 + planes[4 + ID_H].astype(np.float64))).astype(np.float32)


def _trunc_half(d: int) -> int:
    return int(d / 2) if d >= 0 else -((-d) // 2)


def _disk_samples(x, y, a, sigma_c):
    """Sigma_c sqrt(1 - r^2/a^2) at the centre of each cell the disk covers, over the whole plane, rows then columns
    (scene.rs:555-566): (i, j, Sigma) arrays, indices signed."""
    j0, j1, i0, i1 = math.floor(y - a), math.ceil(y + a), math.floor(x - a), math.ceil(x + a)
    if j1 <= j0 or i1 <= i0:
        return np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0)
    jj, ii = np.mgrid[j0:j1, i0:i1]
    dx = ii.astype(np.float64) + 0.5 - x
    dy = jj.astype(np.float64) + 0.5 - y
    r2 = (dx * dx + dy * dy) / (a * a)
    keep = r2 < 1.0
    return ii[keep], jj[keep], sigma_c * np.sqrt(1.0 - r2[keep])


def _clip(i, j, s, w, h):
    k = (i >= 0) & (j >= 0) & (i < w) & (j < h)
    return i[k], j[k], s[k]


def cloud_shape(mass: float) -> tuple[float, float]:
    """The preset cloud's radius a = 40 sqrt(M / M0) capped at 150 and central Sigma_c = 3M / (2 pi a^2)
    (scene.rs:577-586)."""
    a = min(SUN_RADIUS * math.sqrt(mass / UNIT_MASS), MAX_RADIUS)
    return a, 3.0 * mass / (2.0 * math.pi * a * a)


def thermal_over_w(mass: float) -> float:
    """A preset's U_th / |W|: min(0.5, 0.1 max(1, M / M0)^2) (scene.rs:588-596)."""
    ratio = max(mass / UNIT_MASS, 1.0)
    return min(THERMAL_OVER_W * ratio * ratio, THERMAL_OVER_W_MAX)


def _cells_of(obj: Obj, shift, w, h):
    """The cells an object covers in a w x h world shifted by `shift`, with its Sigma there (scene.rs:512-553)."""
    if obj.kind == "preset":
        a, sc = cloud_shape(obj.mass)
        x, y = obj.x + shift[0], obj.y + shift[1]
        whole = _disk_samples(x, y, a, sc)[2]
        total = float(np.cumsum(whole)[-1]) if whole.size else 0.0  # summed in order, as the reference does
        k = obj.mass / total if total > 0.0 else 1.0
        i, j, s = _clip(*_disk_samples(x, y, a, sc), w, h)
        return i, j, s * k
    if obj.kind == "disk":
        return _clip(*_disk_samples(obj.x + shift[0], obj.y + shift[1], obj.a, obj.sigma_c), w, h)
    xa, xb = min(max(obj.x0 + shift[0], 0), w), min(max(obj.x0 + shift[0] + obj.w, 0), w)
    ya, yb = min(max(obj.y0 + shift[1], 0), h), min(max(obj.y0 + shift[1] + obj.h, 0), h)
    jj, ii = np.mgrid[ya:yb, xa:xb]
    return ii.reshape(-1), jj.reshape(-1), np.full(ii.size, obj.sigma)


def _potential(src: np.ndarray) -> np.ndarray:
    """phi = K * src over the box, zero-padded (free space), K(i, j) = -1 / sqrt(i^2 + j^2) and K(0, 0) = -SELF_CELL
    (G = 1; reference/grav.rs:25-34, reference/fft.rs:238-282), in f64."""
    bh, bw = src.shape
    px, py = 1 << max(5, (2 * bw - 1).bit_length()), 1 << max(5, (2 * bh - 1).bit_length())
    dx = np.arange(px)
    dx = np.where(dx < px // 2, dx, dx - px).astype(np.float64)
    dy = np.arange(py)
    dy = np.where(dy < py // 2, dy, dy - py).astype(np.float64)
    r2 = dy[:, None] ** 2 + dx[None, :] ** 2
    with np.errstate(divide="ignore"):
        K = -1.0 / np.sqrt(r2)
    K[0, 0] = -SELF_CELL
    pad = np.zeros((py, px))
    pad[:bh, :bw] = src
    phi = np.fft.irfft2(np.fft.rfft2(pad) * np.fft.rfft2(K), s=(py, px))
    return phi[:bh, :bw]


def _sun_gas(xs, ys, sig, preset_mass, physics: Physics) -> Gas:
    """The preset's gas: the Sun's mix, at rest, at the uniform T that makes U_th = thermal_over_w(M) |W| over its own
    cells, W = 1/2 sum m phi from one gravity solve over the cells' bounding box, vacuum no source (scene.rs:598-618)."""
    sigma_vac = physics.get("sigma_vac")
    x0, x1, y0, y1 = int(xs.min()), int(xs.max()), int(ys.min()), int(ys.max())
    src = np.zeros((y1 - y0 + 1, x1 - x0 + 1))
    src[ys - y0, xs - x0] = np.where(sig >= sigma_vac, sig, 0.0)
    phi = _potential(src)
    w_sum = 0.5 * float(np.cumsum((src * phi).reshape(-1))[-1])
    mass = float(np.cumsum(sig)[-1])
    eps_th = thermal_over_w(preset_mass) * abs(w_sum) / mass
    mu = 1.0 / composition(SUN_MIX)[0]
    return Gas(heat=("t", mu * eps_th), composition=SUN_MIX, v=(0.0, 0.0))


def load(path) -> Scene:
    return Scene.load(path)


def parse(text: str) -> Scene:
    return Scene.parse(text)


def load_into(step, scene: Scene, strict: bool = True) -> np.ndarray:
    """Uploads `scene`'s state (Sigma, Sigma u, Sigma v, E) into `step` (a sandbox_reactions_b200.engine.Step made with
    ``scene.config(...)`` for the same world) and, with heat on, the opacity plane; returns the 14 planes."""
    c, h, w = step.shape
    physics = scene.physics()
    planes, _ = scene.planes((w, h), physics)
    if strict:
        scene.config((w, h), strict=True, planes=planes)
    step.upload(np.ascontiguousarray(planes[:4]))
    if scene.switches.heat:
        step.upload_opacity(Scene.opacity(planes, physics))
    return planes
