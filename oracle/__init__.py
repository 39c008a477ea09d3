"""TEST INFRASTRUCTURE ONLY: ctypes bindings of the CPU f64 oracle (oracle/sr_oracle.c).

The oracle restates the reference's own CPU twin (crates/sr-physics/src/reference/*.rs) in C. Only tests/,
__graft_entry__.smoke() and bench.py's CPU baseline import this module; the product path never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from sandbox_reactions_b200.abi import Config, sr_config

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsroracle.so")

_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)


class or_hydro_report(C.Structure):
    _fields_ = [("kick_net", C.c_double * 2), ("densest", C.c_int64), ("escaped", C.c_double * 4)]


class or_ref_hydro_report(C.Structure):
    _fields_ = [("spared", C.c_double * 2), ("kick_net", C.c_double * 2), ("densest", C.c_int64),
                ("push_net", C.c_double * 2), ("push_abs", C.c_double)]


class or_heat_report(C.Structure):
    _fields_ = [("passes", C.c_int64), ("rounds", C.c_int64), ("delta", C.c_double), ("converged", C.c_int32),
                ("pad", C.c_int32), ("radiated", C.c_double)]


def build() -> str:
    """Compiles the oracle (gcc, OpenMP) when its library is missing or older than its sources."""
    src = [os.path.join(HERE, f) for f in ("sr_oracle.c", "sr_oracle_ref.c", "sr_oracle.h", "Makefile",
                                           os.path.join("..", "include", "sr_cuda.h"))]
    if not os.path.exists(LIB_PATH) or max(os.path.getmtime(s) for s in src) > os.path.getmtime(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER(sr_config)
        L.or_padded_size.restype = C.c_int64
        L.or_padded_size.argtypes = [C.c_int64, C.c_int64]
        L.or_fft.argtypes = [C.c_int64, _D, _D, C.c_int]
        L.or_fft2.argtypes = [C.c_int64, C.c_int64, _D, _D, C.c_int]
        L.or_convolve_ringed.argtypes = [_D, C.c_int64, C.c_int64, C.c_int64, _D, C.c_int64, C.c_int64, _D]
        L.or_kernel_table.argtypes = [P, C.c_int64, C.c_int64, _D]
        L.or_grav_field.argtypes = [P, _D, C.c_int64, C.c_int64, _D, _D, _D]
        L.or_direct_potential.argtypes = [P, _D, C.c_int64, C.c_int64, C.c_int64, _I64, _I64, _D]
        L.or_hydro_step.argtypes = [P, _D, C.c_int64, C.c_int64, C.c_double, _D, _D, C.POINTER(or_hydro_report)]
        L.or_hydro_dt.restype = C.c_double
        L.or_hydro_dt.argtypes = [P, _D, C.c_int64, C.c_int64, _D, _D]
        L.or_floors.argtypes = [P, _D, C.c_int64, C.c_int64]
        L.or_lambda.restype = C.c_double
        L.or_lambda.argtypes = [C.c_double]
        L.or_heat_step.argtypes = [P, _D, _D, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double,
                                   C.POINTER(or_heat_report), _D, _D]
        L.or_heat_law.argtypes = [P, _D, _D, C.c_int64, C.c_int64, _D, _D]
        L.or_heat_system.argtypes = [P, _D, _D, C.c_int64, C.c_int64, C.c_double, _D, _D, _D, _D,
                                     C.POINTER(C.c_uint8)]
        L.or_heat_matvec.argtypes = [C.c_int64, C.c_int64, _D, _D, _D, C.POINTER(C.c_uint8), _D, _D]
        L.or_heat_pcg.restype = C.c_int64
        L.or_heat_pcg.argtypes = [C.c_int64, C.c_int64, _D, _D, _D, _D, C.POINTER(C.c_uint8), C.c_double, C.c_int64,
                                  _D]
        L.or_riemann_solve.argtypes = [C.c_double] * 7 + [_D]
        L.or_riemann_sample.argtypes = [C.c_double] * 7 + [_D, C.c_double, _D]
        L.or_twin_new.restype = C.c_void_p
        L.or_twin_new.argtypes = [P, _D, _D]
        L.or_twin_free.argtypes = [C.c_void_p]
        L.or_twin_step.argtypes = [C.c_void_p]
        L.or_twin_state.argtypes = [C.c_void_p, _D]
        L.or_twin_clock.argtypes = [C.c_void_p, _D]
        L.or_twin_field.argtypes = [C.c_void_p, _D, _D, _D]
        L.or_twin_heat.argtypes = [C.c_void_p, C.POINTER(or_heat_report), _D, _D]
        U8 = C.POINTER(C.c_uint8)
        L.or_cold_pressure.restype = C.c_double
        L.or_cold_pressure.argtypes = [C.c_double] * 3
        L.or_cold_energy_exact.restype = C.c_double
        L.or_cold_energy_exact.argtypes = [C.c_double] * 3
        L.or_cold_table.argtypes = [C.c_double, C.c_double, _D]
        L.or_cold_table_u.restype = C.c_double
        L.or_cold_table_u.argtypes = [_D, C.c_double]
        L.or_composition.argtypes = [_D, _D]
        L.or_ref_hydro_step.argtypes = [P, _D, C.c_int64, C.c_int64, C.c_double, _D, _D, U8, _D, _D,
                                        C.POINTER(or_ref_hydro_report)]
        L.or_ref_dt.restype = C.c_double
        L.or_ref_dt.argtypes = [P, _D, C.c_int64, C.c_int64, _D, _D]
        L.or_ref_floors.argtypes = [P, _D, C.c_int64, C.c_int64, _D]
        L.or_ref_disk_mass.restype = C.c_double
        L.or_ref_disk_mass.argtypes = [_D, C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_double]
        L.or_ref_hold.argtypes = [P, _D, C.c_int64, C.c_int64, U8, _D]
        L.or_ref_twin_new.restype = C.c_void_p
        L.or_ref_twin_new.argtypes = [P, _D, U8]
        L.or_ref_twin_free.argtypes = [C.c_void_p]
        L.or_ref_twin_set_flux.argtypes = [C.c_void_p, _D, _D]
        L.or_ref_twin_step.argtypes = [C.c_void_p]
        L.or_ref_twin_state.argtypes = [C.c_void_p, _D, U8]
        L.or_ref_twin_clock.argtypes = [C.c_void_p, _D]
        L.or_ref_twin_books.argtypes = [C.c_void_p, _D]
        L.or_ref_twin_heat.argtypes = [C.c_void_p, C.POINTER(or_heat_report), _D, _D]
        L.or_ref_heat_sides.argtypes = [P, _D, C.c_int64, C.c_int64, _D, _D, _D]
        L.or_ref_heat_step.argtypes = [P, _D, C.c_int64, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.POINTER(or_heat_report), _D, _D]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_get_threads.restype = C.c_int
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def set_threads(n: int) -> None:
    lib().or_set_threads(int(n))


def threads() -> int:
    return lib().or_get_threads()


# ---------------------------------------------------------------- FFT / gravity
def padded_size(n: int, cap: int = 2048) -> int:
    return int(lib().or_padded_size(n, cap))


def fft(x: np.ndarray, inverse: bool = False) -> np.ndarray:
    re, im = _f64(np.real(x)).copy(), _f64(np.imag(x)).copy()
    if lib().or_fft(len(re), _p(re), _p(im), int(inverse)) != 0:
        raise ValueError(f"FFT length {len(re)} is not a power of two")
    return re + 1j * im


def fft2(x: np.ndarray, inverse: bool = False) -> np.ndarray:
    ny, nx = x.shape
    re, im = _f64(np.real(x)).copy(), _f64(np.imag(x)).copy()
    if lib().or_fft2(nx, ny, _p(re), _p(im), int(inverse)) != 0:
        raise ValueError("not a power of two")
    return re + 1j * im


def convolve_ringed(field: np.ndarray, ktab: np.ndarray, ring: int = 0) -> np.ndarray:
    h, w = field.shape
    py, px = ktab.shape
    out = np.zeros((h + 2 * ring, w + 2 * ring))
    f, k = _f64(field), _f64(ktab)
    if lib().or_convolve_ringed(_p(f), w, h, ring, _p(k), px, py, _p(out)) != 0:
        raise ValueError("bad padded size")
    return out


def kernel_table(cfg: Config, px: int, py: int) -> np.ndarray:
    out = np.zeros((py, px))
    c = cfg.to_c()
    lib().or_kernel_table(C.byref(c), px, py, _p(out))
    return out


def grav_field(cfg: Config, sigma: np.ndarray):
    h, w = sigma.shape
    phi, gx, gy = (np.zeros((h, w)) for _ in range(3))
    c = cfg.to_c()
    s = _f64(sigma)
    if lib().or_grav_field(C.byref(c), _p(s), w, h, _p(phi), _p(gx), _p(gy)) != 0:
        raise ValueError("box pads outside the FFT")
    return phi, gx, gy


def direct_potential(cfg: Config, src: np.ndarray, tx, ty) -> np.ndarray:
    h, w = src.shape
    tx = np.ascontiguousarray(tx, dtype=np.int64)
    ty = np.ascontiguousarray(ty, dtype=np.int64)
    out = np.zeros(len(tx))
    c = cfg.to_c()
    s = _f64(src)
    lib().or_direct_potential(C.byref(c), _p(s), w, h, len(tx), tx.ctypes.data_as(_I64), ty.ctypes.data_as(_I64),
                              _p(out))
    return out


# ---------------------------------------------------------------- hydro
def hydro_step(cfg: Config, planes: np.ndarray, dt: float, g=None):
    """One P4 step on (4, H, W) f64 planes; `g` = (gx, gy) of the start state or None. Returns (planes, report)."""
    p = _f64(planes).copy()
    _, h, w = p.shape
    rep = or_hydro_report()
    c = cfg.to_c()
    if g is None:
        lib().or_hydro_step(C.byref(c), _p(p), w, h, dt, None, None, C.byref(rep))
    else:
        gx, gy = _f64(g[0]), _f64(g[1])
        lib().or_hydro_step(C.byref(c), _p(p), w, h, dt, _p(gx), _p(gy), C.byref(rep))
    return p, rep


def hydro_dt(cfg: Config, planes: np.ndarray, g=None) -> float:
    p = _f64(planes)
    _, h, w = p.shape
    c = cfg.to_c()
    if g is None:
        return lib().or_hydro_dt(C.byref(c), _p(p), w, h, None, None)
    gx, gy = _f64(g[0]), _f64(g[1])
    return lib().or_hydro_dt(C.byref(c), _p(p), w, h, _p(gx), _p(gy))


def floors(cfg: Config, planes: np.ndarray) -> np.ndarray:
    p = _f64(planes).copy()
    _, h, w = p.shape
    c = cfg.to_c()
    lib().or_floors(C.byref(c), _p(p), w, h)
    return p


# ---------------------------------------------------------------- heat
def lam(r: float) -> float:
    return lib().or_lambda(r)


def heat_step(cfg: Config, planes: np.ndarray, dt: float, kappa=None, tol=1e-12, newton_heat=1e-12,
              newton_cell=1e-10):
    """One implicit FLD step; returns (planes, report, fx, fy)."""
    p = _f64(planes).copy()
    _, h, w = p.shape
    fx = np.zeros((h, w + 1))
    fy = np.zeros((h + 1, w))
    rep = or_heat_report()
    c = cfg.to_c()
    k = _f64(kappa) if kappa is not None else None
    lib().or_heat_step(C.byref(c), _p(p), _p(k) if k is not None else None, w, h, dt, tol, newton_heat, newton_cell,
                       C.byref(rep), _p(fx), _p(fy))
    return p, rep, fx, fy


def heat_law(cfg: Config, planes: np.ndarray, kappa=None):
    p = _f64(planes)
    _, h, w = p.shape
    fx = np.zeros((h, w + 1))
    fy = np.zeros((h + 1, w))
    c = cfg.to_c()
    k = _f64(kappa) if kappa is not None else None
    lib().or_heat_law(C.byref(c), _p(p), _p(k) if k is not None else None, w, h, _p(fx), _p(fy))
    return fx, fy


def heat_system(cfg: Config, planes: np.ndarray, dt: float, kappa=None):
    p = _f64(planes)
    _, h, w = p.shape
    diag, rhs = np.zeros((h, w)), np.zeros((h, w))
    kx, ky = np.zeros((h, w + 1)), np.zeros((h + 1, w))
    gas = np.zeros((h, w), dtype=np.uint8)
    c = cfg.to_c()
    k = _f64(kappa) if kappa is not None else None
    lib().or_heat_system(C.byref(c), _p(p), _p(k) if k is not None else None, w, h, dt, _p(diag), _p(rhs), _p(kx),
                         _p(ky), gas.ctypes.data_as(C.POINTER(C.c_uint8)))
    return diag, rhs, kx, ky, gas


def heat_matvec(diag, kx, ky, gas, x):
    h, w = diag.shape
    y = np.zeros((h, w))
    xx = _f64(x)
    lib().or_heat_matvec(w, h, _p(_f64(diag)), _p(_f64(kx)), _p(_f64(ky)), gas.ctypes.data_as(C.POINTER(C.c_uint8)),
                         _p(xx), _p(y))
    return y


def heat_pcg(diag, rhs, kx, ky, gas, rel=1e-8, max_rounds=100000, x0=None):
    h, w = diag.shape
    x = np.zeros((h, w)) if x0 is None else _f64(x0).copy()
    r = lib().or_heat_pcg(w, h, _p(_f64(diag)), _p(_f64(rhs)), _p(_f64(kx)), _p(_f64(ky)),
                          gas.ctypes.data_as(C.POINTER(C.c_uint8)), rel, max_rounds, _p(x))
    return x, int(r)


# ---------------------------------------------------------------- Riemann
class Riemann:
    """The exact solution of a 1D Riemann problem for an ideal gas of index γ (reference/riemann.rs)."""

    def __init__(self, gamma, left, right):
        self.gamma, self.left, self.right = gamma, left, right
        self.sol = np.zeros(10)
        rc = lib().or_riemann_solve(gamma, *left, *right, _p(self.sol))
        if rc:
            raise ValueError({1: "bad state", 2: "vacuum", 3: "no convergence"}[rc])

    @property
    def p_star(self):
        return self.sol[0]

    @property
    def u_star(self):
        return self.sol[1]

    def sample(self, xi: float):
        out = np.zeros(3)
        lib().or_riemann_sample(self.gamma, *self.left, *self.right, _p(self.sol), xi, _p(out))
        return out


# ---------------------------------------------------------------- twin
class Twin:
    """The twin's step driver (reference/mod.rs:94-297) on 4 f64 planes."""

    def __init__(self, cfg: Config, planes: np.ndarray, kappa=None):
        self.cfg = cfg
        self._c = cfg.to_c()
        p = _f64(planes)
        k = _f64(kappa) if kappa is not None else None
        self._t = lib().or_twin_new(C.byref(self._c), _p(p), _p(k) if k is not None else None)

    def __del__(self):
        if getattr(self, "_t", None):
            lib().or_twin_free(self._t)
            self._t = None

    def step(self, n: int = 1):
        for _ in range(n):
            lib().or_twin_step(self._t)

    def state(self) -> np.ndarray:
        out = np.zeros((4, self.cfg.height, self.cfg.width))
        lib().or_twin_state(self._t, _p(out))
        return out

    def clock(self):
        out = np.zeros(4)
        lib().or_twin_clock(self._t, _p(out))
        return {"dt": out[0], "dt_next": out[1], "sim_time": out[2], "steps": int(out[3])}

    def field(self):
        h, w = self.cfg.height, self.cfg.width
        phi, gx, gy = np.zeros((h, w)), np.zeros((h, w)), np.zeros((h, w))
        lib().or_twin_field(self._t, _p(phi), _p(gx), _p(gy))
        return phi, gx, gy

    def heat(self):
        h, w = self.cfg.height, self.cfg.width
        rep = or_heat_report()
        fx, fy = np.zeros((h, w + 1)), np.zeros((h + 1, w))
        lib().or_twin_heat(self._t, C.byref(rep), _p(fx), _p(fy))
        return rep, fx, fy


# ---------------------------------------------------------------- reference mode (14 channels)
def _u8(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint8)


def _pu8(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def cold_pressure(x: float, k1: float, k2: float) -> float:
    return lib().or_cold_pressure(x, k1, k2)


def cold_energy_exact(x: float, k1: float, k2: float) -> float:
    return lib().or_cold_energy_exact(x, k1, k2)


def cold_table(k1: float, k2: float) -> np.ndarray:
    """ln u at the 512 nodes (eos.rs:81-98)."""
    out = np.zeros(512)
    lib().or_cold_table(k1, k2, _p(out))
    return out


def cold_table_u(ln_u: np.ndarray, x: float) -> float:
    return lib().or_cold_table_u(_p(_f64(ln_u)), x)


def composition(x) -> tuple[float, float, float]:
    out = np.zeros(3)
    lib().or_composition(_p(_f64(x)), _p(out))
    return float(out[0]), float(out[1]), float(out[2])


def ref_hydro_step(cfg: Config, planes: np.ndarray, dt: float, g=None, held=None, rad=None):
    """One reference-mode P4 step on (14, H, W) f64 planes (step_held): `g` = (gx, gy) of the start state, `held` the
    hold's (H, W) mask, `rad` = (Fx, Fy) cell-centred for the radiation force. Returns (planes, report)."""
    p = _f64(planes).copy()
    _, h, w = p.shape
    rep = or_ref_hydro_report()
    c = cfg.to_c()
    gx, gy = (_f64(g[0]), _f64(g[1])) if g is not None else (None, None)
    m = _u8(held) if held is not None else None
    rx, ry = (_f64(rad[0]), _f64(rad[1])) if rad is not None else (None, None)
    lib().or_ref_hydro_step(C.byref(c), _p(p), w, h, dt, _p(gx) if gx is not None else None,
                            _p(gy) if gy is not None else None, _pu8(m) if m is not None else None,
                            _p(rx) if rx is not None else None, _p(ry) if ry is not None else None, C.byref(rep))
    return p, rep


def ref_dt(cfg: Config, planes: np.ndarray, g=None) -> float:
    p = _f64(planes)
    _, h, w = p.shape
    c = cfg.to_c()
    if g is None:
        return lib().or_ref_dt(C.byref(c), _p(p), w, h, None, None)
    return lib().or_ref_dt(C.byref(c), _p(p), w, h, _p(_f64(g[0])), _p(_f64(g[1])))


def ref_floors(cfg: Config, planes: np.ndarray):
    """P8's floors on (14, H, W) planes; returns (planes, (vacuum_reset, floor_added))."""
    p = _f64(planes).copy()
    _, h, w = p.shape
    booked = np.zeros(2)
    c = cfg.to_c()
    lib().or_ref_floors(C.byref(c), _p(p), w, h, _p(booked))
    return p, (float(booked[0]), float(booked[1]))


def ref_hold(cfg: Config, planes: np.ndarray, held=None):
    """The hold after P8: returns (planes with newly held momenta zeroed, mask, taken momentum)."""
    p = _f64(planes).copy()
    _, h, w = p.shape
    m = np.zeros((h, w), np.uint8) if held is None else _u8(held).copy()
    taken = np.zeros(2)
    c = cfg.to_c()
    lib().or_ref_hold(C.byref(c), _p(p), w, h, _pu8(m), _p(taken))
    return p, m, (float(taken[0]), float(taken[1]))


def disk_mass(sigma: np.ndarray, x: int, y: int, r: float) -> float:
    s = _f64(sigma)
    h, w = s.shape
    return lib().or_ref_disk_mass(_p(s), w, h, x, y, r)


class RefTwin:
    """The reference-mode twin (reference/mod.rs:129-297 without P5) on 14 f64 planes: the hold's rule on the initial
    state, then per step P1, P2, P4 (step_held), P8 and the hold, P9."""

    def __init__(self, cfg: Config, planes: np.ndarray, mask=None):
        self.cfg = cfg
        self._c = cfg.to_c()
        p = _f64(planes)
        m = _u8(mask) if mask is not None else None
        self._t = lib().or_ref_twin_new(C.byref(self._c), _p(p), _pu8(m) if m is not None else None)

    def __del__(self):
        if getattr(self, "_t", None):
            lib().or_ref_twin_free(self._t)
            self._t = None

    def set_flux(self, fx: np.ndarray, fy: np.ndarray):
        lib().or_ref_twin_set_flux(self._t, _p(_f64(fx)), _p(_f64(fy)))

    def step(self, n: int = 1):
        for _ in range(n):
            lib().or_ref_twin_step(self._t)

    def state(self):
        h, w = self.cfg.height, self.cfg.width
        out = np.zeros((14, h, w))
        m = np.zeros((h, w), np.uint8)
        lib().or_ref_twin_state(self._t, _p(out), _pu8(m))
        return out, m

    def clock(self):
        out = np.zeros(4)
        lib().or_ref_twin_clock(self._t, _p(out))
        return {"dt": out[0], "dt_next": out[1], "sim_time": out[2], "steps": int(out[3])}

    def books(self):
        out = np.zeros(4)
        lib().or_ref_twin_books(self._t, _p(out))
        return {"held": (out[0], out[1]), "vacuum_reset": out[2], "floor_added": out[3]}

    def heat(self):
        h, w = self.cfg.height, self.cfg.width
        rep = or_heat_report()
        fx, fy = np.zeros((h, w + 1)), np.zeros((h + 1, w))
        lib().or_ref_twin_heat(self._t, C.byref(rep), _p(fx), _p(fy))
        return rep, fx, fy


def ref_heat_sides(cfg: Config, planes: np.ndarray):
    """P5's sides of a (14, H, W) state: T⁰, κ and 1/μ per cell (heat.rs:215-231)."""
    p = _f64(planes)
    _, h, w = p.shape
    t0, kappa, inv_mu = np.zeros((h, w)), np.zeros((h, w)), np.zeros((h, w))
    c = cfg.to_c()
    lib().or_ref_heat_sides(C.byref(c), _p(p), w, h, _p(t0), _p(kappa), _p(inv_mu))
    return t0, kappa, inv_mu


def ref_heat_step(cfg: Config, planes: np.ndarray, dt: float, tol=1e-12, newton_heat=1e-12, newton_cell=1e-10):
    """One reference-mode implicit FLD step on (14, H, W) planes; returns (planes, report, fx, fy)."""
    p = _f64(planes).copy()
    _, h, w = p.shape
    fx, fy = np.zeros((h, w + 1)), np.zeros((h + 1, w))
    rep = or_heat_report()
    c = cfg.to_c()
    lib().or_ref_heat_step(C.byref(c), _p(p), w, h, dt, tol, newton_heat, newton_cell, C.byref(rep), _p(fx), _p(fy))
    return p, rep, fx, fy
