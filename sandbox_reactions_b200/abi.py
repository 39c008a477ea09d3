"""ctypes mirror of include/sr_cuda.h: the structs of the C ABI and the defaults of a run.

The defaults are the reference's shipped constants (assets/physics.json) and scheme: the monotonised-central limiter,
bounce edges, γ = 2 and the exact self-cell gravity kernel (crates/sr-physics/src/reference/hydro.rs:1-60,
reference/grav.rs:1-34). `sr_config_default` in the library fills the same values.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field, fields

SR_OK, SR_E_INVALID, SR_E_NONFINITE, SR_E_TIMEOUT, SR_E_CUDA, SR_E_NOMEM, SR_E_UNSUPPORTED = range(7)
STATUS_NAMES = {0: "SR_OK", 1: "SR_E_INVALID", 2: "SR_E_NONFINITE", 3: "SR_E_TIMEOUT", 4: "SR_E_CUDA",
                5: "SR_E_NOMEM", 6: "SR_E_UNSUPPORTED"}

EDGE = {"bounce": 0, "leave": 1}
LIMITER = {"mc": 0, "minmod": 1}
KERNEL = {"self_cell": 0, "softened": 1}
PRECOND = {"mg": 0, "jacobi": 1, "learned": 2}


class sr_config(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32),
        ("width", C.c_uint32), ("height", C.c_uint32),
        ("channels", C.c_uint32), ("edge", C.c_uint32), ("limiter", C.c_uint32), ("thermal_bracket", C.c_uint32),
        ("gravity", C.c_uint32), ("hydro", C.c_uint32), ("heat", C.c_uint32),
        ("kernel", C.c_uint32), ("precond", C.c_uint32), ("flux_limiter", C.c_uint32), ("opacity_plane", C.c_uint32),
        ("mg_pre", C.c_uint32), ("mg_post", C.c_uint32), ("max_passes", C.c_uint32), ("max_rounds", C.c_uint32),
        ("pin_temperature", C.c_uint32), ("active_box", C.c_uint32), ("reserved", C.c_uint32 * 3),
        ("gamma", C.c_double), ("mu", C.c_double), ("t_floor", C.c_double), ("sigma_vac", C.c_double),
        ("sigma_floor", C.c_double), ("cfl", C.c_double), ("eta_g", C.c_double), ("G", C.c_double),
        ("softening", C.c_double), ("a_r", C.c_double), ("c_sb", C.c_double), ("kappa0", C.c_double),
        ("k_cond", C.c_double), ("chi", C.c_double), ("solve_tol", C.c_double), ("newton_heat", C.c_double),
        ("newton_cell", C.c_double), ("dt_fixed", C.c_double), ("dt_cap", C.c_double),
        ("mg_omega", C.c_double), ("inner_tol", C.c_double), ("reserved_d", C.c_double * 2),
        ("k1e", C.c_double), ("k2e", C.c_double), ("k1n", C.c_double), ("k2n", C.c_double),
        ("kappa_dust", C.c_double), ("t_dust", C.c_double), ("sigma_hold", C.c_double), ("eta_hold", C.c_double),
        ("r_hold", C.c_double), ("m_tov", C.c_double),
    ]


class sr_dt_report(C.Structure):
    _fields_ = [("dt", C.c_double), ("dt_next", C.c_double), ("steps", C.c_uint64), ("sim_time", C.c_double),
                ("non_finite", C.c_int32), ("nf_channel", C.c_int32), ("nf_cell", C.c_int64)]


class sr_heat_report(C.Structure):
    _fields_ = [("dt", C.c_double), ("passes", C.c_uint32), ("rounds", C.c_uint32), ("refinements", C.c_uint32),
                ("converged", C.c_uint32), ("delta", C.c_double), ("radiated", C.c_double),
                ("rel_residual", C.c_double), ("fallback_used", C.c_uint32), ("precond", C.c_uint32)]


class sr_box_report(C.Structure):
    _fields_ = [("x0", C.c_uint32), ("y0", C.c_uint32), ("w", C.c_uint32), ("h", C.c_uint32), ("fft_w", C.c_uint32),
                ("fft_h", C.c_uint32), ("fits", C.c_uint64)]


class sr_cost(C.Structure):
    _fields_ = [("steps", C.c_uint32), ("pad", C.c_uint32), ("gravity_ms", C.c_double), ("hydro_ms", C.c_double),
                ("heat_ms", C.c_double), ("floors_ms", C.c_double), ("dt_ms", C.c_double), ("total_ms", C.c_double),
                ("hydro_update_ms", C.c_double), ("hydro_update_launches", C.c_uint32), ("pad2", C.c_uint32),
                ("kernel_launches", C.c_uint64)]


@dataclass
class Config:
    """A run's configuration (the scene's world and switches, the scheme, physics.json's constants)."""
    width: int = 64
    height: int = 64
    channels: int = 4           # 14: reference mode (the reference's EOS with species and cold pressures, the hold)
    edge: str = "bounce"
    limiter: str = "mc"
    thermal_bracket: bool = True
    gravity: bool = False
    hydro: bool = True
    heat: bool = False
    kernel: str = "self_cell"
    precond: str = "mg"
    flux_limiter: bool = True
    opacity_plane: bool = False
    mg_pre: int = 4
    mg_post: int = 4
    max_passes: int = 128
    max_rounds: int = 4096
    pin_temperature: bool = False
    active_box: bool = False    # step only the box around the gas (the reference's BoxMode::Fit); False: the whole world
    gamma: float = 2.0
    mu: float = 1.0
    t_floor: float = 0.05
    sigma_vac: float = 1e-6
    sigma_floor: float = 1e-8
    cfl: float = 0.4
    eta_g: float = 0.3
    G: float = 1.0
    softening: float = 1.0
    a_r: float = 6.25e-7
    c_sb: float = 12800.0
    kappa0: float = 1.0
    k_cond: float = 0.0
    chi: float = 0.0
    solve_tol: float = 1e-8
    newton_heat: float = 1e-6   # the reference GPU path's Newton stop (crates/sr-engine/shaders/heat.wgsl:355-357)
    newton_cell: float = 1e-3
    dt_fixed: float = 0.0
    dt_cap: float = 0.0
    mg_omega: float = 0.0
    inner_tol: float = 0.0
    # reference mode only (channels 14): physics.json's cold pairs, dust stand-in and hold, and m_tov_sb
    # (assets/calibration.json)
    k1e: float = 21.3
    k2e: float = 134.0
    k1n: float = 2.67
    k2n: float = 58.2
    kappa_dust: float = 0.0
    t_dust: float = 0.0
    sigma_hold: float = 10.0
    eta_hold: float = 0.1
    r_hold: float = 24.0
    m_tov: float = 4853.169981814195

    def to_c(self) -> sr_config:
        c = sr_config()
        c.struct_size = C.sizeof(sr_config)
        enums = {"edge": EDGE, "limiter": LIMITER, "kernel": KERNEL, "precond": PRECOND}
        for f in fields(self):
            v = getattr(self, f.name)
            if f.name in enums:
                v = enums[f.name][v]
            setattr(c, f.name, int(v) if isinstance(v, bool) else v)
        return c

    def replace(self, **kw) -> "Config":
        d = {f.name: getattr(self, f.name) for f in fields(self)}
        d.update(kw)
        return Config(**d)

    @property
    def cells(self) -> int:
        return self.width * self.height
