"""Host-side mirror of the reference's `sr-engine` step API over the C ABI (include/sr_cuda.h).

`Step` plays the part of the reference's `Step` + `State` pair (crates/sr-engine/src/step/mod.rs:367-777,
crates/sr-engine/src/state.rs:139-279): it is built from a world configuration, takes the canonical channel-major f32
planes by `upload`, advances by `run(steps)` and reports Δt, the implicit step, the gravity field and the flux through
the same calls. Every call goes through libsrcuda.so; there is no CPU path: when the library cannot be loaded the
constructor raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from .abi import (PRECOND, EDGE, STATUS_NAMES, Config, sr_box_report, sr_config, sr_cost, sr_dt_report,
                  sr_heat_report)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsrcuda.so")

_lib = None


class SrError(RuntimeError):
    """A refused or failed call: the status name and the library's message (the reference's FftError/StateError)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


def load_library(path: str = LIB_PATH):
    """Loads libsrcuda.so (built by `sandbox_reactions_b200.build`); raises when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m sandbox_reactions_b200.build`")
    L = C.CDLL(path)
    P = C.c_void_p
    F = C.POINTER(C.c_float)
    D = C.POINTER(C.c_double)
    L.sr_config_default.argtypes = [C.POINTER(sr_config)]
    L.sr_abi_version.restype = C.c_uint32
    L.sr_create.argtypes = [C.POINTER(sr_config), C.POINTER(P)]
    L.sr_destroy.argtypes = [P]
    L.sr_upload.argtypes = [P, F, C.c_uint32]
    L.sr_readback.argtypes = [P, F, C.c_uint32]
    L.sr_upload_opacity.argtypes = [P, F]
    L.sr_upload_held.argtypes = [P, C.POINTER(C.c_uint32)]
    L.sr_read_held.argtypes = [P, C.POINTER(C.c_uint32)]
    L.sr_read_box.argtypes = [P, C.POINTER(sr_box_report)]
    L.sr_step.argtypes = [P, C.c_uint32]
    L.sr_read_dt.argtypes = [P, C.POINTER(sr_dt_report)]
    L.sr_read_heat.argtypes = [P, C.POINTER(sr_heat_report)]
    L.sr_gravity_field.argtypes = [P, F, F, F]
    L.sr_heat_flux.argtypes = [P, F, F]
    L.sr_set_clock.argtypes = [P, C.c_uint64, C.c_double, C.c_double, C.c_double]
    L.sr_read_heat_rate.argtypes = [P, F]
    L.sr_set_heat_rate.argtypes = [P, F]
    L.sr_read_side_flux.argtypes = [P, F, F]
    L.sr_set_side_flux.argtypes = [P, F, F]
    L.sr_set_edge_mode.argtypes = [P, C.c_uint32]
    L.sr_set_heat_precond.argtypes = [P, C.c_uint32]
    L.sr_set_heat_limits.argtypes = [P, C.c_uint32, C.c_uint32]
    L.sr_set_timing.argtypes = [P, C.c_int32]
    L.sr_read_cost.argtypes = [P, C.POINTER(sr_cost)]
    U32P = C.POINTER(C.c_uint32)
    L.sr_heat_first_solve.argtypes = [P, C.c_double, C.c_uint32, D, U32P, D, D, U32P]
    L.sr_learner_create.argtypes = [C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(P)]
    L.sr_learner_destroy.argtypes = [P]
    L.sr_learner_destroy.restype = None
    L.sr_learner_param_count.argtypes = []
    L.sr_learner_param_count.restype = C.c_uint32
    L.sr_learner_get_params.argtypes = [P, F]
    L.sr_learner_set_params.argtypes = [P, F]
    L.sr_learner_collect.argtypes = [P, P, C.c_double, C.c_uint32, C.c_uint64, U32P]
    L.sr_learner_train.argtypes = [P, C.c_uint32, C.c_uint32, C.c_double, C.c_uint64, D]
    L.sr_learner_loss_grad.argtypes = [P, F, F, C.c_uint32, D, F, F]
    L.sr_attach_learner.argtypes = [P, P]
    L.sr_time_smoother.argtypes = [P, C.c_uint32, D, D]
    L.sr_time_smoother.restype = C.c_int
    for name in ("sr_learner_create", "sr_learner_get_params", "sr_learner_set_params", "sr_learner_collect",
                 "sr_learner_train", "sr_learner_loss_grad", "sr_attach_learner"):
        getattr(L, name).restype = C.c_int
    L.sr_gravity_solve_static.argtypes = [C.POINTER(sr_config), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p]
    L.sr_gravity_solve_static.restype = C.c_int
    L.sr_batch_create.argtypes = [C.POINTER(sr_config), C.c_uint32, C.c_uint32, C.POINTER(P)]
    L.sr_batch_destroy.argtypes = [P]
    L.sr_batch_upload.argtypes = [P, C.c_uint32, F, F]
    L.sr_batch_step.argtypes = [P, C.c_uint32, D]
    L.sr_batch_readback.argtypes = [P, C.c_uint32, F]
    L.sr_batch_ctx.argtypes = [P, C.c_uint32]
    L.sr_batch_ctx.restype = P
    for name in ("sr_batch_create", "sr_batch_upload", "sr_batch_step", "sr_batch_readback"):
        getattr(L, name).restype = C.c_int
    L.sr_last_error.restype = C.c_char_p
    L.sr_last_error.argtypes = [P]
    for name in ("sr_create", "sr_upload", "sr_readback", "sr_upload_opacity", "sr_upload_held", "sr_read_held", "sr_read_box",
                 "sr_step", "sr_read_dt",
                 "sr_read_heat", "sr_gravity_field", "sr_heat_flux", "sr_set_edge_mode", "sr_set_heat_precond",
                 "sr_set_heat_limits", "sr_set_timing", "sr_read_cost", "sr_heat_first_solve", "sr_set_clock",
                 "sr_read_heat_rate", "sr_set_heat_rate", "sr_read_side_flux", "sr_set_side_flux"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def _fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_float))


@dataclass
class DtReport:
    dt: float
    dt_next: float
    steps: int
    sim_time: float
    non_finite: tuple | None


class Step:
    """One world's field update on the GPU (the reference's Step over its State)."""

    def __init__(self, config: Config):
        self.lib = load_library()
        self.config = config
        self._c = config.to_c()
        h = C.c_void_p()
        st = self.lib.sr_create(C.byref(self._c), C.byref(h))
        if st:
            raise SrError(st, self.lib.sr_last_error(None).decode())
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.sr_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int):
        if st:
            raise SrError(st, self.lib.sr_last_error(self._h).decode())

    @property
    def shape(self):
        return (self.config.channels, self.config.height, self.config.width)

    # ---- State::upload / readback (state.rs:251-279)
    def upload(self, planes: np.ndarray):
        p = np.ascontiguousarray(planes, dtype=np.float32)
        if p.shape != self.shape:
            raise SrError(1, f"planes of shape {p.shape}, expected {self.shape}")
        self._check(self.lib.sr_upload(self._h, _fptr(p), self.shape[0]))

    def upload_opacity(self, kappa: np.ndarray):
        k = np.ascontiguousarray(kappa, dtype=np.float32)
        if k.shape != self.shape[1:]:
            raise SrError(1, f"opacity plane of shape {k.shape}, expected {self.shape[1:]}")
        self._check(self.lib.sr_upload_opacity(self._h, _fptr(k)))

    def readback(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.shape, dtype=np.float32)
        self._check(self.lib.sr_readback(self._h, _fptr(out), self.shape[0]))
        return out

    # ---- State::upload_held / read_held (state.rs:198-250), reference mode
    def upload_held(self, mask: np.ndarray):
        m = np.ascontiguousarray(mask, dtype=np.uint32)
        if m.shape != self.shape[1:]:
            raise SrError(1, f"mask of shape {m.shape}, expected {self.shape[1:]}")
        self._check(self.lib.sr_upload_held(self._h, m.ctypes.data_as(C.POINTER(C.c_uint32))))

    def read_box(self) -> sr_box_report:
        """BoxFit::read (boxfit.rs:152-172): the active box's origin and size, its FFT size, the fits so far."""
        r = sr_box_report()
        self._check(self.lib.sr_read_box(self._h, C.byref(r)))
        return r

    def read_held(self) -> np.ndarray:
        m = np.zeros(self.shape[1:], np.uint32)
        self._check(self.lib.sr_read_held(self._h, m.ctypes.data_as(C.POINTER(C.c_uint32))))
        return m

    # ---- Step::run (step/mod.rs:703-718)
    def run(self, steps: int = 1):
        self._check(self.lib.sr_step(self._h, int(steps)))

    # ---- reports
    def read_dt(self) -> DtReport:
        r = sr_dt_report()
        self._check(self.lib.sr_read_dt(self._h, C.byref(r)))
        nf = (int(r.nf_cell), int(r.nf_channel)) if r.non_finite else None
        return DtReport(r.dt, r.dt_next, int(r.steps), r.sim_time, nf)

    def read_heat(self) -> sr_heat_report:
        r = sr_heat_report()
        self._check(self.lib.sr_read_heat(self._h, C.byref(r)))
        return r

    def gravity_field(self):
        h, w = self.shape[1:]
        gx, gy, phi = (np.empty((h, w), np.float32) for _ in range(3))
        self._check(self.lib.sr_gravity_field(self._h, _fptr(gx), _fptr(gy), _fptr(phi)))
        return phi, gx, gy

    # ---- the records a dump carries beyond the cells (dump_state / load_dump, dump.rs:355-410)
    def set_clock(self, steps: int, sim_time: float, dt: float, dt_next: float):
        """Step::restore (step/latch.rs:493-510): the next step's index, the sim time, Δt_n and the next Δt."""
        self._check(self.lib.sr_set_clock(self._h, int(steps), float(sim_time), float(dt), float(dt_next)))

    def read_heat_rate(self, out: np.ndarray | None = None) -> np.ndarray:
        """Step::heat_rate (step/heat.rs:550-565): each cell's P5 rate of the last step, (H, W) f32 (into `out`)."""
        r = np.empty(self.shape[1:], np.float32) if out is None else out
        if r.shape != self.shape[1:] or r.dtype != np.float32 or not r.flags.c_contiguous:
            raise SrError(1, f"rate plane of shape {r.shape} {r.dtype}, expected a contiguous f32 {self.shape[1:]}")
        self._check(self.lib.sr_read_heat_rate(self._h, _fptr(r)))
        return r

    def set_heat_rate(self, rate: np.ndarray | None):
        """Step::set_heat_rate (step/heat.rs:566-582): a dump's rate, or zeros for None."""
        if rate is None:
            self._check(self.lib.sr_set_heat_rate(self._h, None))
            return
        r = np.ascontiguousarray(rate, dtype=np.float32)
        if r.shape != self.shape[1:]:
            raise SrError(1, f"rate plane of shape {r.shape}, expected {self.shape[1:]}")
        self._check(self.lib.sr_set_heat_rate(self._h, _fptr(r)))

    def read_side_flux(self):
        """Step::side_flux (step/heat.rs:584-589): the cell-centred F_x, F_y the next P4 pushes with, (H, W) each."""
        fx, fy = np.empty(self.shape[1:], np.float32), np.empty(self.shape[1:], np.float32)
        self._check(self.lib.sr_read_side_flux(self._h, _fptr(fx), _fptr(fy)))
        return fx, fy

    def set_side_flux(self, fx: np.ndarray, fy: np.ndarray):
        a, b = (np.ascontiguousarray(v, dtype=np.float32) for v in (fx, fy))
        if a.shape != self.shape[1:] or b.shape != self.shape[1:]:
            raise SrError(1, f"flux planes of shape {a.shape} / {b.shape}, expected {self.shape[1:]}")
        self._check(self.lib.sr_set_side_flux(self._h, _fptr(a), _fptr(b)))

    def read_heat_flux(self):
        h, w = self.shape[1:]
        fx, fy = np.empty((h, w + 1), np.float32), np.empty((h + 1, w), np.float32)
        self._check(self.lib.sr_heat_flux(self._h, _fptr(fx), _fptr(fy)))
        return fx, fy

    # ---- switches
    def set_edge_mode(self, edge: str):
        self._check(self.lib.sr_set_edge_mode(self._h, EDGE[edge]))

    def set_heat_precond(self, precond: str):
        self._check(self.lib.sr_set_heat_precond(self._h, PRECOND[precond]))

    def set_heat_limits(self, max_passes: int, max_rounds: int):
        self._check(self.lib.sr_set_heat_limits(self._h, max_passes, max_rounds))

    def set_timing(self, level: int = 1):
        """0 off; 1 (or True) each step's device time, the steps run as they normally do (one captured graph per
        step after the first); 2 the per-pass breakdown, the passes launched one by one."""
        self._check(self.lib.sr_set_timing(self._h, int(level)))

    def read_cost(self) -> sr_cost:
        r = sr_cost()
        self._check(self.lib.sr_read_cost(self._h, C.byref(r)))
        return r

    def heat_first_solve(self, dt: float, precond: str = "mg", want_x: bool = False):
        """The first Newton pass's system solved alone: (device ms, rounds, FP64 rel residual, x or None)."""
        ms, rel = C.c_double(), C.c_double()
        rounds = C.c_uint32()
        h, w = self.shape[1:]
        x = np.empty((h, w), np.float64) if want_x else None
        xp = x.ctypes.data_as(C.POINTER(C.c_double)) if want_x else None
        fb = C.c_uint32()
        self._check(self.lib.sr_heat_first_solve(self._h, dt, PRECOND[precond], C.byref(ms), C.byref(rounds),
                                                 C.byref(rel), xp, C.byref(fb)))
        self.last_fallback = bool(fb.value)
        return ms.value, rounds.value, rel.value, x

    def time_smoother(self, reps: int = 10):
        """(pre ms, post ms): one launch of the level-0 smoothers on the last solved system, L2 flushed before each."""
        pre, post = C.c_double(), C.c_double()
        self._check(self.lib.sr_time_smoother(self._h, reps, C.byref(pre), C.byref(post)))
        return pre.value, post.value

    def attach_learner(self, learner: "Learner | None"):
        """Makes `learner` this world's "learned" preconditioner (None detaches it)."""
        self._check(self.lib.sr_attach_learner(self._h, learner._h if learner is not None else None))
        self._learner = learner  # kept alive while attached


class Batch:
    """Many independent worlds of uneven sizes advanced together on one GPU (sr_batch_*): each world keeps its own
    context and stream, and a pool of host threads, balanced by cell count, steps them concurrently."""

    def __init__(self, configs, threads: int = 0):
        self.lib = load_library()
        self.configs = list(configs)
        arr = (sr_config * len(self.configs))(*[c.to_c() for c in self.configs])
        h = C.c_void_p()
        st = self.lib.sr_batch_create(arr, len(self.configs), threads, C.byref(h))
        if st:
            raise SrError(st, self.lib.sr_last_error(None).decode())
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.sr_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self):
        return len(self.configs)

    def _check(self, st: int):
        if st:
            raise SrError(st, self.lib.sr_last_error(None).decode())

    def upload(self, index: int, planes: np.ndarray, kappa: np.ndarray | None = None):
        cfg = self.configs[index]
        p = np.ascontiguousarray(planes, dtype=np.float32)
        if p.shape != (4, cfg.height, cfg.width):
            raise SrError(1, f"planes of shape {p.shape} for world {index}")
        k = np.ascontiguousarray(kappa, dtype=np.float32) if kappa is not None else None
        self._check(self.lib.sr_batch_upload(self._h, index, _fptr(p), _fptr(k) if k is not None else None))

    def run(self, steps: int = 1) -> float:
        """Every world `steps` steps; returns the device time in ms."""
        ms = C.c_double()
        self._check(self.lib.sr_batch_step(self._h, int(steps), C.byref(ms)))
        return ms.value

    def readback(self, index: int) -> np.ndarray:
        cfg = self.configs[index]
        out = np.empty((4, cfg.height, cfg.width), np.float32)
        self._check(self.lib.sr_batch_readback(self._h, index, _fptr(out)))
        return out

    def read_heat(self, index: int) -> sr_heat_report:
        r = sr_heat_report()
        ctx = self.lib.sr_batch_ctx(self._h, index)
        st = self.lib.sr_read_heat(ctx, C.byref(r))
        if st:
            raise SrError(st, self.lib.sr_last_error(ctx).decode())
        return r


class Learner:
    """The learned preconditioner's network, weights and training samples (sr_learner_*): no reference counterpart."""

    def __init__(self, crop: int = 64, capacity: int = 4096, seed: int = 0):
        self.lib = load_library()
        self.crop = crop
        h = C.c_void_p()
        st = self.lib.sr_learner_create(crop, capacity, seed, C.byref(h))
        if st:
            raise SrError(st, self.lib.sr_last_error(None).decode())
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self.lib.sr_learner_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int):
        if st:
            raise SrError(st, self.lib.sr_last_error(None).decode())

    @property
    def param_count(self) -> int:
        return int(self.lib.sr_learner_param_count())

    def get_params(self) -> np.ndarray:
        theta = np.empty(self.param_count, np.float32)
        self._check(self.lib.sr_learner_get_params(self._h, _fptr(theta)))
        return theta

    def set_params(self, theta: np.ndarray):
        theta = np.ascontiguousarray(theta, np.float32)
        assert theta.shape == (self.param_count,)
        self._check(self.lib.sr_learner_set_params(self._h, _fptr(theta)))

    def collect(self, step: Step, dt: float, crops: int = 16, seed: int = 0) -> int:
        """(residual, error) samples from an MG-PCG solve of `step`'s first implicit system; returns how many."""
        n = C.c_uint32()
        st = self.lib.sr_learner_collect(self._h, step._h, dt, crops, seed, C.byref(n))
        if st:
            raise SrError(st, self.lib.sr_last_error(step._h).decode())
        return int(n.value)

    def train(self, iterations: int, batch: int = 16, lr: float = 1e-3, seed: int = 0) -> float:
        loss = C.c_double()
        self._check(self.lib.sr_learner_train(self._h, iterations, batch, lr, seed, C.byref(loss)))
        return float(loss.value)

    def loss_grad(self, feats: np.ndarray, target: np.ndarray):
        """(loss, gradient, output) of the network on feats (n, 4, crop, crop) against target (n, crop, crop)."""
        feats = np.ascontiguousarray(feats, np.float32)
        target = np.ascontiguousarray(target, np.float32)
        n = feats.shape[0]
        assert feats.shape == (n, 4, self.crop, self.crop) and target.shape == (n, self.crop, self.crop)
        grad = np.empty(self.param_count, np.float32)
        out = np.empty((n, self.crop, self.crop), np.float32)
        loss = C.c_double()
        self._check(self.lib.sr_learner_loss_grad(self._h, _fptr(feats), _fptr(target), n, C.byref(loss),
                                                  _fptr(grad), _fptr(out)))
        return float(loss.value), grad, out
