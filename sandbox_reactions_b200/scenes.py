"""Seeded synthetic scenes for the benchmark configurations (no dataset: every input is generated here).

Seeds follow seed = 1000 + 100 * config + scene. Each generator returns (Config, planes (4, H, W) f32[, κ plane]).
  - sod:        2D Sod tube (config 1): γ = 1.4, ρ 1 | 0.125, p 1 | 0.1 split at x = W/2, leave edges, minmod;
  - disk:       hydro + gravity (config 2): a Gaussian disk (σ = 0.15 W) times lognormal noise (σ_ln = 0.05) over a
                floor of 1e-6, Keplerian rotation from the enclosed mass, p = K Σ^γ, γ = 5/3, 1-cell softened kernel;
  - fld:        implicit FLD alone (config 3): κ lognormal with a 32-cell correlation length spanning six decades
                (0.1-99.9 percentiles), T = 1e3 background with three hot spots at 1e6, Σ = 1, Δt = 50 x the
                explicit diffusion limit;
  - full_step:  the disk of config 2 with the opacity field of config 3 and hot spots at T = 100 over T = 1 (the
                reference's burning temperatures are 56-135), every pass on (the
                hydro+gravity+FLD step of the headline metric);
  - ref_disk:   reference mode (14 channels): a scene-JSON world of a warm solar-mix disk with a hot helium core
                over a thin hydrogen background, laid down with the reference's EOS and species, gravity, hydro and
                heat on (the radiation force from the second step) — the reference-mode P4 kernel's workload.
"""
from __future__ import annotations

import json
import math

import numpy as np

from .abi import Config


def seed_of(config: int, scene: int = 0) -> int:
    return 1000 + 100 * config + scene


def _planes(sigma, u, v, pressure, gamma):
    P = np.zeros((4,) + sigma.shape, dtype=np.float64)
    P[0] = sigma
    P[1] = sigma * u
    P[2] = sigma * v
    P[3] = pressure / (gamma - 1.0) + 0.5 * sigma * (u * u + v * v)
    return P.astype(np.float32)


def sod(n: int = 512) -> tuple[Config, np.ndarray]:
    gamma = 1.4
    cfg = Config(width=n, height=n, edge="leave", limiter="minmod", gamma=gamma, mu=1.0, hydro=True)
    x = np.arange(n)[None, :].repeat(n, 0)
    left = x < n // 2
    sigma = np.where(left, 1.0, 0.125)
    p = np.where(left, 1.0, 0.1)
    z = np.zeros_like(sigma)
    return cfg, _planes(sigma, z, z, p, gamma)


def gaussian_random_field(n: int, corr: float, rng: np.random.Generator, m: int | None = None) -> np.ndarray:
    """Unit-variance Gaussian random field: white noise filtered by exp(-k² corr² / 2) in Fourier space."""
    m = n if m is None else m
    white = rng.standard_normal((m, n))
    ky = np.fft.fftfreq(m)[:, None] * 2 * np.pi
    kx = np.fft.fftfreq(n)[None, :] * 2 * np.pi
    filt = np.exp(-0.5 * (kx * kx + ky * ky) * corr * corr)
    g = np.fft.ifft2(np.fft.fft2(white) * filt).real
    g -= g.mean()
    return g / g.std()


def opacity_field(n: int, rng: np.random.Generator, kappa0: float = 1.0, corr: float = 32.0,
                  decades: float = 6.0) -> np.ndarray:
    """κ = κ0 exp(s G), s set so that the 0.1-99.9 percentile range of κ spans `decades` decades."""
    g = gaussian_random_field(n, corr, rng)
    lo, hi = np.percentile(g, [0.1, 99.9])
    s = decades * math.log(10.0) / (hi - lo)
    return (kappa0 * np.exp(s * g)).astype(np.float32)


def hot_spots(n: int, rng: np.random.Generator, t_bg: float, t_spot: float, count: int = 3,
              radius: float | None = None) -> np.ndarray:
    radius = n / 32.0 if radius is None else radius
    j, i = np.mgrid[0:n, 0:n].astype(np.float64)
    T = np.full((n, n), t_bg)
    for _ in range(count):
        cx, cy = rng.uniform(0.2 * n, 0.8 * n, 2)
        T += (t_spot - t_bg) * np.exp(-((i - cx) ** 2 + (j - cy) ** 2) / (2.0 * radius * radius))
    return T


def face_diffusivity(cfg: Config, T: np.ndarray, sigma: np.ndarray, kappa: np.ndarray):
    """D_f of the frozen flux law at interior faces (reference heat.rs:263-279), for sizing Δt."""
    er = cfg.a_r * T ** 4
    ks = kappa * sigma

    def face(a, b, ka, kb):
        fer = 0.5 * (a + b)
        k = 0.5 * (ka + kb)
        r = np.abs(b - a) / (k * fer)
        lam = (2.0 + r) / (6.0 + 3.0 * r + r * r) if cfg.flux_limiter else 1.0 / 3.0
        return cfg.c_sb * lam / k

    dx = face(er[:, :-1], er[:, 1:], ks[:, :-1], ks[:, 1:])
    dy = face(er[:-1, :], er[1:, :], ks[:-1, :], ks[1:, :])
    return dx, dy


def explicit_limit(cfg: Config, T, sigma, kappa) -> float:
    """min over cells of (C_i / (4 a_r T_i³)) / Σ_f D_f: the explicit diffusion step limit."""
    dx, dy = face_diffusivity(cfg, T, sigma, kappa)
    dsum = np.zeros_like(T)
    dsum[:, :-1] += dx
    dsum[:, 1:] += dx
    dsum[:-1, :] += dy
    dsum[1:, :] += dy
    C = sigma / (cfg.mu * (cfg.gamma - 1.0))
    return float(np.min(C / (4.0 * cfg.a_r * T ** 3) / dsum))


def fld(n: int = 2048, scene: int = 0, dt_factor: float = 50.0):
    """Config 3: returns (cfg, planes, kappa)."""
    rng = np.random.default_rng(seed_of(3, scene))
    gamma, mu = 5.0 / 3.0, 1.0
    kappa = opacity_field(n, rng)
    T = hot_spots(n, rng, 1e3, 1e6)
    sigma = np.ones((n, n))
    cfg = Config(width=n, height=n, hydro=False, gravity=False, heat=True, opacity_plane=True, gamma=gamma, mu=mu,
                 edge="bounce", mg_pre=2, mg_post=2)  # the configuration's preconditioner: V(2,2)
    dt = dt_factor * explicit_limit(cfg, T, sigma, kappa.astype(np.float64))
    cfg = cfg.replace(dt_fixed=dt)
    z = np.zeros((n, n))
    p = sigma * T / mu
    return cfg, _planes(sigma, z, z, p, gamma), kappa


def disk(n: int = 1024, scene: int = 0, sigma0: float = 1.0, K: float = 1e-3):
    """Config 2: returns (cfg, planes)."""
    rng = np.random.default_rng(seed_of(2, scene))
    gamma = 5.0 / 3.0
    sigma, u, v = _disk_fields(n, rng, sigma0)
    p = K * sigma ** gamma
    cfg = Config(width=n, height=n, edge="leave", limiter="mc", gamma=gamma, mu=1.0, gravity=True, hydro=True,
                 kernel="softened", softening=1.0, t_floor=1e-6)
    return cfg, _planes(sigma, u, v, p, gamma)


def _disk_fields(n, rng, sigma0):
    j, i = np.mgrid[0:n, 0:n].astype(np.float64)
    c = (n - 1) / 2.0
    dx, dy = i - c, j - c
    r = np.hypot(dx, dy)
    s = 0.15 * n
    noise = np.exp(0.05 * rng.standard_normal((n, n)) - 0.05 ** 2 / 2)
    sigma = np.maximum(1e-6, sigma0 * np.exp(-r * r / (2 * s * s)) * noise)
    order = np.argsort(r, axis=None)
    enclosed = np.empty(n * n)
    enclosed[order] = np.cumsum(sigma.ravel()[order])
    enclosed = enclosed.reshape(n, n)
    vphi = np.sqrt(enclosed / np.maximum(r, 0.5))
    rr = np.maximum(r, 1e-12)
    u = -vphi * dy / rr
    v = vphi * dx / rr
    return sigma, u, v


def full_step(n: int = 2048, scene: int = 0, sigma0: float = 1.0, t_bg: float = 1.0, t_spot: float = 100.0):
    """Hydro + gravity + FLD on one world: config 2's disk, config 3's opacity field, hot spots in the gas."""
    rng = np.random.default_rng(seed_of(5, scene))
    gamma, mu = 5.0 / 3.0, 1.0
    sigma, u, v = _disk_fields(n, rng, sigma0)
    kappa = opacity_field(n, rng)
    T = hot_spots(n, rng, t_bg, t_spot, radius=n / 64.0)
    p = sigma * T / mu
    cfg = Config(width=n, height=n, edge="leave", limiter="mc", gamma=gamma, mu=mu, gravity=True, hydro=True,
                 heat=True, opacity_plane=True, kernel="softened", softening=1.0, t_floor=0.05)
    return cfg, _planes(sigma, u, v, p, gamma), kappa


def batch_mix(count: int = 64, sizes=(256, 512, 1024, 2048), scene: int = 0):
    """Config 5: `count` worlds of a seeded mix of sizes, each config 2's disk with config 3's opacity field and hot
    spots (scenes.full_step) with its own disk mass and opacity seed. Returns the worlds' specs (n, scene, sigma0);
    `world(spec)` builds one as (cfg, planes, kappa)."""
    rng = np.random.default_rng(seed_of(5, 50 + scene))
    specs = []
    for k in range(count):
        n = int(rng.choice(sizes))
        mass = float(rng.uniform(0.5, 2.0))
        specs.append((n, 100 + 1000 * scene + k, mass))
    return specs


def world(spec):
    n, scene, mass = spec
    return full_step(n, scene=scene, sigma0=mass)


def ref_disk(n: int = 1024):
    """Reference mode: returns (cfg, planes (14, H, W) f32) of a scene laid down by scene.py at n x n."""
    from .scene import Scene

    a, core = 0.3125 * n, 0.0625 * n
    text = json.dumps({
        "version": 1, "world": {"width": n, "height": n, "edge": "leave"}, "slowdown": False,
        "switches": {"gravity": True, "hydro": True, "heat": True, "reactions": False, "neutrinos": False,
                     "sinks": False},
        "objects": [
            {"kind": "rect", "x0": 0, "y0": 0, "w": n, "h": n, "sigma": 2e-3, "t": 1.0, "composition": {"H": 1.0},
             "v": [0, 0]},
            {"kind": "disk", "x": n / 2, "y": n / 2, "a": a, "sigma_c": 1.0, "t": 40.0,
             "composition": {"H": 0.7346, "He": 0.2485, "C": 0.0092, "O": 0.0077}, "v": [0.05, 0.02]},
            {"kind": "disk", "x": 0.41 * n, "y": 0.55 * n, "a": core, "sigma_c": 2.0, "t": 400.0,
             "composition": {"He": 1.0}, "v": [0, 0]}]})
    sc = Scene.parse(text)
    P, _ = sc.planes()
    return sc.ref_config(strict=False).replace(heat=True), P
