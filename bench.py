"""Benchmark of the full per-step field update (hydro + FFT gravity + implicit FLD) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--size S] [--impl ours|reference]

One step = P1 → P2 → P4 (with its half-step gravity solve) → P5 (Newton + FP64-refined MG-PCG to 1e-8) → P8 → P9 on a
seeded synthetic world of S x S cells (default 2048): a Gaussian disk with lognormal noise in Keplerian rotation, a
lognormal opacity field with a 32-cell correlation length over six decades, hot spots in the gas (scenes.full_step).
Under torchrun every rank advances its own world (scene seed = rank): the worlds are independent, no collective on the
data path, weak scaling. The line also carries: the FLD time-to-1e-8 of the 2048² implicit-diffusion configuration
(scenes.fld) with plain MG-PCG (its V(2,2), and V(4,4) as the full step runs it), Jacobi-PCG and the learned
preconditioner; the other single-GPU configurations (Sod 512², the 1024² disk) with their parity against the oracle;
the full-size parity of one step against the f64 twin; and config 5, 64 worlds of a seeded 256²…2048² mix advanced
as one captured graph per batch step against the same worlds one at a time (`batched`).

`--impl reference` times the reference's own CPU algorithm (the f64 twin restated in C, oracle/) on the same 2048²
world with every host thread, for as many of the K steps as fit a bounded time (at least one), and beside it one
thread on a 512² sample of the scene.

`--case fld|full|learned|sod|grav|ref --size S` runs one small self-contained workload per hot kernel family instead (what
the committed ncu summaries were captured on) and prints one line with its device time: fld, the implicit-diffusion
world's first system solved to 1e-8 `--solves` times (smoothers, coarse tail, SpMV, PCG vectors; `--sweeps 4` for
V(4,4)); full, `--steps` full steps of the benchmark world; learned, one flexible-CG round with an untrained learned
preconditioner (the convolution kernels' cost does not depend on the weights); sod, `--steps` hydro-only steps of a
Sod tube (the stencil kernel); grav, `--solves` gravity-only steps of a disk (the FFT kernels); ref, `--steps`
reference-mode steps (14 channels, scenes.ref_disk: the reference-mode P4 kernel).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s hydro+grav+FLD @2048²; FLD time-to-1e-8: learned vs MG-PCG"
UNIT = "Mcell-steps/s"
BREAKDOWN_STEPS = 2  # steps of the per-pass timing leg (passes launched one by one) after the timed steps
# algorithmic bytes per cell of the fused hydro update kernel with gravity: state in 16 + out 16, P2's g 8,
# the half-step source 4, φ_mid 4 and g_mid 8
HYDRO_UPDATE_BYTES_PER_CELL = 56
# the multigrid's level-0 smoothers, the step's dominant kernels (per cell of level 0): the pre-smoother reads
# b, c, dx, dy (16) and the mask (1) and writes x (4) and the coarse right-hand side (4 per 2x2 aggregate: 1);
# the post-smoother reads x, b, c, dx, dy (20), the mask (1) and the coarse correction (1) and writes x2 (4)
SMOOTH_PRE_BYTES_PER_CELL = 22
SMOOTH_POST_BYTES_PER_CELL = 26


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.samples.append([v.strip() for v in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        sm = [float(s[1]) for s in self.samples if len(s) > 2 and s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if len(s) > 2 and s[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            for k, name in enumerate(names):
                if len(s) > 5 + k and s[5 + k].strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def committed_traffic(kernel: str, cells: int):
    """DRAM bytes per launch of `kernel` scaled to `cells`, from the committed ncu summary (profiles/traffic.json)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    k = d.get(kernel)
    if not k:
        return None
    return k["dram_bytes_per_launch"] * cells / k["cells"]


def cpu_twin_run(size: int, steps: int, threads: int, warmup: int = 0, budget_s: float = 20.0, world=None):
    """The oracle's f64 twin (the reference's Twin, restated) on the `size`² world of the benchmark's scene: Twin::new
    (P2 and Δt_0) and `warmup` steps untimed, then up to `steps` timed steps, stopping once `budget_s` seconds are spent
    (at least one). Returns (Mcell-steps/s, seconds, steps timed, twin)."""
    import numpy as np

    import oracle as O
    from sandbox_reactions_b200 import scenes

    O.set_threads(threads)
    cfg, P, kappa = world if world is not None else scenes.full_step(size)
    twin = O.Twin(cfg, P.astype(np.float64), kappa.astype(np.float64))
    twin.step(warmup)
    t0 = time.perf_counter()
    done = 0
    for _ in range(max(1, steps)):
        twin.step(1)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    return size * size * done / dt / 1e6, dt, done, twin


def workload_config(n: int, world: int) -> dict:
    return {"workload": f"full step hydro+gravity+FLD, {n}x{n}, Gaussian disk + lognormal opacity "
                        f"(32-cell correlation, 6 decades) + hot spots; FFT {2 * n}x{2 * n}",
            "cells": n * n, "parallelism": f"replicas x{world}",
            "l2": "working set larger than L2 (state, fields and solver planes > 1 GB)"}


def run_reference(args, rank, world):
    """The reference arm: the twin on the benchmark's own world (same scene, size and seed as this arm's rank 0),
    every host thread; W is capped at one untimed step (the CPU has nothing to warm beyond its caches) and the timed
    steps stop at K or once --ref-budget seconds are spent. One thread on a 512² sample rides along."""
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    n = args.size
    warm = min(args.warmup, 1)
    value, secs, done, _ = cpu_twin_run(n, args.steps, threads, warmup=warm, budget_s=args.ref_budget)
    sample = (f"{done} twin steps of the {n}x{n} benchmark world itself (hydro + gravity + FLD, f64, the reference's "
              f"Jacobi-PCG to 1e-12), {secs:.1f} s on {threads} threads after Twin::new and {warm} untimed step(s)")
    one_n = min(512, n)
    v1, s1, d1, _ = cpu_twin_run(one_n, 1, 1, budget_s=0.0)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": done,
            "warmup": args.warmup, "warmup_steps_run": warm, "steps_requested": args.steps,
            "ms_per_step": 1e3 * secs / max(done, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(n, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "one_thread": {"value": v1, "unit": UNIT, "cores": 1, "kind": "port",
                           "sample": f"{d1} twin step of a {one_n}x{one_n} world of the same scene, {s1:.1f} s"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def rel_l1(a, b) -> float:
    import numpy as np

    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))


def full_step_parity(step, twin, P, kappa) -> dict:
    """One GPU step of the benchmark world from the same f32 start as the twin's step: rel L1 per field (the bar is
    1e-5) and the implicit solve's FP64 residual (the bar is 1e-8)."""
    step.upload(P)
    step.upload_opacity(kappa)
    step.run(1)
    gpu = step.readback()
    heat = step.read_heat()
    ref = twin.state()
    errs = {name: rel_l1(gpu[k], ref[k]) for k, name in enumerate(("sigma", "sigma_u", "sigma_v", "E"))}
    return {"what": "one step from the same f32 start vs the f64 twin (Newton 1e-12, Jacobi-PCG 1e-12)",
            "rel_l1": errs, "max_rel_l1": max(errs.values()), "bar": 1e-5, "heat_rel_residual": heat.rel_residual,
            "heat_passes": heat.passes, "ok": max(errs.values()) <= 1e-5 and heat.rel_residual <= 1e-8}


def run_case(args, local):
    """One profiling workload (see the module docstring); prints one line with its device time."""
    import torch

    from sandbox_reactions_b200 import build as lib_build
    from sandbox_reactions_b200 import scenes
    from sandbox_reactions_b200.engine import Learner, Step

    torch.cuda.set_device(local)
    lib_build.build()
    n = args.size
    if args.case == "fld":
        cfg, P, kappa = scenes.fld(n)
        if args.sweeps:
            cfg = cfg.replace(mg_pre=args.sweeps, mg_post=args.sweeps)
        with Step(cfg) as s:
            s.upload(P)
            s.upload_opacity(kappa)
            for _ in range(args.solves):
                ms, rounds, rel, _ = s.heat_first_solve(cfg.dt_fixed, args.precond)
        print(f"fld {n}: {args.precond} first solve V({cfg.mg_pre},{cfg.mg_post}) {ms:.3f} ms, {rounds} rounds, "
              f"rel residual {rel:.2e}")
    elif args.case == "full":
        cfg, P, kappa = scenes.full_step(n)
        with Step(cfg) as s:
            s.upload(P)
            s.upload_opacity(kappa)
            s.set_timing(True)
            s.run(args.steps)
            cost = s.read_cost()
        print(f"full {n}: {args.steps} steps, {cost.total_ms / args.steps:.3f} ms per step")
    elif args.case == "learned":
        cfg, P, kappa = scenes.fld(n)
        with Learner(crop=64, capacity=1, seed=1) as L, Step(cfg) as s:
            s.upload(P)
            s.upload_opacity(kappa)
            s.attach_learner(L)
            s.set_heat_limits(128, 1)
            ms, _, _, _ = s.heat_first_solve(cfg.dt_fixed, "learned")
            s.attach_learner(None)
        print(f"learned {n}: one round {ms:.3f} ms")
    elif args.case == "ref":
        cfg, P = scenes.ref_disk(n)
        with Step(cfg) as s:
            s.upload(P)
            s.set_timing(2)
            s.run(args.steps)
            cost = s.read_cost()
        print(f"ref {n}: {args.steps} reference-mode steps, {cost.total_ms / args.steps:.3f} ms per step, "
              f"P4 {cost.hydro_ms / args.steps:.3f} ms per step")
    elif args.case == "sod":
        cfg, P = scenes.sod(n)
        with Step(cfg) as s:
            s.upload(P)
            s.set_timing(True)
            s.run(args.steps)
            cost = s.read_cost()
        print(f"sod {n}: {args.steps} steps, {cost.total_ms / args.steps:.3f} ms per step")
    else:
        cfg, P = scenes.disk(n)
        with Step(cfg.replace(hydro=False, heat=False)) as s:
            s.upload(P)
            s.set_timing(2)
            s.run(args.solves)  # each step: P2's solve, P8, P9
            cost = s.read_cost()
        print(f"grav {n}: {args.solves} solves, {cost.gravity_ms / args.solves:.3f} ms per solve")
    return 0


def train_learner(train_size: int = 256, worlds: int = 32, iterations: int = 1500):
    """The learned preconditioner trained as its tests train it: MG-PCG samples of `worlds` seeded implicit-diffusion
    worlds of train_size² (every round's whole world), Adam on the GPU. Returns (learner, samples, seconds)."""
    from sandbox_reactions_b200 import scenes
    from sandbox_reactions_b200.engine import Learner, Step

    t0 = time.perf_counter()
    L = Learner(crop=train_size, capacity=20 * worlds, seed=1)
    samples = 0
    for k in range(worlds):
        cfg, P, kappa = scenes.fld(train_size, scene=1000 + k)
        with Step(cfg) as s:
            s.upload(P)
            s.upload_opacity(kappa)
            samples += L.collect(s, cfg.dt_fixed, crops=1, seed=k)
    loss = L.train(iterations, batch=8, lr=3e-4, seed=0)
    return L, samples, loss, time.perf_counter() - t0


def fld_time_to_tol(size: int):
    """The implicit-diffusion configuration's first system (a held-out seed) solved to 1e-8 with MG-PCG, Jacobi-PCG
    and the learned preconditioner in flexible CG (device ms of the solve; training is reported apart)."""
    from sandbox_reactions_b200 import scenes
    from sandbox_reactions_b200.engine import SrError, Step

    cfg, P, kappa = scenes.fld(size)
    out = {"size": size, "dt": cfg.dt_fixed}
    learner = None
    try:
        learner, samples, loss, secs = train_learner()
        out["learned_training"] = {"worlds": "32 x 256x256 (seeds 1000..1031)", "samples": samples,
                                   "iterations": 1500, "batch": 8, "final_loss": loss, "seconds": secs}
    except SrError as e:
        out["learned_training"] = {"unavailable": e.message}
    with Step(cfg) as s:
        s.upload(P)
        s.upload_opacity(kappa)
        if learner is not None:
            s.attach_learner(learner)
        x_mg = None
        for pc in ("mg", "jacobi", "learned"):
            try:
                s.heat_first_solve(cfg.dt_fixed, pc)  # warm-up
                ms, rounds, rel, x = s.heat_first_solve(cfg.dt_fixed, pc, want_x=(pc == "mg"))
                if pc == "mg":
                    x_mg = x
                out[pc] = {"ms": ms, "rounds": rounds, "rel_residual": rel}
                if pc == "learned":
                    out[pc]["fallback"] = s.last_fallback
            except SrError as e:
                out[pc] = {"unavailable": e.message}
        s.attach_learner(None)
    # the same system with the full step's V(4,4) (the configuration names V(2,2))
    with Step(cfg.replace(mg_pre=4, mg_post=4)) as s:
        s.upload(P)
        s.upload_opacity(kappa)
        s.heat_first_solve(cfg.dt_fixed, "mg")
        ms, rounds, rel, _ = s.heat_first_solve(cfg.dt_fixed, "mg")
        out["mg_v44"] = {"ms": ms, "rounds": rounds, "rel_residual": rel}
    if learner is not None:
        learner.close()
    if "ms" in out.get("learned", {}) and "ms" in out.get("mg", {}):
        out["learned_speedup_vs_mg"] = out["mg"]["ms"] / out["learned"]["ms"]
        # why it does not pay: a learned round is two V-cycles (the second removes the BF16 output's rounding noise)
        # plus the network; its break-even network cost from the measured MG round
        mg_round = out["mg"]["ms"] / max(1, out["mg"]["rounds"])
        lr = max(1, out["learned"]["rounds"])
        out["learned_break_even"] = {
            "mg_round_ms": mg_round,
            "learned_round_ms": out["learned"]["ms"] / lr,
            "network_ms_per_round": out["learned"]["ms"] / lr - 2.0 * mg_round,
            "learned_ms_with_a_free_network": lr * 2.0 * mg_round,
            "break_even_network_ms": (out["mg"]["ms"] - lr * 2.0 * mg_round) / lr,
            "rounds_a_free_network_must_reach": out["mg"]["ms"] / (2.0 * mg_round),
        }
    out.update(fld_system_checks(cfg, P, kappa, x_mg))
    return out


def system_stiffness(diag, kx, ky, gas) -> dict:
    """How far the implicit system is from its diagonal: per cell, the couplings' sum Σ_f D_f Δt over the mass term
    C/(4 a_r T³) (= the cell's Δt over its explicit diffusion limit)."""
    import numpy as np

    off = np.zeros_like(diag)
    off[:, :] += kx[:, :-1] + kx[:, 1:]
    off[:, :] += ky[:-1, :] + ky[1:, :]
    mass = diag - off
    r = (off / np.maximum(mass, 1e-300))[gas.astype(bool)]
    return {"max": float(r.max()), "median": float(np.median(r)), "p99": float(np.percentile(r, 99))}


def fld_system_checks(cfg, P, kappa, x_mg) -> dict:
    """The implicit-diffusion world's first system, built by the oracle: its stiffness, and the GPU's MG-PCG solution
    against the twin's f64 Jacobi-PCG solve to 1e-12 (max norm over gas cells, relative; the bar is 1e-6)."""
    import numpy as np

    import oracle as O

    O.set_threads(os.cpu_count() or 1)
    diag, rhs, kx, ky, gas = O.heat_system(cfg, P.astype(np.float64), cfg.dt_fixed, kappa.astype(np.float64))
    out = {"stiffness": system_stiffness(diag, kx, ky, gas)}
    if x_mg is not None:
        x_ref, rounds = O.heat_pcg(diag, rhs, kx, ky, gas, rel=1e-12, max_rounds=200000)
        g = gas.astype(bool)
        out["parity"] = {"solution_max_rel": float(np.abs(x_mg - x_ref)[g].max() / np.abs(x_ref[g]).max()),
                         "bar": 1e-6, "twin_rounds_to_1e-12": rounds}
    return out


def config_runs(peak_gbs: float):
    """The other single-GPU configurations as side measurements (device time of the steps, library events): C1, the
    Sod tube at 512² with minmod (hydro only, 200 steps), and C2, the disk at 1024² with its FFT gravity (100 steps);
    each with its hydro update kernel's HBM roofline (32 B/cell without gravity, 56 B/cell with) and its parity: one
    GPU step against the oracle's step from the same f32 start (bar 1e-5 per field); for C1 also the 200 steps against
    the twin's (the reference's G-REF band, 1e-3), for C2 the start state's potential against an f64 direct sum on a
    128² subsample of target cells."""
    import numpy as np

    import oracle as O
    from sandbox_reactions_b200 import scenes
    from sandbox_reactions_b200.engine import Step

    O.set_threads(os.cpu_count() or 1)
    out = {}
    for name, (cfg, P), steps, bpc in (("C1_sod_512_minmod", scenes.sod(512), 200, 32),
                                       ("C2_disk_hydro_grav_1024", scenes.disk(1024), 100, 56)):
        with Step(cfg) as s:
            s.upload(P)
            phi = s.gravity_field()[0] if cfg.gravity else None
            s.run(1)
            one = s.readback()
            dt1 = s.read_dt().dt
            s.run(2)
            s.set_timing(1)
            s.run(steps)
            c = s.read_cost()
            s.set_timing(2)  # a short per-pass leg for the hydro update kernel's own time
            s.run(4)
            cu = s.read_cost()
            s.set_timing(0)
            if not cfg.gravity:
                s.upload(P)
                s.run(steps)
                final = s.readback()
                sim_time = s.read_dt().sim_time
        n = cfg.width * cfg.height
        upd = cu.hydro_update_ms / max(1, cu.hydro_update_launches)
        gbs = bpc * n / (upd / 1e3) / 1e9
        P64 = P.astype(np.float64)
        g = O.grav_field(cfg, P64[0])[1:] if cfg.gravity else None
        ref = O.floors(cfg, O.hydro_step(cfg, P64, dt1, g)[0])
        par = {"one_step_rel_l1": max(rel_l1(one[k], ref[k]) for k in range(4) if np.abs(ref[k]).sum() > 0),
               "bar": 1e-5}
        if not cfg.gravity:
            twin = O.Twin(cfg, P64)
            twin.step(steps)
            tref = twin.state()
            par[f"{steps}_steps_rel_l1"] = {"sigma": rel_l1(final[0], tref[0]), "E": rel_l1(final[3], tref[3]),
                                           "clock": abs(sim_time - twin.clock()["sim_time"]) / twin.clock()["sim_time"],
                                           "bar": 1e-3}
        else:
            src = np.where(P[0] >= np.float32(cfg.sigma_vac), P[0], 0.0).astype(np.float64)
            ty, tx = np.mgrid[4:cfg.height:8, 4:cfg.width:8]
            direct = O.direct_potential(cfg, src, tx.ravel(), ty.ravel())
            got = phi[ty.ravel(), tx.ravel()]
            par["potential_vs_direct_sum"] = {"rel_l1": rel_l1(got, direct),
                                              "max_rel": float((np.abs(got - direct) / np.abs(direct)).max()),
                                              "targets": int(direct.size)}
        out[name] = {"value": n * steps / (c.total_ms / 1e3) / 1e6, "unit": "Mcell-steps/s", "steps": steps,
                     "ms_per_step": c.total_ms / steps,
                     "hydro_update": {"ms_per_launch": upd, "algorithmic_bytes_per_cell": bpc, "achieved_gbs": gbs,
                                      "frac_of_measured_hbm": gbs / peak_gbs},
                     "parity": par}
    return out


def box_measure(n: int = 2048, steps: int = 16, warmup: int = 17):
    """The active box (boxfit.rs) on a vacuum-heavy world: the benchmark's 2048² world (hydro + gravity + FLD) with
    the gas past r = 480 cells replaced by the floor state (a box of 976², whose FFT pads to 2048² where the world's
    pads to 4096²), stepped whole and in its box (warm-up past the first refit, then `steps` steps timed on the
    device); the two final states compared (rel L1 per field) and each rate given in cells of the whole world per
    second."""
    import numpy as np

    from sandbox_reactions_b200 import scenes
    from sandbox_reactions_b200.engine import Step

    cfg, P, kappa = scenes.full_step(n)
    yy, xx = np.mgrid[0:n, 0:n]
    radius = 480.0 * n / 2048.0
    out = np.hypot(xx - (n - 1) / 2.0, yy - (n - 1) / 2.0) > radius
    P = P.copy()
    P[0][out] = cfg.sigma_floor
    P[1][out] = 0.0
    P[2][out] = 0.0
    P[3][out] = cfg.sigma_floor * cfg.t_floor / (cfg.mu * (cfg.gamma - 1.0))
    res, states = {}, {}
    for box in (False, True):
        with Step(cfg.replace(active_box=box)) as s:
            s.upload(P)
            s.upload_opacity(kappa)
            s.run(warmup)
            s.set_timing(1)
            s.run(steps)
            ms = s.read_cost().total_ms
            s.set_timing(0)
            b = s.read_box()
            states[box] = s.readback()
        res["box" if box else "whole"] = {"ms_per_step": ms / steps, "value": n * n * steps / (ms / 1e3) / 1e6,
                                          "unit": UNIT, "box": [b.x0, b.y0, b.w, b.h], "fft": [b.fft_w, b.fft_h]}
    res["speedup"] = res["whole"]["ms_per_step"] / res["box"]["ms_per_step"]
    res["box_vs_whole_rel_l1"] = max(rel_l1(states[True][k], states[False][k]) for k in range(4))
    res["what"] = (f"{n}x{n} hydro+grav+FLD world, vacuum past r = {radius:.0f}: whole world vs the active box, "
                   f"{warmup} warm-up steps then {steps} timed")
    return res


def batch_measure(count: int, steps: int, warmup: int, rank: int = 0, world: int = 1, dist=None):
    """Config 5 on this rank: its share (by cell count) of `count` worlds of a seeded 256²…2048² mix advanced as one
    batch — after the first step each batch step is one captured CUDA graph over all of them — against the same worlds
    stepped one at a time; device ms of the timed steps (max over ranks) and the cells. The warm-up covers the first,
    host-driven step and the capture of the two state-buffer parities' graphs."""
    from concurrent.futures import ThreadPoolExecutor

    from sandbox_reactions_b200 import distributed, scenes
    from sandbox_reactions_b200.engine import Batch, Step

    specs = scenes.batch_mix(count, sizes=(256, 512, 1024, 2048))
    cells = [n * n for n, _, _ in specs]
    mine = distributed.partition(cells, world)[rank]
    with ThreadPoolExecutor(8) as ex:  # numpy's FFTs and sorts release the GIL
        worlds = list(ex.map(scenes.world, [specs[i] for i in mine]))
    batch = Batch([w[0] for w in worlds])
    for i, (cfg, P, kappa) in enumerate(worlds):
        batch.upload(i, P, kappa)
    for _ in range(warmup):
        batch.run(1)
    if dist:
        dist.barrier()
    ms = batch.run(steps)
    batch.close()
    alone = 0.0
    for cfg, P, kappa in worlds:
        with Step(cfg) as s:
            s.upload(P)
            s.upload_opacity(kappa)
            for _ in range(warmup):
                s.run(1)
            s.set_timing(True)
            s.run(steps)
            alone += s.read_cost().total_ms
    if dist:
        ms = distributed.max_over_ranks(dist, ms, device="cuda")
        alone = distributed.max_over_ranks(dist, alone, device="cuda")
    total = sum(cells)
    return {"value": total * steps / (ms / 1e3) / 1e6, "unit": UNIT, "ms_per_step": ms / steps, "steps": steps,
            "warmup": warmup, "worlds": count, "cells": total,
            "sizes": {str(n): sum(1 for c in cells if c == n * n) for n in (256, 512, 1024, 2048)},
            "one_at_a_time": {"value": total * steps / (alone / 1e3) / 1e6, "unit": UNIT,
                              "ms_per_step": alone / steps},
            "speedup_vs_one_at_a_time": alone / ms}


def run_batch(args, rank, world, local):
    """Config 5 as the benchmark: the batch's aggregate Mcell-steps/s, worlds split over the ranks by cell count."""
    import torch

    from sandbox_reactions_b200 import build as lib_build
    from sandbox_reactions_b200 import distributed

    torch.cuda.set_device(local)
    dist = distributed.init("nccl")
    if rank == 0:
        lib_build.build()
    if dist:
        dist.barrier()
    out = batch_measure(args.batch, args.steps, max(args.warmup, 3), rank, world, dist)
    if rank == 0:
        line = {"metric": "Mcell-steps/s batched hydro+grav+FLD (config 5)", "value": out["value"], "unit": UNIT,
                "n_gpus": world, "steps": args.steps, "warmup": out["warmup"], "ms_per_step": out["ms_per_step"],
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic",
                "config": {"workload": f"{args.batch} worlds, seeded mix of 256/512/1024/2048 square, full step "
                                       f"hydro+gravity+FLD (MG-PCG), one captured graph per batch step",
                           "cells": out["cells"], "sizes": out["sizes"],
                           "parallelism": f"worlds split over {world} GPU(s) by cell count"},
                "one_at_a_time": out["one_at_a_time"]}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--size", type=int, default=2048)
    ap.add_argument("--ref-budget", type=float, default=120.0,
                    help="seconds of timed twin steps the reference arm may spend (at least one step)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--case", choices=["fld", "full", "learned", "sod", "grav", "ref"],
                    help="run one profiling workload instead of the benchmark")
    ap.add_argument("--solves", type=int, default=3)
    ap.add_argument("--precond", default="mg")
    ap.add_argument("--sweeps", type=int, default=0,
                    help="--case fld: red-black sweeps a side of the V-cycle (0: the configuration's V(2,2))")
    ap.add_argument("--no-fld", action="store_true", help="skip the FLD time-to-1e-8 measurement")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-world batch (config 5) side measurement")
    ap.add_argument("--no-box", action="store_true", help="skip the active box side measurement")
    ap.add_argument("--batch", type=int, default=0,
                    help="run config 5 instead: this many worlds of a seeded 256..2048 mix, batched vs one at a time")
    args = ap.parse_args()

    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.case:
        return run_case(args, local)
    if args.batch:
        return run_batch(args, rank, world, local)

    import numpy as np
    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from sandbox_reactions_b200 import build as lib_build

    if rank == 0:
        lib_build.build()
    if dist:
        dist.barrier()
    from sandbox_reactions_b200 import scenes
    from sandbox_reactions_b200.engine import Step, load_library

    load_library()
    n = args.size
    cfg, P, kappa = scenes.full_step(n, scene=rank)
    step = Step(cfg)
    step.upload(P)
    step.upload_opacity(kappa)
    for _ in range(args.warmup):
        step.run(1)

    # ---- device-resident throughput: K steps timed on the device (events on the library's stream)
    sampler = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    step.set_timing(1)  # each step's device time, the steps run as they always do (one captured graph per step)
    with sampler:
        step.run(args.steps)
    torch.cuda.synchronize()
    cost = step.read_cost()
    # a short second leg with the passes launched one by one: the per-pass breakdown and the hydro update's own time
    step.set_timing(2)
    step.run(BREAKDOWN_STEPS)
    parts = step.read_cost()
    step.set_timing(0)
    total_ms = cost.total_ms
    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    value = world * n * n * args.steps / (max_ms / 1e3) / 1e6
    heat = step.read_heat()
    # the dominant kernels, timed live on the library's stream with CUDA events (L2 flushed before each launch)
    pre_ms, post_ms = step.time_smoother(10)

    # ---- end to end through the C ABI: per step the run's resumable state from pinned host memory in — the cells, κ
    # and P5's rate (the next step's first iterate, which a dump carries) — and the cells and the rate out; beside it
    # the cells and κ alone, each step then starting its implicit solve cold (sr_upload zeroes the rate)
    pin_in = torch.empty((4, n, n), dtype=torch.float32, pin_memory=True)
    pin_k = torch.empty((n, n), dtype=torch.float32, pin_memory=True)
    pin_out = torch.empty((4, n, n), dtype=torch.float32, pin_memory=True)
    pin_rate = torch.empty((n, n), dtype=torch.float32, pin_memory=True)
    step.readback(pin_in.numpy())  # the state the timed steps left: the end-to-end steps continue from it
    step.read_heat_rate(pin_rate.numpy())
    pin_k.numpy()[...] = kappa
    e2e_steps = max(1, min(args.steps, 5))
    bufs = [pin_in, pin_out]

    def e2e_leg(with_rate: bool) -> float:
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(e2e_steps):
            src, dst = bufs
            bufs.reverse()  # this step's result is the next step's input
            step.upload(src.numpy())
            step.upload_opacity(pin_k.numpy())
            if with_rate:
                step.set_heat_rate(pin_rate.numpy())
            step.run(1)
            step.readback(dst.numpy())
            if with_rate:
                step.read_heat_rate(pin_rate.numpy())
        ev1.record()
        torch.cuda.synchronize()
        t = torch.tensor([ev0.elapsed_time(ev1)], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return world * n * n * e2e_steps / (float(t.item()) / 1e3) / 1e6

    e2e_value = e2e_leg(True)
    e2e_cold = e2e_leg(False)

    cpu = parity = None
    if rank == 0 and world == 1:
        # the CPU baseline on the same world: one f64 twin step of the benchmark's own start state, all host threads;
        # its result doubles as the full-size parity check of one GPU step from the same f32 start
        threads = os.cpu_count() or 1
        v, secs, done, twin = cpu_twin_run(n, 1, threads, budget_s=0.0, world=(cfg, P, kappa))
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{done} f64 twin step of the {n}x{n} benchmark world itself (Twin::new untimed), "
                         f"{secs:.1f} s on {threads} threads"}
        parity = full_step_parity(step, twin, P, kappa)
        del twin
    fld = None
    configs = None
    batched = None
    if rank == 0 and not args.no_fld and world == 1:
        step.close()
        fld = fld_time_to_tol(2048 if n >= 2048 else n)
        configs = config_runs(measured_peaks()[0])
    step.close()
    if rank == 0 and not args.no_batch and world == 1:
        batched = batch_measure(64, 2, 3)
    boxed = None
    if rank == 0 and not args.no_box and world == 1:
        boxed = box_measure()

    if rank == 0:
        peak, peak_kind = measured_peaks()
        upd_ms = parts.hydro_update_ms / max(1, parts.hydro_update_launches)
        upd_gbs = HYDRO_UPDATE_BYTES_PER_CELL * n * n / (upd_ms / 1e3) / 1e9
        sm_bytes = (SMOOTH_PRE_BYTES_PER_CELL + SMOOTH_POST_BYTES_PER_CELL) * n * n
        sm_ms = pre_ms + post_ms
        achieved = sm_bytes / (sm_ms / 1e3) / 1e9 if sm_ms > 0 else None
        tr_pre, tr_post = committed_traffic("mg_smooth_pre_level0", n * n), committed_traffic("mg_smooth_post_level0", n * n)
        roofline = {"kernel": "mg_rowband_tma_kernel level 0 (pre + post, one V-cycle)", "bound": "hbm",
                    "achieved": achieved, "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                    "frac": achieved / peak if achieved else None,
                    "traffic": (tr_pre + tr_post) if tr_pre and tr_post else None,
                    "algorithmic_bytes": sm_bytes, "ms_per_launch": {"pre": pre_ms, "post": post_ms},
                    "algorithmic_bytes_per_cell": {"pre": SMOOTH_PRE_BYTES_PER_CELL,
                                                   "post": SMOOTH_POST_BYTES_PER_CELL},
                    "peak_kind": "burst copy bandwidth (kernels timed alone)",
                    "other": {"hydro_band_kernel<kHydroUpdateGrav>": {
                        "achieved": upd_gbs, "frac": upd_gbs / peak, "ms_per_launch": upd_ms,
                        "algorithmic_bytes_per_cell": HYDRO_UPDATE_BYTES_PER_CELL,
                        "traffic": committed_traffic("hydro_update", n * n)}}}
        clocks = sampler.summary()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(n, world),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 6 * 4 * n * n,
                    "d2h_bytes_per_step": 5 * 4 * n * n, "steps": e2e_steps,
                    "what": "per step through the C ABI: the cells, κ and P5's rate in from pinned host memory, the "
                            "cells and the rate out (the run's resumable state, as a dump carries it)",
                    "cells_only": {"value": e2e_cold, "h2d_bytes_per_step": 5 * 4 * n * n,
                                   "d2h_bytes_per_step": 4 * 4 * n * n,
                                   "what": "the cells and κ in, the cells out: each step's implicit solve starts cold"}},
            "gpu_launches": int(cost.kernel_launches),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clocks,
            "breakdown_ms_per_step": {"gravity": parts.gravity_ms / BREAKDOWN_STEPS,
                                      "hydro": parts.hydro_ms / BREAKDOWN_STEPS,
                                      "heat": parts.heat_ms / BREAKDOWN_STEPS,
                                      "floors_dt": parts.dt_ms / BREAKDOWN_STEPS,
                                      "total": parts.total_ms / BREAKDOWN_STEPS,
                                      "how": f"{BREAKDOWN_STEPS} further steps with the passes launched one by one"},
            "heat_last_step": {"passes": heat.passes, "rounds": heat.rounds, "refinements": heat.refinements,
                               "converged": heat.converged, "rel_residual": heat.rel_residual},
            "parity": parity,
            "fld_time_to_1e-8": fld,
            "other_configs": configs,
            "batched": batched,
            "active_box": boxed,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
