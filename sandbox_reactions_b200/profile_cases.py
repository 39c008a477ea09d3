"""Small, self-contained workloads to run under a profiler (ncu), one per hot kernel family.

    python -m sandbox_reactions_b200.profile_cases fld --size 2048 --precond mg --solves 3
    python -m sandbox_reactions_b200.profile_cases full --size 2048 --steps 2
    python -m sandbox_reactions_b200.profile_cases learned --size 1024
    python -m sandbox_reactions_b200.profile_cases sod --size 2048 --steps 3
    python -m sandbox_reactions_b200.profile_cases grav --size 2048 --solves 3

fld: the implicit-diffusion world's first system solved to 1e-8 (smoothers, the coarse tail, SpMV, PCG vectors).
full: full steps of the benchmark world (every pass). learned: one flexible-CG round with the learned preconditioner
(an untrained network: the convolution kernels' cost does not depend on the weights). sod: hydro-only steps of a Sod
tube (the stencil kernel). grav: gravity-only steps of a disk (the FFT kernels).
Each prints one line with its device time; every size stays a few GB on the device.
"""
from __future__ import annotations

import argparse
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from sandbox_reactions_b200 import scenes  # noqa: E402
from sandbox_reactions_b200.engine import Learner, Step  # noqa: E402


def fld(size: int, precond: str, solves: int):
    cfg, P, kappa = scenes.fld(size)
    with Step(cfg) as s:
        s.upload(P)
        s.upload_opacity(kappa)
        for _ in range(solves):
            ms, rounds, rel, _ = s.heat_first_solve(cfg.dt_fixed, precond)
    print(f"fld {size}: {precond} first solve {ms:.3f} ms, {rounds} rounds, rel residual {rel:.2e}")


def full(size: int, steps: int):
    cfg, P, kappa = scenes.full_step(size)
    with Step(cfg) as s:
        s.upload(P)
        s.upload_opacity(kappa)
        s.set_timing(True)
        s.run(steps)
        cost = s.read_cost()
    print(f"full {size}: {steps} steps, {cost.total_ms / steps:.3f} ms per step")


def learned(size: int):
    cfg, P, kappa = scenes.fld(size)
    with Learner(crop=64, capacity=1, seed=1) as L, Step(cfg) as s:
        s.upload(P)
        s.upload_opacity(kappa)
        s.attach_learner(L)
        s.set_heat_limits(128, 1)
        ms, rounds, rel, _ = s.heat_first_solve(cfg.dt_fixed, "learned")
        s.attach_learner(None)
    print(f"learned {size}: one round {ms:.3f} ms")


def sod(size: int, steps: int):
    cfg, P = scenes.sod(size)
    with Step(cfg) as s:
        s.upload(P)
        s.set_timing(True)
        s.run(steps)
        cost = s.read_cost()
    print(f"sod {size}: {steps} steps, {cost.total_ms / steps:.3f} ms per step")


def grav(size: int, solves: int):
    cfg, P = scenes.disk(size)
    with Step(cfg.replace(hydro=False, heat=False)) as s:
        s.upload(P)
        s.set_timing(True)
        s.run(solves)  # each step: P2's solve, P8, P9
        cost = s.read_cost()
    print(f"grav {size}: {solves} solves, {cost.gravity_ms / solves:.3f} ms per solve")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["fld", "full", "learned", "sod", "grav"])
    ap.add_argument("--size", type=int, default=2048)
    ap.add_argument("--precond", default="mg")
    ap.add_argument("--solves", type=int, default=3)
    ap.add_argument("--steps", type=int, default=2)
    a = ap.parse_args()
    if a.case == "fld":
        fld(a.size, a.precond, a.solves)
    elif a.case == "full":
        full(a.size, a.steps)
    elif a.case == "learned":
        learned(a.size)
    elif a.case == "sod":
        sod(a.size, a.steps)
    else:
        grav(a.size, a.solves)


if __name__ == "__main__":
    main()
