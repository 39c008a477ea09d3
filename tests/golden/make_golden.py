"""Writes the golden fixtures under tests/golden/: seeded inputs and the f64 twin's (oracle/) output after a fixed
number of steps at a fixed Δt, stored as f32 (the GPU parity bar, rel L1 <= 1e-5, is far above f32 rounding).

    python tests/golden/make_golden.py

Cases (64² worlds, the benchmark configurations in small): a Sod tube (γ = 1.4, minmod, leave edges, 5 steps), the
implicit FLD step of the opacity-field world (1 step), the full hydro + gravity + FLD step of the disk with hot spots
(2 steps). The reference itself cannot run here (Rust twin, WGSL GPU path); these pin the oracle against itself over
time and give the GPU tests committed arrays to compare with.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle as O  # noqa: E402
from sandbox_reactions_b200 import scenes  # noqa: E402

N = 64


def natural_dt(cfg, P, kappa):
    """The Δt the twin's own step takes from this state (P9's CFL and gravity bounds)."""
    twin = O.Twin(cfg, P.astype(np.float64), None if kappa is None else kappa.astype(np.float64))
    twin.step(1)
    return float(twin.clock()["dt"])


def cases():
    cfg, P = scenes.sod(N)
    yield "sod_64", cfg.replace(dt_fixed=natural_dt(cfg, P, None)), P, None, 5
    cfg, P, kappa = scenes.fld(N)
    yield "fld_64", cfg, P, kappa, 1
    cfg, P, kappa = scenes.full_step(N)
    yield "full_step_64", cfg.replace(dt_fixed=natural_dt(cfg, P, kappa)), P, kappa, 2


def run(cfg, P, kappa, steps):
    twin = O.Twin(cfg, P.astype(np.float64), None if kappa is None else kappa.astype(np.float64))
    twin.step(steps)
    return twin.state()


def main():
    for name, cfg, P, kappa, steps in cases():
        out = run(cfg, P, kappa, steps)
        arrays = {"planes": P.astype(np.float32), "out": out.astype(np.float32), "steps": np.int32(steps),
                  "dt": np.float64(cfg.dt_fixed)}
        if kappa is not None:
            arrays["kappa"] = kappa.astype(np.float32)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
        moved = [float(np.abs(out[k] - P[k]).sum() / np.abs(P[k]).sum()) if np.abs(P[k]).sum() > 0 else None
                 for k in range(4)]
        print(name, "dt", cfg.dt_fixed, "rel L1 change per field", moved)


if __name__ == "__main__":
    main()
