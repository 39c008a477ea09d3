"""The golden fixtures of tests/golden/ (written by tests/golden/make_golden.py) with the configurations they were
made with."""
import os

import numpy as np

from sandbox_reactions_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ("sod_64", "fld_64", "full_step_64")


def load(name):
    """(config with the fixture's fixed Δt, input planes, κ or None, steps, the twin's output)."""
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    cfg = {"sod_64": lambda: scenes.sod(64)[0], "fld_64": lambda: scenes.fld(64)[0],
           "full_step_64": lambda: scenes.full_step(64)[0]}[name]()
    cfg = cfg.replace(dt_fixed=float(d["dt"]))
    kappa = d["kappa"] if "kappa" in d.files else None
    return cfg, d["planes"], kappa, int(d["steps"]), d["out"]


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))
