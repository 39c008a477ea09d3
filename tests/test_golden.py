"""The oracle against the committed golden fixtures (tests/golden/, made by tests/golden/make_golden.py): the seeded
scene generators still give the stored inputs bit for bit, and the f64 twin run from them reproduces the stored
output (stored as f32: within 1e-6 rel L1 per field)."""
import numpy as np
import pytest

import oracle as O
from golden_cases import CASES, load, rel_l1
from sandbox_reactions_b200 import scenes


@pytest.mark.parametrize("name", CASES)
def test_the_seeded_inputs_are_the_stored_ones(name):
    cfg, planes, kappa, steps, out = load(name)
    made = {"sod_64": lambda: (scenes.sod(64)[1], None), "fld_64": lambda: scenes.fld(64)[1:],
            "full_step_64": lambda: scenes.full_step(64)[1:]}[name]()
    assert np.array_equal(made[0].astype(np.float32), planes)
    if kappa is not None:
        assert np.array_equal(made[1].astype(np.float32), kappa)


@pytest.mark.parametrize("name", CASES)
def test_the_twin_reproduces_the_golden_output(name):
    cfg, planes, kappa, steps, out = load(name)
    twin = O.Twin(cfg, planes.astype(np.float64), None if kappa is None else kappa.astype(np.float64))
    twin.step(steps)
    got = twin.state()
    for k in range(4):
        if np.abs(out[k]).sum() == 0.0:
            assert np.abs(got[k]).max() < 1e-30
            continue
        assert rel_l1(got[k], out[k]) <= 1e-6, (name, k, rel_l1(got[k], out[k]))
