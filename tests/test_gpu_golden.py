"""The CUDA path against the committed golden fixtures (tests/golden/): the same inputs, configuration, fixed Δt and
step count as the f64 twin's stored output, within rel L1 <= 1e-5 per field."""
import numpy as np
import pytest

from golden_cases import CASES, load, rel_l1
from sandbox_reactions_b200.engine import Step

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", CASES)
def test_the_gpu_step_matches_the_golden_output(name):
    cfg, planes, kappa, steps, out = load(name)
    with Step(cfg) as s:
        s.upload(planes)
        if kappa is not None:
            s.upload_opacity(kappa)
        s.run(steps)
        gpu = s.readback()
        if cfg.heat:
            assert s.read_heat().converged
    for k in range(4):
        if np.abs(out[k]).sum() == 0.0:
            assert np.abs(gpu[k]).max() == 0.0, (name, k)
            continue
        assert rel_l1(gpu[k], out[k]) <= 1e-5, (name, k, rel_l1(gpu[k], out[k]))
