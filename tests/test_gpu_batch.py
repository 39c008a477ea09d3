"""Batches (config 5's machinery): worlds of uneven sizes stepped together through sr_batch_* give exactly what each
world gives stepped alone through its own context; a refused world names its index."""
import numpy as np
import pytest

from sandbox_reactions_b200 import scenes
from sandbox_reactions_b200.abi import Config
from sandbox_reactions_b200.engine import Batch, SrError, Step

pytestmark = pytest.mark.gpu


def test_a_batch_matches_its_worlds_stepped_alone():
    worlds = [scenes.full_step(n, scene=s) for s, n in enumerate((64, 128, 96 + 32, 64))]
    worlds[2] = scenes.full_step(128, scene=7, sigma0=2.0)
    with Batch([w[0] for w in worlds], threads=3) as b:
        for i, (cfg, P, kappa) in enumerate(worlds):
            b.upload(i, P, kappa)
        ms = b.run(3)
        assert ms > 0.0
        got = [b.readback(i) for i in range(len(worlds))]
        reps = [b.read_heat(i) for i in range(len(worlds))]
    for i, (cfg, P, kappa) in enumerate(worlds):
        with Step(cfg) as s:
            s.upload(P)
            s.upload_opacity(kappa)
            s.run(3)
            want = s.readback()
        assert np.array_equal(got[i], want), i
        assert reps[i].converged


def test_a_refused_world_is_named():
    good = Config(width=64, height=64)
    with pytest.raises(SrError, match="world 1"):
        Batch([good, Config(width=60, height=64)])
