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


def test_a_captured_step_matches_the_launched_one():
    # after the first step (which tunes the multigrid) a context runs each whole step as one captured graph, the
    # implicit step under device control; with timing on the passes are launched one by one: the same state either way
    cfg, P, kappa = scenes.full_step(96, scene=5)
    out = []
    for timed in (False, True):
        with Step(cfg) as s:
            s.upload(P)
            s.upload_opacity(kappa)
            s.set_timing(2 if timed else 0)
            for _ in range(3):
                s.run(1)
            out.append((s.readback(), s.read_heat()))
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1].rounds == out[1][1].rounds and out[0][1].passes == out[1][1].passes
