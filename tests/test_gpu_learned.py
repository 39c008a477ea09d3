"""The learned preconditioner (no reference counterpart): its tcgen05 BF16 convolutions, hand-written backward pass and
Adam training on the GPU, checked against the f64 CPU network of oracle/unet.py, and its use inside flexible CG on the
implicit FLD system, judged by the true FP64 residual.

Tolerances: against the CPU network with the same BF16 rounding of every convolution's operands (what the tensor
cores are fed), the output and every layer's gradient agree to rel L2 <= 1e-3 (FP32 against f64 accumulation, and
the rare operand whose FP32 and f64 values round to different BF16 neighbours); against the exact f64 network, within
BF16's own error, rel L2 <= 5e-2. Solves reach an FP64 relative residual <= 1e-8 (cfg.solve_tol)."""
import numpy as np
import pytest

from oracle import unet
from sandbox_reactions_b200 import scenes
from sandbox_reactions_b200.engine import Learner, Step

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def layer_slices():
    k = 0
    for ci, co, _, _ in unet.LAYERS:
        yield slice(k, k + co * 9 * ci), slice(k + co * 9 * ci, k + co * 9 * ci + co)
        k += co * 9 * ci + co


def random_batch(n, crop, seed):
    rng = np.random.default_rng(seed)
    feats = np.empty((n, 4, crop, crop))
    feats[:, 0] = rng.normal(size=(n, crop, crop))
    feats[:, 1:3] = rng.uniform(0.0, 0.25, size=(n, 2, crop, crop))  # Â diagonally dominant
    feats[:, 3] = rng.uniform(0.0, 1.0, size=(n, crop, crop))
    target = rng.normal(size=(n, crop, crop))
    return feats.astype(np.float32), target.astype(np.float32)


@pytest.mark.parametrize("crop,n", [(32, 3), (24, 2)])
def test_forward_and_gradients_match_the_cpu_network(crop, n):
    theta = unet.init_params(5)
    rng = np.random.default_rng(6)
    for _, b in layer_slices():
        theta[b] = 0.05 * rng.normal(size=b.stop - b.start)
    theta = theta.astype(np.float32)
    feats, target = random_batch(n, crop, 7)
    with Learner(crop=crop, capacity=16) as L:
        assert L.param_count == unet.param_count() == 110153
        L.set_params(theta)
        assert np.array_equal(L.get_params(), theta)
        loss, grad, out = L.loss_grad(feats, target)
    f64 = (theta.astype(np.float64), feats.astype(np.float64), target.astype(np.float64))
    e_loss, e_grad, e_out = unet.loss_and_grad(*f64, bf16=True)
    x_loss, x_grad, x_out = unet.loss_and_grad(*f64)
    assert rel_l2(out, e_out) <= 1e-3
    assert abs(loss - e_loss) <= 1e-3 * e_loss
    for li, (w, b) in enumerate(layer_slices()):
        assert rel_l2(grad[w], e_grad[w]) <= 1e-3, (li, rel_l2(grad[w], e_grad[w]))
        assert rel_l2(grad[b], e_grad[b]) <= 1e-3, (li, rel_l2(grad[b], e_grad[b]))
    assert rel_l2(out, x_out) <= 5e-2
    assert rel_l2(grad, x_grad) <= 5e-2


def collect(L, n, scenes_from, count, crops):
    total = 0
    for k in range(count):
        cfg, P, kappa = scenes.fld(n, scene=scenes_from + k)
        with Step(cfg) as s:
            s.upload(P)
            s.upload_opacity(kappa)
            total += L.collect(s, cfg.dt_fixed, crops=crops, seed=k)
    return total


def test_training_on_mg_pcg_pairs_lowers_the_loss():
    """Whole 128² worlds as samples: the untrained network (a zero head) leaves all of the V-cycle's error energy
    (loss ~1); training on the GPU removes most of it."""
    with Learner(crop=128, capacity=512, seed=1) as L:
        got = collect(L, 128, 100, 16, 1)
        assert got >= 32
        first = L.train(1, batch=8, lr=1e-12, seed=0)
        assert 0.9 <= first <= 1.0
        last = L.train(400, batch=8, lr=3e-4, seed=1)
        assert np.isfinite(last)
        assert last < 0.5 * first, (first, last)


def test_the_trained_network_gains_over_the_preconditioner_without_it():
    """Trained on MG-PCG samples of some 256² worlds, evaluated on another world at 512²: with the network's correction
    between its two V-cycles, flexible CG reduces the residual several times more per round than with the untrained
    network (a zero head: the same two V-cycles and nothing between), and needs no more rounds to reach 1e-8."""
    with Learner(crop=256, capacity=600, seed=1) as L, Learner(crop=256, capacity=1, seed=1) as U:
        assert collect(L, 256, 1000, 32, 1) >= 100
        L.train(1500, batch=8, lr=3e-4, seed=0)
        cfg, P, kappa = scenes.fld(512, scene=5001)
        res = {}
        with Step(cfg) as s:
            s.upload(P)
            s.upload_opacity(kappa)
            for name, lr in (("untrained", U), ("trained", L)):
                s.attach_learner(lr)
                s.set_heat_limits(128, 2)
                _, r2, rel2, _ = s.heat_first_solve(cfg.dt_fixed, "learned")
                s.set_heat_limits(128, 4096)
                _, rounds, rel, _ = s.heat_first_solve(cfg.dt_fixed, "learned")
                assert rel <= 1e-8 and not s.last_fallback
                res[name] = (rel2, rounds)
            _, res["mg"], rel, _ = s.heat_first_solve(cfg.dt_fixed, "mg")
    assert res["trained"][0] <= 0.5 * res["untrained"][0], res
    assert res["trained"][1] <= res["untrained"][1] < res["mg"], res


def test_the_untrained_network_adds_nothing_to_the_v_cycles():
    """A zero head: the learned preconditioner is two V-cycles per round, which converges no slower than one."""
    cfg, P, kappa = scenes.fld(128, scene=140)
    with Learner(crop=32, capacity=16) as L, Step(cfg) as s:
        s.upload(P)
        s.upload_opacity(kappa)
        _, r_mg, rel_mg, x_mg = s.heat_first_solve(cfg.dt_fixed, "mg", want_x=True)
        s.attach_learner(L)
        _, r_l, rel_l, x_l = s.heat_first_solve(cfg.dt_fixed, "learned", want_x=True)
        assert not s.last_fallback
    assert rel_mg <= 1e-8 and rel_l <= 1e-8
    assert r_l <= r_mg
    assert np.abs(x_l - x_mg).max() <= 1e-6 * np.abs(x_mg).max()


def test_a_bad_network_falls_back_to_mg_pcg():
    """Weights that make the correction harmful: the solve still reaches 1e-8, through the MG-PCG fallback."""
    cfg, P, kappa = scenes.fld(128, scene=150)
    theta = unet.init_params(9).astype(np.float32) * 2.0  # zero biases: the output grows 2^15-fold
    with Learner(crop=32, capacity=16) as L, Step(cfg) as s:
        L.set_params(theta)
        s.upload(P)
        s.upload_opacity(kappa)
        s.attach_learner(L)
        _, rounds, rel, _ = s.heat_first_solve(cfg.dt_fixed, "learned")
        assert rel <= 1e-8
        fell_back = s.last_fallback
    assert fell_back


def test_a_full_step_runs_with_the_learned_preconditioner():
    cfg, P, kappa = scenes.fld(128, scene=160)
    with Learner(crop=32, capacity=16) as L:
        outs = {}
        for pc in ("mg", "learned"):
            with Step(cfg.replace(precond="mg")) as s:
                s.upload(P)
                s.upload_opacity(kappa)
                if pc == "learned":
                    s.attach_learner(L)
                    s.set_heat_precond("learned")
                s.run(1)
                rep = s.read_heat()
                assert rep.converged and rep.rel_residual <= 1e-8
                outs[pc] = s.readback()
    assert rel_l2(outs["learned"][3], outs["mg"][3]) <= 1e-6
