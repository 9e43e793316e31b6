"""The duck-typed drop-ins on the GPU, driven by the reference trainer's own
call sequence (DiffPhyTrainer.simulate, multitask/diffphy_trainer.py:219-268,
recorded from the reference source into simulate_trace.json): the training
trace reproduces the reference's golden loss and observables and the FP64
oracle's gradients; get_TNS and gradient_update match the oracle's Adam
(nn.py:163-191); the evaluation trace reproduces the golden evaluation loss.

Tolerances: FP64 1e-9 (loss, observables) and 1e-8 (gradients); FP32 1e-5
on observables and 1e-4 on losses and gradients."""
import numpy as np
import pytest

from helpers import load_golden, load_simulate_trace, max_rel, oracle_from_golden, rel_err, \
    replay_simulate_trace
from test_trainer_cpu import golden_config

pytestmark = pytest.mark.gpu

TOL = {64: dict(obs=1e-9, loss=1e-9, grad=1e-8), 32: dict(obs=1e-5, loss=1e-4, grad=1e-4)}


def _objects(case, precision):
    from cls_b200.dropin import ModelCUDA, TaichiEnvCUDA
    from cls_b200.trainer import load_config
    g = load_golden(case)
    cfg = load_config(golden_config(g), seed=3)
    env = TaichiEnvCUDA(cfg, precision=precision, checkpoint_every=9)
    nn = ModelCUDA(cfg, env.max_steps, env.batch_size, env.n_input_states, env.n_springs, env.input_state,
                   env.actuation, env.n_hidden, method=cfg["nn"]["optimizer"])
    env.setup_robot()
    for field, key in ((nn.weights1, "W1"), (nn.weights2, "W2"), (nn.bias1, "b1"), (nn.bias2, "b2")):
        field.from_numpy(g[key])
    return g, env, nn


@pytest.mark.parametrize("precision", [64, 32])
def test_reference_training_trace_matches_golden_and_oracle(precision):
    from cls_b200.dropin import Tape
    g, env, nn = _objects("quad_ref", precision)
    tol = TOL[precision]
    try:
        B, N = int(g["B"]), len(g["objects"])
        np.testing.assert_allclose(env.initial_objects_np, g["x0"][0], rtol=0, atol=1e-15)
        env.inject_targets(g["target_v"], g["target_h"], g["target_c"])
        tr = load_simulate_trace("quad_ref")
        replay_simulate_trace(tr["calls"], env, nn, Tape)
        steps = tr["steps"]
        assert abs(env.loss[None] - float(g["loss"])) <= tol["loss"] * abs(float(g["loss"]))
        np.testing.assert_allclose(env.loss_batch.to_numpy(), g["loss_batch"], rtol=10 * tol["loss"])
        assert max_rel(env.center.to_numpy()[:steps], g["center"][:steps]) < tol["obs"]
        assert max_rel(env.x.to_numpy()[:steps], g["x"][:steps]) < tol["obs"]
        o = oracle_from_golden(g)
        o.run(steps)
        for field, ref in ((nn.weights1, o.gW[0]), (nn.weights2, o.gW[1]), (nn.bias1, o.gb[0]),
                           (nn.bias2, o.gb[1])):
            assert rel_err(field.grad.to_numpy(), ref) < tol["grad"]
        # run_step's optimiser calls (diffphy_trainer.py:287-289)
        tns = nn.get_TNS()
        assert tns == pytest.approx(o.tns(), rel=tol["grad"])
        nn.gradient_update(0)
        m = [np.zeros_like(a) for l in range(2) for a in (o.W[l], o.b[l])]
        v = [np.zeros_like(a) for a in m]
        o.adam(m, v, 3e-4, 0.9, 0.9, 0)
        atol = 1e-12 if precision == 64 else 1e-6
        np.testing.assert_allclose(nn.weights1.to_numpy(), o.W[0], rtol=0, atol=atol)
        np.testing.assert_allclose(nn.bias2.to_numpy(), o.b[1], rtol=0, atol=atol)
    finally:
        env.close()


def test_reference_evaluation_trace_matches_golden():
    from cls_b200.dropin import Tape
    g, env, nn = _objects("snake_eval", 64)
    try:
        tr = load_simulate_trace("snake_eval")
        replay_simulate_trace(tr["calls"], env, nn, Tape)
        steps = tr["steps"]
        assert abs(env.loss[None] - float(g["loss"])) <= 1e-9 * abs(float(g["loss"]))
        assert max_rel(env.center.to_numpy()[:steps + 1], g["center"][:steps + 1]) < 1e-9
    finally:
        env.close()


def test_rounded_train_calls_carry_the_last_state():
    """copy_robot then reset_robot (diffphy_trainer.py:270-275): envs at
    start, start + step, ... restart from the initial objects, the others
    continue from the last state of the previous rollout."""
    from cls_b200.dropin import Tape
    g, env, nn = _objects("quad_ref", 64)
    try:
        env.inject_targets(g["target_v"], g["target_h"], g["target_c"])
        replay_simulate_trace(load_simulate_trace("quad_ref")["calls"], env, nn, Tape)
        xf, vf = env.batch.final_state()
        env.copy_robot(int(g["steps"]))
        env.reset_robot(1, 2, 1)
        N = len(g["objects"])
        x0 = env.x.to_numpy()   # trajectory of the last rollout; x[0] is read back after the next
        env.batch.forward(4)
        x_new = env.batch.trajectory()[0]
        np.testing.assert_allclose(x_new[:N], xf[:N], rtol=0, atol=1e-15)
        np.testing.assert_allclose(x_new[N:2 * N], env.initial_objects_np, rtol=0, atol=1e-15)
        assert x0.shape[1:] == (env.batch_size, N, 3)
    finally:
        env.close()
