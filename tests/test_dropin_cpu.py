"""The duck-typed drop-ins (cls_b200.dropin) accept the reference trainer's
own call sequence -- DiffPhyTrainer.simulate (multitask/diffphy_trainer.py:
219-268) recorded from the reference source into simulate_trace.json -- and
turn it into the fused rollout calls, without a GPU (a recording stand-in
replaces the CUDA batch)."""
import types

import numpy as np
import pytest

from helpers import load_golden, load_simulate_trace, replay_simulate_trace
from test_trainer_cpu import golden_config


class FakeBatch:
    """Records the batch calls the drop-in makes; shapes of the golden run."""

    def __init__(self, g, T):
        self.calls = []
        self.T, self.B = T, int(g["B"])
        self.N, self.S, self.H = len(g["objects"]), len(g["springs"]), int(g["n_hidden"])
        self.n_in = int(g["W1"].shape[1])
        self.tv, self.th, self.tc = np.zeros((T, self.B, 3)), np.zeros((T, self.B)), np.zeros((T, self.B))

    def __getattr__(self, name):
        def f(*a, **k):
            self.calls.append((name,) + a)
        return f

    def layer_shape(self, r, l):
        return (self.H, self.n_in) if l == 0 else (self.S, self.H)

    def targets(self):
        return self.tv.copy(), self.th.copy(), self.tc.copy()

    def set_targets(self, tv, th, tc=None):
        self.calls.append(("set_targets",))
        self.tv, self.th = np.asarray(tv, float), np.asarray(th, float)
        if tc is not None:
            self.tc = np.asarray(tc, float)

    def loss(self):
        self.calls.append(("loss",))
        env = np.tile(np.arange(8.0)[:, None], (1, self.B))
        return dict(zip(("total", "velocity", "height", "pose", "rotation", "weight", "actuation",
                         "crawl"), np.arange(8.0) * self.B)), env


def _env(case):
    from cls_b200.dropin import ModelCUDA, TaichiEnvCUDA
    from cls_b200.trainer import load_config
    g = load_golden(case)
    cfg = load_config(golden_config(g), seed=3)
    fake = FakeBatch(g, int(g["T"]) + 2)
    env = TaichiEnvCUDA(cfg, batch=fake)
    nn = ModelCUDA(cfg, env.max_steps, env.batch_size, env.n_input_states, env.n_springs, env.input_state,
                   env.actuation, env.n_hidden, method="adam")
    return g, env, nn, fake


def test_training_trace_runs_one_rollout_and_one_reverse_pass():
    from cls_b200.dropin import Tape
    g, env, nn, fake = _env("quad_ref")
    tr = load_simulate_trace("quad_ref")
    replay_simulate_trace(tr["calls"], env, nn, Tape)
    names = [c[0] for c in fake.calls]
    assert names == ["initialize_train", "set_loss", "forward", "loss", "backward"]
    assert fake.calls[2] == ("forward", tr["steps"])
    assert set(fake.calls[1][1]) == {"velocity", "rotation"}
    assert env.loss[None] == 0.0 * env.batch_size           # the fake's total
    assert env.loss_dict["loss_rotation"][None] == 4.0 * env.batch_size
    np.testing.assert_array_equal(env.loss_batch.to_numpy(), np.zeros(env.batch_size))


def test_injected_targets_replace_the_draw():
    from cls_b200.dropin import Tape
    g, env, nn, fake = _env("quad_ref")
    env.inject_targets(g["target_v"], g["target_h"], g["target_c"])
    replay_simulate_trace(load_simulate_trace("quad_ref")["calls"], env, nn, Tape)
    assert [c[0] for c in fake.calls][:1] == ["set_targets"]
    T = g["target_v"].shape[0]
    np.testing.assert_array_equal(fake.tv[:T], g["target_v"])     # padded to the batch's length
    assert np.all(fake.tv[T:] == 0.0)


def test_evaluation_trace_runs_the_evaluation_rollout():
    from cls_b200.dropin import Tape
    g, env, nn, fake = _env("snake_eval")
    tr = load_simulate_trace("snake_eval")
    replay_simulate_trace(tr["calls"], env, nn, Tape)
    names = [c[0] for c in fake.calls]
    assert names == ["set_targets", "set_loss", "forward_eval", "loss"]
    assert fake.calls[2] == ("forward_eval", tr["steps"])
    # initialize_script's phases (taichi_env.py:340-376) for t < steps
    assert np.all(fake.tv[:tr["steps"], :, 0] == -float(g["max_speed"]))
    assert np.all(fake.tv[tr["steps"]:] == 0.0) and np.all(fake.th == 0.0)


def test_out_of_order_calls_are_rejected():
    from cls_b200.dropin import Tape
    g, env, nn, fake = _env("quad_ref")
    env.solver.clear_states(10)
    env.solver.pre_advance(0)
    with pytest.raises(RuntimeError, match="out-of-order"):
        nn.forward(0)                     # nn_input(0) was skipped
    env.solver.clear_states(10)
    for t in range(5):
        env.solver.pre_advance(t)
        env.nn_input(t, 0, 0.1, 0.1)
        nn.forward(t)
        env.solver.advance(t)
    with pytest.raises(RuntimeError, match="after 5 substeps"):
        env.get_loss(10, loss_enable={"velocity"})
    with pytest.raises(RuntimeError, match="without a training rollout"):
        with Tape(env.loss):
            pass


def test_patch_tape_routes_only_drop_in_losses():
    from cls_b200.dropin import Tape, patch_tape
    g, env, nn, fake = _env("quad_ref")

    class Own:
        def __init__(self, loss):
            self.loss = loss

    ti = types.SimpleNamespace(ad=types.SimpleNamespace(Tape=Own))
    patch_tape(ti)
    assert isinstance(ti.ad.Tape(env.loss), Tape)
    assert isinstance(ti.ad.Tape(object()), Own)


def test_model_shape_and_pickle_layout(tmp_path):
    g, env, nn, fake = _env("quad_ref")
    assert nn.weights1.shape == (env.n_hidden, env.n_input_states)
    with pytest.raises(ValueError):
        from cls_b200.dropin import ModelCUDA
        ModelCUDA(env.config, 10, env.batch_size, env.n_input_states + 1, env.n_springs, None,
                  env.actuation, env.n_hidden)


def test_gym_actions_map_to_controller_outputs():
    """MassSpringEnvCUDA turns the actions of the actuated springs into the
    controller-output rows of cls_env_step: one shared row (the reference
    passes action[i] to every env, mass_spring_env.py:56-58) or one per env."""
    from cls_b200.clients import MassSpringEnvCUDA
    env = MassSpringEnvCUDA.__new__(MassSpringEnvCUDA)
    env.batch_size = 2
    env.act_spring = np.array([1, 3])
    env.n_outputs = 5
    env.spring_output = np.arange(5)
    out = env._outputs([0.5, -0.25])
    np.testing.assert_array_equal(out, [[0, 0.5, 0, -0.25, 0]] * 2)
    out = env._outputs([[1, 2], [3, 4]])
    np.testing.assert_array_equal(out, [[0, 1, 0, 2, 0], [0, 3, 0, 4, 0]])
    env.spring_output = np.array([-1, 0, -1, 1, -1])      # outputs for actuated springs only
    env.n_outputs = 2
    np.testing.assert_array_equal(env._outputs([7, 8]), [[7, 8], [7, 8]])
    with pytest.raises(ValueError):
        env._outputs([1, 2, 3])
