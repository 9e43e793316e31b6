"""Headless clients on the GPU (cls_b200.clients).

* The gym environment (MassSpringEnv, multitask/mass_spring_env.py:15-219)
  driven by an outside policy that evaluates the reference controller on the
  host (sin MLP, multitask/nn.py:130-146) from each observation reproduces
  the reference's golden rollout: the observations equal the reference's
  input_state rows and the centres its centre field (FP64, rel 1e-9).
* The interactive session (interactive_3d.py:38-74) advancing frames of a
  running episode, with a goal change between frames, equals one plain
  rollout with the same targets (FP64, rel 1e-12)."""
import numpy as np
import pytest

from helpers import load_golden, max_rel, params_from_golden

pytestmark = pytest.mark.gpu


def _quad_robot(g, **kw):
    import cls_b200
    return cls_b200.Robot(g["objects"], g["springs"], robot_id=int(g["robot_id"]), hidden=[int(g["n_hidden"])],
                          **kw)


def test_gym_steps_with_host_policy_reproduce_the_golden_rollout():
    from cls_b200.clients import MassSpringEnvCUDA
    g = load_golden("quad_ref")
    B, steps = int(g["B"]), int(g["steps"])
    env = MassSpringEnvCUDA(_quad_robot(g), B, params_from_golden(g, precision=64), training=False,
                            interactive=True, initial_objects=g["x0"][0])
    try:
        env.batch.set_state(g["x0"].reshape(-1, 3))
        env.x0 = g["x0"][0]
        env.tv, env.th, env.tc = g["target_v"].copy(), g["target_h"].copy(), g["target_c"].copy()
        env._push_targets()
        env.reset()
        n_in = env.n_input_states
        for t in range(steps - 1):
            obs = env.get_state(t, clip=False).reshape(B, n_in)
            assert max_rel(obs, g["input_state"][t]) < 1e-9, t
            h = np.sin(obs @ g["W1"].T + g["b1"])
            act = np.sin(h @ g["W2"].T + g["b2"])
            _, reward, done, _ = env.step(act[:, env.act_spring])
            assert np.isfinite(reward)
        assert max_rel(env.center[:steps - 1], g["center"][:steps - 1]) < 1e-9
        assert max_rel(env.height[1:steps - 1], g["height"][1:steps - 1]) < 1e-9
        assert np.all(np.abs(env.get_state()) <= 1.0)
    finally:
        env.close()


def _plain_final_state(g, params, targets, steps):
    import cls_b200
    b = cls_b200.MassSpringBatch([_quad_robot(g)], [0], params)
    b.set_state(g["x0"][0])
    b.set_weights(0, 0, g["W1"], g["b1"])
    b.set_weights(0, 1, g["W2"], g["b2"])
    b.set_targets(*targets)
    b.forward(steps + 1)          # training rollout: `steps` substeps
    x = b.final_state()[0]
    b.close()
    return x


def test_interactive_frames_equal_a_plain_rollout():
    from cls_b200.clients import InteractiveSession
    g = load_golden("quad_ref")
    T, K = 48, 8
    params = params_from_golden(g, precision=64, K=K, max_steps=T)
    s = InteractiveSession(_quad_robot(g), [(g["W1"], g["b1"]), (g["W2"], g["b2"])], params,
                           x0=g["x0"][0], target=(0.05, 0.1, 0.0))
    try:
        for _ in range(2):
            s.step_frame()
        s.set_target(target_v=-0.08, target_h=0.12)
        x = s.step_frame()
    finally:
        s.close()
    tv = np.zeros((T, 1, 3))
    th = np.full((T, 1), 0.1)
    tv[:, 0, 0] = 0.05
    tv[16:, 0, 0] = -0.08
    th[16:] = 0.12
    ref = _plain_final_state(g, params, (tv, th, np.zeros((T, 1))), 3 * K)
    assert max_rel(x, ref) < 1e-12
