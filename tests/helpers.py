"""Shared builders for the tests: golden fixtures, oracle and GPU batches."""
import os

import numpy as np

from oracle.ms_oracle import MassSpringOracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TRAIN_CASES = ("quad_ref", "spider_ref", "x_all_losses")


def load_golden(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: g[k] for k in g.files}


def golden_kwargs(g):
    return dict(n_sin=int(g["n_sin"]), dup_v=int(g["dup_v"]), dup_h=int(g["dup_h"]),
                dup_c=int(g["dup_c"]), dt=float(g["dt"]), gravity=float(g["gravity"]),
                ground=float(g["ground"]), drag=float(g["drag"]), dashpot=float(g["dashpot"]),
                spring_omega=float(g["spring_omega"]), run_period=int(g["run_period"]),
                turn_period=int(g["turn_period"]), jump_period=int(g["jump_period"]),
                robot_id=int(g["robot_id"]), max_speed=float(g["max_speed"]),
                max_height=float(g["max_height"]),
                loss=[str(s) for s in g["loss_names"]])


def oracle_from_golden(g, **over):
    kw = golden_kwargs(g)
    kw.update(over)
    custom = "hidden" in kw or "out_index" in kw
    hidden = kw.pop("hidden", [int(g["n_hidden"])])
    o = MassSpringOracle(g["objects"], g["springs"], int(g["B"]), int(g["T"]),
                         hidden=hidden, initial_objects=g["x0"][0], **kw)
    if not custom:
        o.set_weights([g["W1"], g["W2"]], [g["b1"], g["b2"]])
    o.x[0] = g["x0"]
    o.set_targets(g["target_v"], g["target_h"], g["target_c"])
    return o


def params_from_golden(g, precision=64, K=10, **over):
    import cls_b200
    loss = [str(s) for s in g["loss_names"]]
    p = dict(max_steps=int(g["T"]), dt=float(g["dt"]), gravity=float(g["gravity"]),
             ground_height=float(g["ground"]), drag_damping=float(g["drag"]),
             dashpot_damping=float(g["dashpot"]), friction=0.4, stiffness_scale=0.1,
             run_period=int(g["run_period"]), turn_period=int(g["turn_period"]),
             jump_period=int(g["jump_period"]), spring_omega=float(g["spring_omega"]),
             n_sin_waves=int(g["n_sin"]), duplicate_v=int(g["dup_v"]),
             duplicate_h=int(g["dup_h"]), duplicate_c=int(g["dup_c"]),
             activation_hidden="sin", activation_output="sin", loss=loss,
             precision=precision, checkpoint_every=K, max_speed=float(g["max_speed"]),
             max_height=float(g["max_height"]))
    p.update(over)
    return cls_b200.default_params(**p)


def batch_from_golden(g, precision=64, K=10, **over):
    import cls_b200
    robot = cls_b200.Robot(g["objects"], g["springs"], robot_id=int(g["robot_id"]),
                           hidden=[int(g["n_hidden"])])
    B = int(g["B"])
    b = cls_b200.MassSpringBatch([robot], [0] * B, params_from_golden(g, precision, K, **over))
    b.set_state(g["x0"].reshape(-1, 3))
    b.set_weights(0, 0, g["W1"], g["b1"])
    b.set_weights(0, 1, g["W2"], g["b2"])
    b.set_targets(g["target_v"], g["target_h"], g["target_c"])
    return b


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


def max_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def many_env_batch(precision, n_envs, hidden, K, steps_max, path):
    """n_envs envs of the quadruped golden robot with a custom controller
    (hidden widths `hidden`, Xavier-uniform weights), seeded perturbed
    states and targets, on controller path `path`."""
    import cls_b200
    g = load_golden("quad_ref")
    robot = cls_b200.Robot(g["objects"], g["springs"], robot_id=int(g["robot_id"]), hidden=hidden,
                           n_outputs=0)
    p = params_from_golden(g, precision=precision, K=K, max_steps=steps_max,
                           loss=["velocity", "height", "rotation"])
    b = cls_b200.MassSpringBatch([robot], [0] * n_envs, p)
    b.set_controller_path(path)
    rng = np.random.default_rng(11)
    b.set_state(np.tile(g["x0"][0], (n_envs, 1)) + rng.normal(0, 1e-3, (n_envs * g["objects"].shape[0], 3)))
    b.set_targets(rng.uniform(-0.1, 0.1, (steps_max, n_envs, 3)), rng.choice([-1.0, 0.0, 1.0], (steps_max, n_envs)))
    for l in range(len(hidden) + 1):
        rows, cols = b.layer_shape(0, l)
        b.set_weights(0, l, rng.uniform(-1, 1, (rows, cols)) * np.sqrt(6 / cols), rng.uniform(-0.1, 0.1, rows))
    return b
