"""Drop-in for the reference's training path (``main_diff_phy.py --train``).

* ``load_config``: a cfg3d JSON (path or dict) with the reference's derived
  and overwritten keys (multitask/config_sim.py:67-147): the robot built from
  ``robot.robot_id`` (robot_design.py:572-587), dt forced to 0.004, gravity to
  -1.8, dashpot 0.1 (3D), ``spring_omega = 2 pi / (dt run_period)``,
  ``nn.n_input_states``, ``nn.adam_a``, a time-based ``train.random_seed``.
  Explicit ``overrides`` (nested dict) are applied after the derivation, so a
  synthetic configuration can set dt, gravity or friction (the reference
  hard-codes friction 0.4, solver_mass_spring.py:136; ``simulator.friction``
  is this loader's key for it).
* ``DiffPhyTrainer``: the reference trainer's ``simulate`` / ``run_step`` /
  ``train`` / ``evaluate`` (multitask/diffphy_trainer.py:219-435) over one
  ``MassSpringBatch`` of ``nn.batch_size`` envs: forward, loss and the
  checkpointed reverse pass on the GPU (in place of ``ti.ad.Tape``), Adam on
  the device (nn.py:173-191), the ``rounded_train`` state carry-over after
  iteration 5000 (:270-275), weights in the reference's pickle layout
  ``[W1 (H x n_in), W2 (n_out x H), b1 (H), b2 (n_out)]`` of float64
  (nn.py:152-161), and JSONL metrics in place of TensorBoard.
* ``RolloutLoss``: a ``torch.autograd.Function`` whose forward is the rollout
  loss of the controller weights and whose backward is the hand-written
  adjoint, so torch optimisers can train the controller.
"""
import copy
import json
import math
import os
import pickle
import time

import numpy as np

from . import robot_design
from .batch import MassSpringBatch, Robot, default_params

INITIAL_SHIFT_X = 0.4   # setup_robot moves the robot by +0.4 in x (taichi_env.py:497-504)


# ------------------------------------------------------------------ config
def _merge(dst, src):
    for k, v in src.items():
        if isinstance(v, dict) and isinstance(dst.get(k), dict):
            _merge(dst[k], v)
        else:
            dst[k] = v


def load_config(src, overrides=None, skeleton=None, seed=None):
    """cfg3d config (path or dict) with the derived keys; see the module
    docstring.  `skeleton`: path of the spider's node/link table (robot 103)."""
    if isinstance(src, (str, os.PathLike)):
        with open(src) as f:
            cfg = json.load(f)
        name = os.path.splitext(os.path.basename(str(src)))[0]
    else:
        cfg = copy.deepcopy(src)
        name = cfg.get("train", {}).get("name", "config")
    robot = cfg["robot"]
    if robot.get("simulator", "mass_spring") != "mass_spring" or int(robot.get("dim", 3)) != 3:
        raise NotImplementedError("the trainer drives 3D mass-spring robots (MPM: cls_b200.mpm)")
    objects, springs, faces = robot_design.reference_robot(
        int(robot["robot_id"]), float(robot["spring_stiffness"]), float(robot["spring_actuation"]),
        skeleton=skeleton, faces=True)
    robot["objects"] = objects
    robot["springs"] = springs
    robot["faces"] = faces
    robot["n_objects"] = int(len(objects))
    robot["n_springs"] = int(len(springs))
    pr, sim, nn = cfg["process"], cfg["simulator"], cfg["nn"]
    pr["dt"] = 0.004
    pr["spring_omega"] = 2 * math.pi / pr["dt"] / pr["run_period"]
    sim["gravity"] = -1.8
    sim["dashpot_damping"] = 0.1
    sim["n_particles"] = robot["n_objects"]
    if "mpm" in sim:
        sim["mpm"]["dx"] = 1 / sim["mpm"]["n_grid"]
        sim["mpm"]["inv_dx"] = 1 / sim["mpm"]["dx"]
    dim = 3
    nn["n_input_states"] = (nn["n_sin_waves"] + dim * 2 * robot["n_objects"] + nn["duplicate_v"] * (dim - 1)
                            + nn["duplicate_h"] + nn["duplicate_c"])
    nn["adam_a"] = nn["learning_rate"]
    cfg["train"]["random_seed"] = int(seed if seed is not None else (time.time() * 1e6) % 10000)
    cfg["train"].setdefault("config_name", name)
    if overrides:
        _merge(cfg, overrides)
    return cfg


def sim_params(cfg, precision=32, checkpoint_every=50, max_steps=None, keep_trajectory=False):
    """Batch parameters of a loaded config (the solver's constants:
    solver_mass_spring.py:58-148, taichi_env.py:149-183, nn.py:173-191)."""
    pr, sim, nn = cfg["process"], cfg["simulator"], cfg["nn"]
    return default_params(
        max_steps=int(max_steps if max_steps is not None else pr["max_steps"]), dt=float(pr["dt"]),
        gravity=float(sim["gravity"]), ground_height=float(sim["ground_height"]),
        drag_damping=float(sim.get("drag_damping", 0.0)), dashpot_damping=float(sim["dashpot_damping"]),
        friction=float(sim.get("friction", 0.4)), stiffness_scale=0.1, run_period=int(pr["run_period"]),
        turn_period=int(pr["turn_period"]), jump_period=int(pr["jump_period"]),
        spring_omega=float(pr["spring_omega"]), n_sin_waves=int(nn["n_sin_waves"]),
        duplicate_v=int(nn["duplicate_v"]), duplicate_h=int(nn["duplicate_h"]),
        duplicate_c=int(nn["duplicate_c"]), activation_hidden="sin", activation_output="sin",
        loss=list(cfg["train"]["task"]), precision=precision, checkpoint_every=checkpoint_every,
        max_speed=float(pr["max_speed"]), max_height=float(pr["max_height"]), adam_b1=float(nn["adam_b1"]),
        adam_b2=float(nn["adam_b2"]), learning_rate=float(nn["learning_rate"]),
        keep_trajectory=1 if keep_trajectory else 0)


def write_obj_frames(x, faces, folder, stride=10):
    """Headless mesh export of one env's trajectory (the evaluation
    visualiser's 3D branch, diffphy_trainer.py:334-347): every `stride`-th
    state of x [T][N][3] becomes ``{i:06d}.obj`` (i = index of the written
    frame) with ``v x y z`` lines (6 decimals) and 1-based ``f a b c``
    triangles.  Returns the paths written."""
    os.makedirs(folder, exist_ok=True)
    frames = np.asarray(x, np.float64)[::stride]
    face_lines = "".join("f %d %d %d\n" % (a + 1, b + 1, c + 1) for a, b, c in np.asarray(faces).reshape(-1, 3))
    paths = []
    for i, xt in enumerate(frames):
        path = os.path.join(folder, "%06d.obj" % i)
        with open(path, "w") as f:
            f.write("".join("v %.6f %.6f %.6f\n" % (p[0], p[1], p[2]) for p in xt))
            f.write(face_lines)
        paths.append(path)
    return paths


def script_targets(T, steps, max_speed):
    """Evaluation targets (initialize_script, taichi_env.py:340-376, with the
    arguments DiffPhyTrainer.simulate passes for 3D: -v, 0, 0, v, v, 0, 0, -v):
    1000-step phases of target velocity, then height targets -1 and 1."""
    tv = np.zeros((T, 3))
    th = np.zeros(T)
    phases = [(-max_speed, 0.0), (0.0, max_speed), (max_speed, 0.0), (0.0, -max_speed)]
    for t in range(min(steps, T)):
        ph = t // 1000
        if ph < 4:
            tv[t, 0], tv[t, 2] = phases[ph]
        else:
            th[t] = -1.0 if ph == 4 else 1.0
    return tv, th


# ---------------------------------------------------------- weight pickles
def to_reference_list(layers):
    """[(W, b) per layer] -> the reference pickle list [W1, W2, b1, b2]
    (two-layer controllers, nn.py:43)."""
    if len(layers) != 2:
        raise ValueError("the reference layout holds one hidden layer (two weight matrices)")
    (W1, b1), (W2, b2) = layers
    return [np.asarray(W1, np.float64), np.asarray(W2, np.float64), np.asarray(b1, np.float64),
            np.asarray(b2, np.float64)]


def from_reference_list(vals):
    W1, W2, b1, b2 = [np.asarray(v, np.float64) for v in vals]
    return [(W1, b1), (W2, b2)]


class DiffPhyTrainer:
    """Training / evaluation driver with the reference trainer's interface."""

    change_iter = 5000

    def __init__(self, config, batch_size=None, precision=32, checkpoint_every=50, evaluate=False,
                 weights_seed=0, log_path=None, stream=None, keep_trajectory=False):
        self.config = config if isinstance(config, dict) and "objects" in config.get("robot", {}) \
            else load_config(config)
        cfg = self.config
        pr, nn = cfg["process"], cfg["nn"]
        self.max_steps = int(pr["evaluate_max_steps"] if evaluate else pr["max_steps"])
        self.batch_size = int(batch_size if batch_size is not None else nn["batch_size"])
        self.max_speed = float(pr["max_speed"])
        self.max_height = float(pr["max_height"])
        self.max_reset_step = int(nn.get("max_reset_step", 4))
        self.loss_enable = set(cfg["train"]["task"])
        robot = cfg["robot"]
        self.robot = Robot(np.asarray(robot["objects"], np.float64), np.asarray(robot["springs"], np.float64),
                           robot_id=int(robot["robot_id"]), hidden=[int(nn["n_hidden"])])
        # the reference steps max_steps + 1 states in evaluation (t in [0, steps])
        T = self.max_steps + 2 if evaluate else self.max_steps
        self.faces = np.asarray(robot.get("faces", np.zeros((0, 3), np.int64)), np.int64).reshape(-1, 3)
        self.params = sim_params(cfg, precision, checkpoint_every, max_steps=T,
                                 keep_trajectory=keep_trajectory)
        self.batch = MassSpringBatch([self.robot], [0] * self.batch_size, self.params)
        if stream is not None:
            self.batch.set_stream(stream)
        self.initial_objects = self.robot.objects + np.array([INITIAL_SHIFT_X, 0.0, 0.0])
        self.reset_state()
        self.batch.weights_init(weights_seed)
        self.seed = int(cfg["train"].get("random_seed", 0))
        self.iter = 0
        self.reset_step = 2
        self.best = 1e15
        self.losses_list = []
        self.loss = None
        self.loss_dict = {}
        self.loss_batch = None
        self.total_norm_sqr = 0.0
        self.log_path = log_path

    def close(self):
        self.batch.close()

    # ------------------------------------------------------------- state
    def reset_state(self):
        """Every env at the robot's initial objects, at rest (setup_robot)."""
        x0 = np.tile(self.initial_objects, (self.batch_size, 1))
        self.batch.set_state(x0, np.zeros_like(x0))

    def rounded_train(self, steps, it, reset_step):
        """State carry-over (diffphy_trainer.py:270-275): every env starts from
        the last state of the previous episode, and every reset_step-th env
        (offset it % reset_step) from the initial objects (reset_robot only
        resets positions, taichi_env.py:488-490).  The reference copies
        x[steps] (an index past the training rollout's last written state);
        here the last computed state is carried."""
        x, v = self.batch.final_state()
        n = self.robot.n_vertices
        x = x.reshape(self.batch_size, n, 3)
        start = it % reset_step
        for k in range(start, self.batch_size, reset_step):
            x[k] = self.initial_objects
        self.batch.set_state(x.reshape(-1, 3), v)

    # --------------------------------------------------------- rollouts
    def set_targets(self, target_v, target_h, target_c=None):
        self.batch.set_targets(target_v, target_h, target_c)

    def simulate(self, steps, output_v=None, output_h=None, output_c=None, train=True, iter=0,
                 max_speed=0.08, max_height=0.1, loss_enable=None, targets=None):
        """One episode (diffphy_trainer.py:219-268).  Training: targets sampled
        on the device for iteration `iter` (initialize_train) unless `targets`
        (tv [T][B][3], th [T][B][, tc]) are given; first pass over steps - 1
        substeps, loss, checkpointed reverse pass.  Evaluation: the scripted
        targets over steps + 1 substeps and the loss.  Returns the loss."""
        if targets is not None:
            self.batch.set_targets(*targets)
        if train:
            if targets is None:
                self.batch.initialize_train(iter, steps, self.seed, max_speed)
            self.batch.forward(steps)
            terms, env = self.batch.loss()
            self.batch.backward()
        else:
            if targets is None:
                tv, th = script_targets(self.batch.T, steps, max_speed)
                B = self.batch_size
                self.batch.set_targets(np.repeat(tv[:, None, :], B, 1), np.repeat(th[:, None], B, 1))
            self.batch.forward_eval(steps)
            terms, env = self.batch.loss()
        self.loss = terms["total"]
        self.loss_dict = terms
        self.loss_batch = env[0]
        return self.loss

    def run_step(self):
        """One training iteration (diffphy_trainer.py:277-302)."""
        if self.iter > self.change_iter:
            if self.iter % 500 == 0 and self.reset_step < self.max_reset_step:
                self.reset_step += 1
            self.rounded_train(self.max_steps, self.iter, self.reset_step)
        loss = self.simulate(self.max_steps, iter=self.iter, max_height=self.max_height,
                             max_speed=self.max_speed, loss_enable=self.loss_enable)
        self.total_norm_sqr = self.batch.adam_step(self.iter)
        self.losses_list.append(loss)
        self.iter += 1
        return loss

    def train(self, n_iter, save_dir=None, log_every=1):
        """Iterations with metrics (JSONL) and weight pickles: best.pkl when
        the loss improves, last.pkl, and iter{N}.pkl every 50 iterations
        (diffphy_trainer.py:133-147)."""
        log = open(self.log_path, "a") if self.log_path else None
        try:
            for _ in range(n_iter):
                t0 = time.perf_counter()
                loss = self.run_step()
                dt = time.perf_counter() - t0
                rec = {"iter": self.iter - 1, "loss": loss, "tns": self.total_norm_sqr, "seconds": dt,
                       "env_substeps_per_s": self.batch_size * (self.max_steps - 1) / dt}
                rec.update({"loss_" + k: v for k, v in self.loss_dict.items() if k != "total"})
                if log and (self.iter - 1) % log_every == 0:
                    log.write(json.dumps(rec) + "\n")
                    log.flush()
                if save_dir:
                    os.makedirs(save_dir, exist_ok=True)
                    if loss < self.best:
                        self.best = loss
                        self.dump_weights(os.path.join(save_dir, "best.pkl"))
                    self.dump_weights(os.path.join(save_dir, "last.pkl"))
                    if (self.iter - 1) % 50 == 0:
                        self.dump_weights(os.path.join(save_dir, "iter%d.pkl" % (self.iter - 1)))
                elif loss < self.best:
                    self.best = loss
        finally:
            if log:
                log.close()
        return self.losses_list

    def evaluate(self, load_path=None, steps=None, max_speed=None, mesh_dir=None, mesh_stride=10):
        """Evaluation rollout (diffphy_trainer.py:304-435, one weights file):
        loads `load_path` (a reference pickle) when given and returns the loss
        terms of the scripted episode.  With `mesh_dir`, env k's trajectory is
        written as OBJ frames under ``mesh_dir/k`` (export_meshes)."""
        if load_path is not None:
            self.load_weights(load_path)
        self.reset_state()
        steps = self.batch.T - 2 if steps is None else steps
        self.simulate(steps, train=False, max_speed=self.max_speed if max_speed is None else max_speed)
        if mesh_dir is not None:
            for k in range(self.batch_size):
                self.export_meshes(os.path.join(mesh_dir, str(k)), env=k, stride=mesh_stride)
        return dict(self.loss_dict)

    def export_meshes(self, folder, env=0, stride=10):
        """OBJ frames of env `env`'s last rollout (write_obj_frames); needs the
        trajectory kept (keep_trajectory=True, or a rotation / pose loss)."""
        x = self.batch.trajectory()[:, self.batch.env_slice(env)]
        return write_obj_frames(x, self.faces, folder, stride)

    # ------------------------------------------------------------ weights
    def weights(self):
        return [self.batch.get_weights(0, l) for l in range(self.batch.n_layers(0))]

    def set_weights(self, layers):
        for l, (W, b) in enumerate(layers):
            self.batch.set_weights(0, l, W, b)

    def grads(self):
        return [self.batch.get_grads(0, l) for l in range(self.batch.n_layers(0))]

    def dump_weights(self, name="save.pkl"):
        with open(name, "wb") as f:
            pickle.dump(to_reference_list(self.weights()), f)

    def load_weights(self, name="save.pkl"):
        with open(name, "rb") as f:
            self.set_weights(from_reference_list(pickle.load(f)))


# ------------------------------------------------------------ autograd
def _rollout_function():
    import torch

    class RolloutLoss(torch.autograd.Function):
        """loss = rollout loss of the controller weights (W, b per layer, any
        torch device); backward = the hand-written adjoint of the rollout."""

        @staticmethod
        def forward(ctx, trainer, steps, targets, *params):
            layers = [(params[2 * l].detach().cpu().double().numpy(),
                       params[2 * l + 1].detach().cpu().double().numpy()) for l in range(len(params) // 2)]
            trainer.set_weights(layers)
            trainer.reset_state()
            loss = trainer.simulate(steps, train=True, targets=targets)
            ctx.trainer = trainer
            ctx.meta = [(p.device, p.dtype) for p in params]
            return torch.tensor(loss, dtype=params[0].dtype, device=params[0].device)

        @staticmethod
        def backward(ctx, g):
            grads = ctx.trainer.grads()
            out = []
            for l, (gW, gb) in enumerate(grads):
                for arr, (dev, dt) in ((gW, ctx.meta[2 * l]), (gb, ctx.meta[2 * l + 1])):
                    out.append(torch.from_numpy(arr).to(device=dev, dtype=dt) * g)
            return (None, None, None, *out)

    return RolloutLoss


_ROLLOUT = None


def rollout_loss(trainer, steps, params, targets=None):
    """Differentiable rollout loss: params = [W1, b1, W2, b2, ...] torch
    tensors; the loss's backward runs the checkpointed reverse pass (the
    reference records the same episode under ti.ad.Tape,
    diffphy_trainer.py:246-256)."""
    global _ROLLOUT
    if _ROLLOUT is None:
        _ROLLOUT = _rollout_function()
    return _ROLLOUT.apply(trainer, steps, targets, *params)


# ----------------------------------------------------------------- CLI
def main(argv=None):
    """``python -m cls_b200.trainer --config_file cfg.json --train`` (the
    reference's main_diff_phy.py flags that the training path reads)."""
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--config_file", required=True)
    ap.add_argument("--train", action="store_true")
    ap.add_argument("--evaluate", action="store_true")
    ap.add_argument("--evaluate_path", default=None)
    ap.add_argument("--iters", type=int, default=100)
    ap.add_argument("--skeleton", default=None)
    ap.add_argument("--save_dir", default=None)
    ap.add_argument("--precision", type=int, default=32)
    a = ap.parse_args(argv)
    cfg = load_config(a.config_file, skeleton=a.skeleton)
    tr = DiffPhyTrainer(cfg, precision=a.precision, evaluate=a.evaluate,
                        log_path=os.path.join(a.save_dir, "metrics.jsonl") if a.save_dir else None)
    try:
        if a.evaluate:
            print(json.dumps(tr.evaluate(a.evaluate_path)))
        else:
            tr.train(a.iters, save_dir=a.save_dir)
            print(json.dumps({"iters": tr.iter, "last_loss": tr.losses_list[-1], "best": tr.best}))
    finally:
        tr.close()


if __name__ == "__main__":
    main()
