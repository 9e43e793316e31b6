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


# --------------------------------------------------------------------------
# Benchmarked workloads against per-robot oracles

def workload_oracle_kwargs(p, robot):
    """MassSpringOracle keyword arguments for a robot under the C-ABI
    parameter block `p` (a cls_b200 SimParams)."""
    inv = {v: k for k, v in (("sin", 0), ("tanh", 1))}
    bits = {"velocity": 1, "height": 2, "pose": 4, "actuation": 8, "rotation": 16, "crawl": 32}
    kw = dict(n_sin=p.n_sin_waves, dup_v=p.duplicate_v, dup_h=p.duplicate_h,
              dup_c=p.duplicate_c, dt=p.dt, gravity=p.gravity, ground=p.ground_height,
              drag=p.drag_damping, dashpot=p.dashpot_damping, spring_omega=p.spring_omega,
              run_period=p.run_period, turn_period=p.turn_period, jump_period=p.jump_period,
              robot_id=robot.robot_id, friction=p.friction, max_speed=p.max_speed,
              max_height=p.max_height, act_hidden=inv[p.activation_hidden],
              act_out=inv[p.activation_output],
              loss=[n for n, b in bits.items() if p.loss_mask & b],
              stiffness_div=1.0 / p.stiffness_scale, hidden=list(robot.hidden))
    if robot.spring_output is not None:
        kw.update(out_index=robot.spring_output,
                  n_out=robot.n_outputs if robot.n_outputs > 0 else robot.n_springs)
    return kw


class WorkloadCase:
    """A GPU batch of `robots` (env e runs robots[env_robot[e]]) and one FP64
    oracle per robot type holding that type's envs, fed identical seeded
    initial states (the robots' rest poses plus N(0, 1e-3) noise), targets
    (vx, vz, height ~ U(-0.1, 0.1) held per turn period) and Xavier-uniform
    weights with U(-0.1, 0.1) biases."""

    def __init__(self, robots, env_robot, params, seed=0, path="per_env"):
        import cls_b200
        from oracle.ms_oracle import MassSpringOracle
        self.robots, self.env_robot, self.p = robots, list(env_robot), params
        T, E = params.max_steps, len(env_robot)
        rng = np.random.default_rng(seed)
        self.b = cls_b200.MassSpringBatch(robots, env_robot, params)
        self.b.set_controller_path(path)
        x0 = [robots[r].objects + rng.normal(0.0, 1e-3, robots[r].objects.shape) for r in env_robot]
        self.b.set_state(np.concatenate(x0))
        n_blocks = T // params.turn_period + 1
        draws = rng.uniform(-0.1, 0.1, size=(n_blocks, E, 3))
        idx = np.arange(T) // params.turn_period
        tv = np.zeros((T, E, 3))
        tv[:, :, 0], tv[:, :, 2] = draws[idx, :, 0], draws[idx, :, 1]
        th = draws[idx, :, 2]
        self.b.set_targets(tv, th)
        self.weights = []
        for r, rb in enumerate(robots):
            Ws, bs = [], []
            for l in range(len(rb.hidden) + 1):
                rows, cols = self.b.layer_shape(r, l)
                W = rng.uniform(-1, 1, (rows, cols)) * np.sqrt(6.0 / cols)
                bb = rng.uniform(-0.1, 0.1, rows)
                self.b.set_weights(r, l, W, bb)
                Ws.append(W)
                bs.append(bb)
            self.weights.append((Ws, bs))
        self.oracles, self.envs = [], []
        for r, rb in enumerate(robots):
            envs = [e for e, rr in enumerate(env_robot) if rr == r]
            self.envs.append(envs)
            if not envs:
                self.oracles.append(None)
                continue
            o = MassSpringOracle(rb.objects, rb.springs, len(envs), T,
                                 initial_objects=rb.objects, **workload_oracle_kwargs(params, rb))
            o.set_weights(*self.weights[r])
            o.x[0] = np.stack([x0[e] for e in envs])
            o.set_targets(tv[:, envs], th[:, envs])
            self.oracles.append(o)

    def run_oracles(self, steps):
        """forward + loss + backward of every oracle; returns the summed loss."""
        return sum(o.run(steps) for o in self.oracles if o is not None)

    def errors(self, steps, traj_steps=None):
        """Runs the GPU batch (forward, loss, backward) and returns the worst
        relative errors against the oracles (which must have run):
        traj (max |dx| / max |x| over the first traj_steps substeps of every
        env), loss, gW, gb (per layer and robot, 2-norm relative), gx0, gv0."""
        b = self.b
        loss = b.simulate(steps)
        ref = sum(o.loss[0] for o in self.oracles if o is not None)
        err = dict(loss=abs(loss - ref) / abs(ref), traj=0.0, gW=0.0, gb=0.0, gx0=0.0, gv0=0.0)
        traj = b.trajectory() if traj_steps else None
        gx0, gv0 = b.state_grads()
        for r, o in enumerate(self.oracles):
            if o is None:
                continue
            for l in range(o.L):
                gW, gb = b.get_grads(r, l)
                err["gW"] = max(err["gW"], rel_err(gW, o.gW[l]))
                err["gb"] = max(err["gb"], rel_err(gb, o.gb[l]))
            for j, e in enumerate(self.envs[r]):
                s = b.env_slice(e)
                err["gx0"] = max(err["gx0"], rel_err(gx0[s], o.gx[0, j]))
                err["gv0"] = max(err["gv0"], rel_err(gv0[s], o.gv[0, j]))
                if traj is not None:
                    err["traj"] = max(err["traj"], max_rel(traj[:traj_steps, s], o.x[:traj_steps, j]))
        return loss, err

    def close(self):
        self.b.close()


# --------------------------------------------------------------------------
# The reference trainer's call sequence (tests/golden/simulate_trace.json)

def load_simulate_trace(case):
    """Calls DiffPhyTrainer.simulate made on its env / solver / model for a
    golden case, recorded from the reference's own source by make_golden.py."""
    import json
    with open(os.path.join(GOLDEN, "simulate_trace.json")) as f:
        return json.load(f)[case]


def replay_simulate_trace(calls, env, nn, tape):
    """Issues the recorded calls on drop-in objects: [object, method, args,
    kwargs] rows; ``tape`` rows open and close ``tape(env.loss)``."""
    objs = {"env": env, "solver": env.solver, "nn": nn, "env.loss": env.loss}
    for i, l in enumerate(env.losses):
        objs["env.losses[%d]" % i] = l
    open_tapes = []
    for obj, method, args, kwargs in calls:
        if obj == "tape":
            if method == "__enter__":
                t = tape(env.loss)
                t.__enter__()
                open_tapes.append(t)
            else:
                open_tapes.pop().__exit__(None, None, None)
            continue
        getattr(objs[obj], method)(*args, **kwargs)
    assert not open_tapes
