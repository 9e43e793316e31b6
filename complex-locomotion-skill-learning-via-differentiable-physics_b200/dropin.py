"""Duck-typed drop-ins for the reference trainer's env / solver / model objects.

The reference trainer drives Taichi fields through three Python objects:
``TaichiEnv`` (multitask/taichi_env.py:20-147) with its solver
``SolverMassSpring`` (multitask/solver_mass_spring.py:8-198), whose fields the
env aliases (taichi_env.py:136-144), and ``Model`` (multitask/nn.py:79-191).
``DiffPhyTrainer.simulate`` (multitask/diffphy_trainer.py:219-268) calls, per
episode::

    solver.clear_states(steps); nn.clear(); env.initialize_train(...) |
    env.initialize_script(...); env.loss[None] = 0; l[None] = 0 for env.losses
    with ti.ad.Tape(env.loss):                    # training only
        for t in range(steps - 1):                # range(steps + 1) evaluating
            solver.pre_advance(t); env.nn_input(t, 0, max_speed, max_height)
            nn.forward(t); solver.advance(t)
        env.get_loss(steps, loss_enable=...)

``TaichiEnvCUDA``, ``SolverMassSpringCUDA`` and ``ModelCUDA`` accept that
protocol unchanged.  Per-substep calls only record the schedule: the fused
CUDA segment kernels run a whole rollout in one pass, so the rollout is
launched when the loss is requested (``env.get_loss``), and the checkpointed
reverse pass when the ``Tape`` context closes.  Calls out of the reference's
order raise ``RuntimeError`` (the fused kernels cannot run a partial substep).

Integration with the reference trainer source::

    import multitask.diffphy_trainer as dt
    from cls_b200 import dropin
    dt.TaichiEnv, dt.Model = dropin.TaichiEnvCUDA, dropin.ModelCUDA
    dropin.patch_tape(dt.ti)         # ti.ad.Tape(env.loss) -> dropin.Tape

Fields are read-only host views of the device state (downloaded on access):
``x`` (needs the trajectory, which the drop-in keeps), ``center``,
``height``, ``upper_height``, ``rotation``, the targets; ``v`` at the last
state.  ``control_length`` must be 1 (every cfg3d configuration's value);
the trainer's ``diff_copy`` path for longer control intervals is not
supported.
"""
import pickle

import numpy as np

from .batch import MassSpringBatch, Robot

LOSS_NAMES = ("velocity", "height", "pose", "actuation", "rotation", "crawl")
# env.loss_dict order (taichi_env.py:82-88) and the cls_loss slot of each
LOSS_DICT = (("loss_velocity", 1), ("loss_height", 2), ("loss_pose", 3), ("loss_rotation", 4),
             ("loss_weight", 5), ("loss_actuation", 6), ("loss_crawl", 7))
INITIAL_SHIFT_X = 0.4   # setup_robot's +0.4 in x (taichi_env.py:497-504)


class ScalarField:
    """A 0-d field: ``f[None]`` reads and writes the value."""

    def __init__(self, value=0.0):
        self.value = float(value)

    def __getitem__(self, key):
        if key is not None and key != ():
            raise IndexError("a 0-d field is indexed with None")
        return self.value

    def __setitem__(self, key, value):
        if key is not None and key != ():
            raise IndexError("a 0-d field is indexed with None")
        self.value = float(value)

    def to_numpy(self):
        return np.array(self.value)

    def fill(self, value):
        self.value = float(value)


class EnvField:
    """A per-env field (``loss_batch`` and the per-term batch losses)."""

    def __init__(self, n):
        self.arr = np.zeros(n)

    def __getitem__(self, k):
        return self.arr[k]

    def __setitem__(self, k, value):
        self.arr[k] = value

    def to_numpy(self):
        return self.arr.copy()

    def fill(self, value):
        self.arr[:] = value


class FieldView:
    """Read-only view of a device field, downloaded on access; indexed like
    the reference's field (``[t, k, i]``)."""

    def __init__(self, fetch, what):
        self._fetch = fetch
        self._what = what

    def to_numpy(self):
        return np.array(self._fetch())

    def __getitem__(self, key):
        return self._fetch()[key]

    def __setitem__(self, key, value):
        raise RuntimeError("%s is a view of the device state; write it through the env "
                           "(setup_robot / reset_robot / copy_robot)" % self._what)

    @property
    def shape(self):
        return self._fetch().shape


class _Episode:
    """Checks the per-substep calls against the reference loop and records the
    rollout's extent."""

    ORDER = ("pre_advance", "nn_input", "forward", "advance")

    def __init__(self, steps):
        self.steps = int(steps)
        self.t = 0          # substep being recorded
        self.stage = 0      # next call expected for substep t

    def call(self, name, t):
        if t != self.t or self.ORDER[self.stage] != name:
            raise RuntimeError("out-of-order call %s(%d): expected %s(%d); the fused kernels run "
                               "whole substeps in the reference's order" % (name, t, self.ORDER[self.stage],
                                                                             self.t))
        self.stage += 1
        if self.stage == len(self.ORDER):
            self.stage, self.t = 0, self.t + 1

    @property
    def substeps(self):
        if self.stage != 0:
            raise RuntimeError("substep %d is incomplete (%s not called)" % (self.t, self.ORDER[self.stage]))
        return self.t


def _config_dict(config):
    return config.get_config() if hasattr(config, "get_config") else config


class SolverMassSpringCUDA:
    """SolverMassSpring's interface (solver_mass_spring.py:8-198) over the
    env's CUDA batch."""

    def __init__(self, env):
        self.env = env
        self.x = FieldView(env._x_field, "x")
        self.v = FieldView(env._v_field, "v")
        self.center = FieldView(lambda: env._observables()["center"], "center")
        self.height = FieldView(lambda: env._observables()["height"], "height")
        self.upper_height = FieldView(lambda: env._observables()["upper_height"], "upper_height")
        self.rotation = FieldView(lambda: env._observables()["rotation"], "rotation")
        self.actuation = FieldView(env._no_field("actuation"), "actuation")

    def clear_states(self, steps):
        self.env._begin(steps)

    def initialize_robot(self):
        """The spring table is uploaded when the batch is created."""

    def pre_advance(self, t):
        self.env._step("pre_advance", t)

    def advance(self, t):
        self.env._step("advance", t)


class TaichiEnvCUDA:
    """TaichiEnv's interface (taichi_env.py:20-510) for 3D mass-spring robots.

    ``config``: the reference's ConfigSim (or its ``get_config()`` dict) after
    the robot was built (``robot.objects``/``springs``, as cls_b200.trainer's
    load_config produces).  ``batch`` replaces the CUDA batch (tests)."""

    def __init__(self, config, precision=32, checkpoint_every=50, stream=None, batch=None, seed=None):
        self.config_ = config
        self.config = cfg = _config_dict(config)
        robot, pr, nn, sim = cfg["robot"], cfg["process"], cfg["nn"], cfg["simulator"]
        if int(robot.get("dim", 3)) != 3 or robot.get("simulator", "mass_spring") != "mass_spring":
            raise NotImplementedError("the drop-in env drives 3D mass-spring robots")
        if int(robot.get("control_length", 1)) != 1:
            raise NotImplementedError("control_length > 1 (the trainer's diff_copy path) is not supported")
        self.dim = 3
        self.max_steps = int(pr["max_steps"])
        self.batch_size = int(nn["batch_size"])
        self.n_hidden = int(nn["n_hidden"])
        self.robot_id = int(robot["robot_id"])
        self.n_input_states = int(nn["n_input_states"])
        self.n_springs = int(robot["n_springs"])
        self.n_objects = int(robot["n_objects"])
        self.objects = robot["objects"]
        self.simulator = "mass_spring"
        self.turn_period, self.run_period = int(pr["turn_period"]), int(pr["run_period"])
        self.jump_period = int(pr["jump_period"])
        self.n_sin_waves, self.spring_omega, self.dt = int(nn["n_sin_waves"]), float(pr["spring_omega"]), \
            float(pr["dt"])
        self.duplicate_v, self.duplicate_h = int(nn["duplicate_v"]), int(nn["duplicate_h"])
        self.duplicate_c = int(nn["duplicate_c"])
        self.ground_height = float(sim["ground_height"])
        self.task = list(cfg["train"]["task"])
        self.seed = int(cfg["train"].get("random_seed", 0) if seed is None else seed)
        for tsk in self.task:
            if tsk not in LOSS_NAMES:
                raise ValueError("unknown loss %r" % (tsk,))
        self.loss = ScalarField()
        self.loss_dict = {name: ScalarField() for name, _ in LOSS_DICT}
        self.losses = list(self.loss_dict.values())
        self.loss_batch = EnvField(self.batch_size)
        self.loss_dict_batch = {name: EnvField(self.batch_size) for name, _ in LOSS_DICT}
        self.losses_batch = list(self.loss_dict_batch.values())
        self.current_max_height = ScalarField()
        self.robot = Robot(np.asarray(robot["objects"], np.float64), np.asarray(robot["springs"], np.float64),
                           robot_id=self.robot_id, hidden=[self.n_hidden])
        if self.robot.n_vertices != self.n_objects or self.robot.n_springs != self.n_springs:
            raise ValueError("robot.n_objects / n_springs disagree with the robot's arrays")
        if batch is None:
            from .trainer import sim_params
            # two states more than max_steps: an evaluation rollout steps t in
            # [0, max_steps] (diffphy_trainer.py:257-266)
            params = sim_params(cfg, precision, checkpoint_every, max_steps=self.max_steps + 2,
                                keep_trajectory=True)
            batch = MassSpringBatch([self.robot], [0] * self.batch_size, params)
            if stream is not None:
                batch.set_stream(stream)
        self.batch = batch
        self.initial_objects_np = self.robot.objects + np.array([INITIAL_SHIFT_X, 0.0, 0.0])
        self._x0 = np.tile(self.robot.objects, (self.batch_size, 1))
        self._v0 = np.zeros_like(self._x0)
        self._episode = None
        self._ran = None          # (substeps, train) of the last rollout
        self._in_tape = False
        self._loss_ready = False
        self._injected = None
        self._obs = None
        self.solver = SolverMassSpringCUDA(self)
        self.x, self.v = self.solver.x, self.solver.v
        self.center, self.height = self.solver.center, self.solver.height
        self.upper_height, self.rotation = self.solver.upper_height, self.solver.rotation
        self.actuation = self.solver.actuation
        self.input_state = FieldView(self._no_field("input_state"), "input_state")
        self.target_v = FieldView(lambda: self.batch.targets()[0], "target_v")
        self.target_h = FieldView(lambda: self.batch.targets()[1], "target_h")
        self.target_c = FieldView(lambda: self.batch.targets()[2], "target_c")
        # the Tape and the model find the env through these fields
        self.loss._env = self
        self.actuation._env = self

    def close(self):
        self.batch.close()

    # --------------------------------------------------------- field views
    def _no_field(self, name):
        def fetch():
            raise RuntimeError("%s is not kept by the fused CUDA kernels" % name)
        return fetch

    def _x_field(self):
        T, B, N = self.batch.T, self.batch_size, self.n_objects
        return self.batch.trajectory().reshape(T, B, N, 3)

    def _v_field(self):
        """v at t = 0 (the state set by setup / reset / copy) and at the last
        state of the last rollout; other times are not kept."""
        B, N = self.batch_size, self.n_objects
        out = np.full((self.max_steps, B, N, 3), np.nan)
        out[0] = self._v0.reshape(B, N, 3)
        if self._ran is not None:
            out[min(self._ran[0], self.max_steps - 1)] = self.batch.final_state()[1].reshape(B, N, 3)
        return out

    def _observables(self):
        if self._obs is None:
            self._obs = self.batch.observables()
        return self._obs

    # ---------------------------------------------------------- robot state
    def _push_state(self):
        self.batch.set_state(self._x0, self._v0)

    def setup_robot(self):
        """Every env at the robot's objects shifted by +0.4 in x, at rest
        (taichi_env.py:497-504)."""
        self._x0 = np.tile(self.initial_objects_np, (self.batch_size, 1))
        self._v0 = np.zeros_like(self._x0)
        self._push_state()

    def reset_robot(self, start, step, times):
        """x[0] of envs start, start + step, ... back to the initial objects
        (taichi_env.py:487-490; velocities are kept)."""
        N = self.n_objects
        for k in range(times):
            e = k * step + start
            self._x0[e * N:(e + 1) * N] = self.initial_objects_np
        self._push_state()

    def copy_robot(self, steps):
        """x[0], v[0] <- the last state of the previous rollout (the reference
        copies index `steps`, one past a training rollout's last written
        state; the last computed state is carried)."""
        x, v = self.batch.final_state()
        self._x0, self._v0 = x, v
        self._push_state()

    # --------------------------------------------------------------- targets
    def inject_targets(self, target_v, target_h, target_c=None):
        """Targets used instead of the next initialize_train draw (parity
        tests inject the reference's draws; ti.random is time-seeded).
        Arrays of max_steps rows (the reference's fields) are zero-padded to
        the batch's trajectory length."""
        T = self.batch.T

        def pad(a, tail):
            if a is None:
                return None
            a = np.asarray(a, np.float64)
            out = np.zeros((T,) + tail)
            out[:min(T, a.shape[0])] = a[:T]
            return out

        B = self.batch_size
        self._injected = (pad(target_v, (B, 3)), pad(target_h, (B,)), pad(target_c, (B,)))

    def initialize_train(self, iter, steps, max_velocity, max_height):
        if self._injected is not None:
            self.batch.set_targets(*self._injected)
            self._injected = None
            return
        self.batch.initialize_train(int(iter), int(steps), self.seed, float(max_velocity))

    def initialize_script(self, steps, x0, y0, x1, y1, x2, y2, x3, y3):
        """Scripted evaluation targets (taichi_env.py:340-376): 1000-step
        phases of (vx, vz), then height targets -1 and 1; t >= steps keeps
        its targets."""
        tv, th, tc = self.batch.targets()
        phases = [(x0, y0), (x1, y1), (x2, y2), (x3, y3)]
        for t in range(min(int(steps), self.batch.T)):
            ph = t // 1000
            if ph < 4:
                tv[t, :, 0], tv[t, :, 2], th[t] = phases[ph][0], phases[ph][1], 0.0
            else:
                tv[t, :, 0], tv[t, :, 2], th[t] = 0.0, 0.0, (-1.0 if ph == 4 else 1.0)
        self.batch.set_targets(tv, th, tc)

    def initialize_interactive(self, steps, output_v, output_h, output_c):
        """Constant targets for every env (taichi_env.py:333-338)."""
        tv, th, tc = self.batch.targets()
        n = min(int(steps), self.batch.T)
        tv[:n, :, 0], th[:n], tc[:n] = output_v, output_h, output_c
        self.batch.set_targets(tv, th, tc)

    def initialize_validate(self, steps, output_v, output_h, output_c):
        """Per-env constant targets (taichi_env.py:378-383)."""
        tv, th, tc = self.batch.targets()
        n = min(int(steps), self.batch.T)
        tv[:n, :, 0] = np.asarray(output_v, np.float64)[None, :]
        th[:n] = np.asarray(output_h, np.float64)[None, :]
        tc[:n] = np.asarray(output_c, np.float64)[None, :]
        self.batch.set_targets(tv, th, tc)

    # -------------------------------------------------------------- episode
    def _begin(self, steps):
        self._episode = _Episode(steps)
        self._loss_ready = False
        self._obs = None

    def _step(self, name, t):
        if self._episode is None:
            raise RuntimeError("%s(%d) before solver.clear_states(steps)" % (name, t))
        self._episode.call(name, int(t))

    def nn_input(self, t, offset, max_speed, max_height):
        """Recorded: the fused kernels build the controller input in place
        (taichi_env.py:149-183).  `offset` must be 0, the trainer's value."""
        if offset != 0:
            raise NotImplementedError("nn_input offset != 0")
        self._step("nn_input", t)

    def get_loss(self, steps, loss_enable=None, *args, **kwargs):
        """Runs the recorded rollout (t in [0, steps - 2]: training; [0,
        steps]: evaluation) and the loss (taichi_env.py:295-331)."""
        if self._episode is None:
            raise RuntimeError("get_loss before solver.clear_states(steps)")
        n = self._episode.substeps
        steps = int(steps)
        enable = set(self.task if loss_enable is None else loss_enable)
        self.batch.set_loss(enable)
        if n == steps - 1:
            self.batch.forward(steps)
            train = True
        elif n == steps + 1:
            if self._in_tape:
                raise RuntimeError("an evaluation rollout (t in [0, steps]) has no reverse pass")
            self.batch.forward_eval(steps)
            train = False
        else:
            raise RuntimeError("get_loss(%d) after %d substeps: the trainer runs steps - 1 (training) "
                               "or steps + 1 (evaluation)" % (steps, n))
        terms, env = self.batch.loss()
        self.loss[None] = terms["total"]
        for name, slot in LOSS_DICT:
            key = ("velocity", "height", "pose", "rotation", "weight", "actuation", "crawl")[slot - 1]
            self.loss_dict[name][None] = terms[key]
            self.loss_dict_batch[name].arr[:] = env[slot]
        self.loss_batch.arr[:] = env[0]
        self._ran = (n, train)
        self._loss_ready = True
        self._obs = None
        self._episode = None
        return self.loss[None]

    def _tape_enter(self):
        self._in_tape = True
        self._loss_ready = False

    def _tape_exit(self):
        self._in_tape = False
        if not self._loss_ready or not self._ran or not self._ran[1]:
            raise RuntimeError("the Tape closed without a training rollout's loss (env.get_loss)")
        self.batch.backward()


class Tape:
    """ti.ad.Tape(env.loss) for the drop-in env: the rollout recorded inside
    runs its checkpointed reverse pass when the context closes
    (diffphy_trainer.py:246)."""

    def __init__(self, loss, env=None):
        self.env = env if env is not None else getattr(loss, "_env", None)
        if self.env is None:
            raise ValueError("Tape needs the drop-in env's loss field")

    def __enter__(self):
        self.env._tape_enter()
        return self

    def __exit__(self, exc_type, exc, tb):
        if exc_type is None:
            self.env._tape_exit()
        else:
            self.env._in_tape = False
        return False


def patch_tape(ti_module):
    """Route ``ti_module.ad.Tape(loss)`` to ``Tape`` when `loss` belongs to a
    drop-in env; other losses keep the module's own Tape."""
    original = ti_module.ad.Tape

    def tape(loss, *args, **kwargs):
        if getattr(loss, "_env", None) is not None:
            return Tape(loss)
        return original(loss, *args, **kwargs)

    ti_module.ad.Tape = tape
    return original


class WeightField:
    """One of Model's weight fields with a ``grad`` view (nn.py:31-43)."""

    def __init__(self, model, layer, bias):
        self.model, self.layer, self.bias = model, layer, bias
        self.grad = FieldView(self._grad, "grad")

    def _get(self):
        W, b = self.model.env.batch.get_weights(0, self.layer)
        return b if self.bias else W

    def _grad(self):
        gW, gb = self.model.env.batch.get_grads(0, self.layer)
        return gb if self.bias else gW

    def to_numpy(self):
        return self._get()

    def from_numpy(self, value):
        W, b = self.model.env.batch.get_weights(0, self.layer)
        if self.bias:
            b = np.asarray(value, np.float64).reshape(b.shape)
        else:
            W = np.asarray(value, np.float64).reshape(W.shape)
        self.model.env.batch.set_weights(0, self.layer, W, b)

    def fill(self, value):
        self.from_numpy(np.full(self.shape, float(value)))

    def __getitem__(self, key):
        return self._get()[key]

    @property
    def shape(self):
        rows, cols = self.model.env.batch.layer_shape(0, self.layer)
        return (rows,) if self.bias else (rows, cols)


class ModelCUDA:
    """Model's interface (nn.py:79-191) over the env's CUDA batch:
    ``Model(config, steps, batch_size, n_input, n_output, input_field,
    output_field, n_hidden, method)`` with ``output_field`` the drop-in env's
    ``actuation`` (which names the env)."""

    def __init__(self, config, steps, batch_size, n_input, n_output, input_field, output_field, n_hidden,
                 method="adam", env=None):
        self.env = env if env is not None else getattr(output_field, "_env", None)
        if not isinstance(self.env, TaichiEnvCUDA):
            raise ValueError("ModelCUDA needs the drop-in env (pass env= or its actuation field)")
        cfg = _config_dict(config)
        self.steps, self.batch_size = int(steps), int(batch_size)
        self.n_input, self.n_output, self.n_hidden = int(n_input), int(n_output), int(n_hidden)
        if (self.n_hidden, self.n_input) != self.env.batch.layer_shape(0, 0) or \
                (self.n_output, self.n_hidden) != self.env.batch.layer_shape(0, 1):
            raise ValueError("model shape disagrees with the env's controller")
        self.method = method
        if method not in ("adam", "sgd"):
            raise ValueError("optimizer %r" % (method,))
        self.learning_rate = float(cfg["nn"]["learning_rate"])
        self.weights1, self.weights2 = WeightField(self, 0, False), WeightField(self, 1, False)
        self.bias1, self.bias2 = WeightField(self, 0, True), WeightField(self, 1, True)
        self.weights = [self.weights1, self.weights2, self.bias1, self.bias2]
        self.TNS = ScalarField()
        self._init_count = 0

    def clear(self):
        """The fused kernels keep no accumulators between substeps (nn.py:116-121)."""

    def clear_single(self, t):
        """See clear."""

    def clear_adam(self):
        self.env.batch.clear_adam()

    def weights_init(self):
        """W = (2u - 1) sqrt(6 / fan_in) on the device, biases untouched
        (nn.py:59-67); u from (env seed, call count) in place of ti.random."""
        self.env.batch.weights_init(self.env.seed * 1000003 + self._init_count)
        self._init_count += 1

    def forward(self, t):
        self.env._step("forward", t)

    def get_TNS(self):
        """Sum of squared weight gradients (nn.py:173-182)."""
        tns = 0.0
        for l in range(2):
            gW, gb = self.env.batch.get_grads(0, l)
            tns += float((gW * gW).sum() + (gb * gb).sum())
        self.TNS[None] = tns
        return tns

    def gradient_update(self, iter=0):
        """Adam (on the device) or SGD (nn.py:163-171, 184-197)."""
        if self.method == "adam":
            self.env.batch.adam_step(int(iter))
            return
        for l in range(2):
            W, b = self.env.batch.get_weights(0, l)
            gW, gb = self.env.batch.get_grads(0, l)
            self.env.batch.set_weights(0, l, W - gW * self.learning_rate, b - gb * self.learning_rate)

    def dump_weights(self, name="save.pkl"):
        with open(name, "wb") as f:
            pickle.dump([w.to_numpy() for w in self.weights], f)

    def load_weights(self, name="save.pkl"):
        with open(name, "rb") as f:
            vals = pickle.load(f)
        (W1, W2, b1, b2) = [np.asarray(v, np.float64) for v in vals]
        self.env.batch.set_weights(0, 0, W1, b1)
        self.env.batch.set_weights(0, 1, W2, b2)

