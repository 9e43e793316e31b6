"""Headless clients of the simulator for the reference's two interactive
entry points, with the state resident on the device.

* ``MassSpringEnvCUDA`` -- the gym environment of
  multitask/mass_spring_env.py:15-219 for an external policy (reinforcement
  learning): ``reset()`` returns the observation of t = 0, ``step(action)``
  applies the actions to the actuated springs of every env
  (``pass_actuation``), advances one substep and returns ``(observation,
  reward, done, info)`` with the reference's reward (``get_reward``,
  :105-135) and its observation clipping (``get_state``, :141-150).  One
  ``cls_env_step`` launch per step.  Rendering / video output is graphics and
  not built; ``gym`` is optional (``action_space`` / ``observation_space``
  are ``gym.spaces.Box`` when it is installed, else (low, high) pairs).
* ``InteractiveSession`` -- the loop of interactive_3d.py:38-74 (set target
  -> make_decision with the embedded controller -> substeps -> refresh) as
  frames of ``frame_substeps`` substeps of one env's running episode
  (``cls_serve_forward`` windows) whose goal can change between frames
  (``cls_serve_set_targets``); GGUI drawing is replaced by returning the
  vertex positions of the frame.  When the episode reaches max_steps it
  continues from its last state as a new episode; the controller's sine
  inputs keep their phase when max_steps is a multiple of run_period.
"""
import numpy as np

from .batch import MassSpringBatch


class MassSpringEnvCUDA:
    """MassSpringEnv (multitask/mass_spring_env.py) over a CUDA batch of
    ``batch_size`` envs of one robot.  ``robot``: a batch.Robot; ``params``:
    batch.default_params of the episode (max_steps, max_speed, ...).
    ``act_spring``: the springs an action drives (default: actuated
    springs, coefficient > 0, the reference's act_list,
    solver_mass_spring.py:58-67)."""

    def __init__(self, robot, batch_size, params, training=True, interactive=False, seed=0,
                 initial_objects=None):
        self.robot = robot
        self.batch_size = int(batch_size)
        self.params = params
        self.batch = MassSpringBatch([robot], [0] * self.batch_size, params)
        self.max_steps = int(params.max_steps)
        self.rollout_length = self.max_steps
        self.max_speed, self.max_height = float(params.max_speed), float(params.max_height)
        self.turn_period = int(params.turn_period)
        self.training, self.interactive, self.seed = training, interactive, int(seed)
        self.act_spring = np.nonzero(robot.springs[:, 4] > 0)[0].astype(np.int64)
        n_out = robot.n_outputs if robot.n_outputs > 0 else robot.n_springs
        self.n_outputs = n_out
        self.spring_output = (np.arange(robot.n_springs) if robot.spring_output is None
                              else robot.spring_output)
        self.n_input_states = self.batch.layer_shape(0, 0)[1]
        self.x0 = np.asarray(robot.objects if initial_objects is None else initial_objects, np.float64)
        self.t = 0
        self.rollout_times = 0
        self.last_height = [0.1] * self.batch_size
        self.reward_v, self.reward_h = [], []
        self.center = np.zeros((self.max_steps, self.batch_size, 3))
        self.height = np.zeros((self.max_steps, self.batch_size))
        self._obs = None
        self.tv = np.zeros((self.max_steps, self.batch_size, 3))
        self.th = np.zeros((self.max_steps, self.batch_size))
        self.tc = np.zeros((self.max_steps, self.batch_size))
        max_act = np.ones(self.batch_size * len(self.act_spring))
        max_obs = np.ones(self.batch_size * self.n_input_states)
        try:
            from gym import spaces
            self.action_space = spaces.Box(-max_act, max_act)
            self.observation_space = spaces.Box(-max_obs, max_obs)
        except ImportError:
            self.action_space = (-max_act, max_act)
            self.observation_space = (-max_obs, max_obs)

    def close(self):
        self.batch.close()

    # ------------------------------------------------------------- targets
    def _push_targets(self):
        self.batch.set_targets(self.tv, self.th, self.tc)

    def initialize_targets(self, validate_v=0.0, validate_h=0.1):
        """Training: the device's task sampler (TaichiEnv.initialize_train);
        otherwise constant validation targets (initialize_validate)."""
        if self.training:
            self.batch.initialize_train(0, self.rollout_length, self.seed, self.max_speed)
            self.tv, self.th, self.tc = self.batch.targets()
        else:
            n = self.rollout_length
            self.tv[:n, :, 0] = validate_v
            self.th[:n] = validate_h
            self.tc[:n] = 0.0
            self._push_targets()

    def set_targets(self, target_v, target_h, target_c):
        """Constant targets for t < self.t + 2 (mass_spring_env.py:187-190,
        initialize_interactive)."""
        if self.t + 2 <= self.max_steps:
            n = self.t + 2
            self.tv[:n, :, 0], self.th[:n], self.tc[:n] = target_v, target_h, target_c
            self._push_targets()

    # ------------------------------------------------------------ episode
    def _outputs(self, action):
        """Controller-output rows of every env from the actions of the
        actuated springs: the reference passes action[i] to spring
        act_spring[i] of every env (mass_spring_env.py:56-58); an action of
        batch_size x n_act values gives each env its own row."""
        a = np.asarray(action, np.float64).ravel()
        n_act = len(self.act_spring)
        rows = a.reshape(-1, n_act)
        if rows.shape[0] not in (1, self.batch_size):
            raise ValueError("action must hold n_act or batch_size x n_act values")
        rows = np.broadcast_to(rows, (self.batch_size, n_act))
        out = np.zeros((self.batch_size, self.n_outputs))
        out[:, self.spring_output[self.act_spring]] = rows
        return out

    def _observe(self, obs, ch):
        self._obs = obs.reshape(self.batch_size, -1)[:, :self.n_input_states].copy()
        ch = ch.reshape(self.batch_size, 4)
        self.center[self.t] = ch[:, :3]
        self.height[self.t] = ch[:, 3]

    def _call(self, outputs):
        B = self.batch_size
        obs = np.zeros(B * self.n_input_states)
        ch = np.zeros(B * 4)
        from ._capi import ptr
        self.batch._c(self.batch.lib.cls_env_step(self.batch.h, self.t, ptr(outputs), ptr(obs), ptr(ch)))
        return obs, ch

    def reset(self):
        """Back to the initial state at t = 0 (mass_spring_env.py:201-224)."""
        if not self.interactive:
            self.initialize_targets()
        self.t = 0
        self.rollout_times += 1
        self.last_height = [0.1] * self.batch_size
        self.batch.set_state(np.tile(self.x0, (self.batch_size, 1)))
        self.center[:] = 0.0
        self.height[:] = 0.0
        self._observe(*self._call(None))
        return self.get_state(self.t)

    def step(self, action):
        if self._obs is None:
            raise RuntimeError("reset() first: the state on the device is set by reset")
        if self.t + 1 >= self.max_steps:
            raise RuntimeError("the rollout is over (t = %d); reset()" % self.t)
        outputs = np.ascontiguousarray(self._outputs(action))
        self.t += 1
        self._observe(*self._call(outputs))
        observation = self.get_state(self.t)
        if self.t % 500 == 0:
            self.last_height = [0.1] * self.batch_size
        reward = 0.0
        if self.t == 1:
            self.reward_h, self.reward_v = [], []
        if not self.interactive:
            reward, reward_v, reward_h = self.get_reward()
            self.reward_v.append(reward_v)
            self.reward_h.append(reward_h)
        done = self.t == self.rollout_length - 1
        return observation, reward, done, {}

    def get_state(self, t=None, clip=True):
        """The observation rows of every env, flattened; clipped to [-1, 1]
        as the reference does (mass_spring_env.py:141-150) unless clip is
        False."""
        s = self._obs.ravel()
        return np.clip(s, -1.0, 1.0) if clip else s.copy()

    def get_reward(self):
        """mass_spring_env.py:105-135: velocity reward over the last 100
        substeps of the turn period and the height reward, averaged over the
        batch; returns (reward, reward_v, reward_h)."""
        B, t = self.batch_size, self.t
        reward = np.zeros(B)
        reward_v = np.zeros(B)
        reward_h = np.zeros(B)
        d = t // 500 * 500
        for k in range(B):
            target_v = self.tv[t, k, 0]
            target_h = self.th[t, k]
            post = self.center[t, k, 0]
            post_ = self.center[t - 1, k, 0]
            for i in range(max(t - 100, d), t):
                tar = self.center[i, k, 0] + target_v
                pre_r = -(post_ - tar) ** 2
                now_r = -(post - tar) ** 2
                reward_v[k] += (now_r - pre_r) / (self.max_speed ** 2) / 400.
            height = self.height[t, k]
            d_reward = ((height - target_h) ** 2 - (self.last_height[k] - target_h) ** 2) / (target_h ** 2) * 10.0
            reward_h[k] -= d_reward
            if height > self.last_height[k]:
                self.last_height[k] = height
            reward[k] += reward_v[k] + reward_h[k]
        return sum(reward) / B, sum(reward_v) / B, sum(reward_h) / B


class InteractiveSession:
    """interactive_3d.py's control loop for one robot with the embedded
    controller (weights [(W, b) per layer]); ``params.checkpoint_every`` is
    the frame length (the reference advances 10 substeps per drawn frame)."""

    def __init__(self, robot, weights, params, x0=None, target=(0.0, 0.1, 0.0)):
        self.robot = robot
        self.params = params
        self.batch = MassSpringBatch([robot], [0], params)
        for l, (W, b) in enumerate(weights):
            self.batch.set_weights(0, l, W, b)
        self.T = int(params.max_steps)
        self.K = int(params.checkpoint_every)
        if self.T % self.K:
            raise ValueError("max_steps must be a multiple of the frame length (checkpoint_every)")
        self.frames_per_episode = (self.T - 1) // self.K
        self.target = tuple(float(v) for v in target)
        self.t = 0
        self.episodes = 0
        self._start(np.asarray(robot.objects if x0 is None else x0, np.float64), None)

    def close(self):
        self.batch.close()

    def _columns(self, n):
        v, h, c = self.target
        tv = np.zeros((n, 3))
        tv[:, 0] = v
        return tv, np.full(n, h), np.full(n, c)

    def _start(self, x, v):
        tv, th, tc = self._columns(self.T)
        self.batch.serve_reset_env(0, x, v, tv, th, tc)
        self.t = 0
        self.episodes += 1

    def set_target(self, target_v=None, target_h=None, target_c=None):
        """A new goal from the next substep on (set_target's key handling,
        interactive_3d.py:13-28)."""
        v, h, c = self.target
        self.target = (v if target_v is None else float(target_v), h if target_h is None else float(target_h),
                       c if target_c is None else float(target_c))
        tv, th, tc = self._columns(self.T - self.t)
        from ._capi import ptr
        self.batch._c(self.batch.lib.cls_serve_set_targets(self.batch.h, 0, self.t, ptr(tv), ptr(th), ptr(tc)))

    def step_frame(self):
        """Advances one frame (frame_substeps substeps of controller and
        physics); returns the vertex positions after it ([n_v][3])."""
        if self.t + self.K > self.T - 1:
            x, v = self.batch.serve_env_state(0)
            self._start(x, v)
        win = np.array([[self.t, self.t + self.K, self.t // self.K, 0]], dtype=np.int32)
        self.batch.serve_forward(win, np.array([self.T], dtype=np.int32))
        self.t += self.K
        return self.batch.serve_env_state(0)[0]

    def state(self):
        return self.batch.serve_env_state(0)
