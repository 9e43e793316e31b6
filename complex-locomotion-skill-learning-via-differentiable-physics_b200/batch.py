"""Host front-end of the batched mass-spring simulator (``cls_*`` C ABI).

A ``MassSpringBatch`` holds any number of environments of one or more robot
types on one GPU.  Each robot type has its own geometry and its own controller
weights; environments of the same type share the weights, as the reference's
batch shares one ``Model`` (multitask/diffphy_trainer.py:178-185).
"""
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import ctypes
import numpy as np

from . import _capi
from ._capi import check, ptr


@dataclass
class Robot:
    """One robot type: the reference builder's ``objects`` / ``springs`` rows
    ``[a, b, rest_length, stiffness, actuation]`` (robot_design.py:344-349) and
    the controller shape."""
    objects: np.ndarray
    springs: np.ndarray
    robot_id: int = -1
    hidden: Sequence[int] = (64,)
    n_outputs: int = 0                       # 0: one output per spring (reference)
    spring_output: Optional[np.ndarray] = None

    def __post_init__(self):
        self.objects = np.ascontiguousarray(np.asarray(self.objects, np.float64).reshape(-1, 3))
        self.springs = np.ascontiguousarray(np.asarray(self.springs, np.float64).reshape(-1, 5))
        if self.spring_output is not None:
            self.spring_output = np.ascontiguousarray(self.spring_output, dtype=np.int32)

    @property
    def n_vertices(self):
        return self.objects.shape[0]

    @property
    def n_springs(self):
        return self.springs.shape[0]

    @classmethod
    def actuated_outputs(cls, objects, springs, **kw):
        """Controller outputs only for actuated springs (actuation coef > 0)."""
        springs = np.asarray(springs, np.float64).reshape(-1, 5)
        act = springs[:, 4] > 0
        so = np.full(springs.shape[0], -1, dtype=np.int32)
        so[act] = np.arange(int(act.sum()), dtype=np.int32)
        return cls(objects, springs, n_outputs=int(act.sum()), spring_output=so, **kw)


def default_params(**over):
    """Reference defaults (cfg3d/sim_quad.json after ConfigSim) with overrides."""
    p = _capi.SimParams()
    _capi.load().cls_default_params(ctypes.byref(p))
    for k, v in over.items():
        if k in ("activation_hidden", "activation_output") and isinstance(v, str):
            v = _capi.ACT[v]
        if k == "loss" and not isinstance(v, int):
            k, v = "loss_mask", sum(_capi.LOSS_BITS[n] for n in v)
        if k == "precision" and isinstance(v, str):
            v = {"fp32": 32, "fp64": 64, "float32": 32, "float64": 64}[v]
        setattr(p, k, v)
    return p


class MassSpringBatch:
    """A batch of environments advanced by the fused sm_100a segment kernels."""

    def __init__(self, robots: List[Robot], env_robot: Sequence[int], params=None, **over):
        self.lib = _capi.load()
        self.robots = list(robots)
        self.env_robot = np.ascontiguousarray(env_robot, dtype=np.int32)
        self.params = params if params is not None else default_params(**over)
        descs = (_capi.RobotDesc * len(self.robots))()
        self._keep = []
        for d, r in zip(descs, self.robots):
            d.n_vertices = r.n_vertices
            d.n_springs = r.n_springs
            d.objects = ptr(r.objects)
            d.springs = ptr(r.springs)
            d.robot_id = r.robot_id
            d.n_outputs = r.n_outputs
            d.spring_output = ptr(r.spring_output, _capi.P_I)
            d.n_hidden_layers = len(r.hidden)
            for i, h in enumerate(r.hidden):
                d.hidden[i] = h
            self._keep.append(r)
        h = ctypes.c_void_p()
        rc = self.lib.cls_create(descs, len(self.robots), ptr(self.env_robot, _capi.P_I),
                                 len(self.env_robot), ctypes.byref(self.params), ctypes.byref(h))
        check(rc, None)
        self.h = h
        ne, nv, T = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        check(self.lib.cls_get_sizes(self.h, ctypes.byref(ne), ctypes.byref(nv), ctypes.byref(T)), self.h)
        self.n_envs, self.n_vertices_total, self.T = ne.value, nv.value, T.value
        self.env_vertex_offset = np.concatenate(
            [[0], np.cumsum([self.robots[r].n_vertices for r in self.env_robot])]).astype(np.int64)
        self._stream = None

    # -------------------------------------------------------------- lifecycle
    def close(self):
        if getattr(self, "h", None):
            self.lib.cls_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        check(rc, self.h)

    def set_stream(self, stream_handle):
        """Bind to a cudaStream_t (int handle, e.g. torch.cuda.Stream().cuda_stream)."""
        self._stream = stream_handle
        self._c(self.lib.cls_set_stream(self.h, ctypes.c_void_p(stream_handle)))

    def layer_shape(self, robot, layer):
        r, c = ctypes.c_int32(), ctypes.c_int32()
        self._c(self.lib.cls_get_layer_shape(self.h, robot, layer, ctypes.byref(r), ctypes.byref(c)))
        return r.value, c.value

    def n_layers(self, robot=0):
        return len(self.robots[robot].hidden) + 1

    # ------------------------------------------------------------------ inputs
    @staticmethod
    def _f64(a, shape=None):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
        if shape is not None:
            a = a.reshape(shape)
        return a

    def set_state(self, x0, v0=None):
        x0 = self._f64(x0, (self.n_vertices_total, 3))
        v0 = None if v0 is None else self._f64(v0, (self.n_vertices_total, 3))
        self._c(self.lib.cls_set_state(self.h, ptr(x0), ptr(v0)))

    def set_targets(self, target_v, target_h, target_c=None):
        tv = self._f64(target_v, (self.T, self.n_envs, 3))
        th = self._f64(target_h, (self.T, self.n_envs))
        tc = None if target_c is None else self._f64(target_c, (self.T, self.n_envs))
        self._c(self.lib.cls_set_targets(self.h, ptr(tv), ptr(th), ptr(tc)))

    def set_weights(self, robot, layer, W, b):
        rows, cols = self.layer_shape(robot, layer)
        W = None if W is None else self._f64(W, (rows, cols))
        b = None if b is None else self._f64(b, (rows,))
        self._c(self.lib.cls_set_weights(self.h, robot, layer, ptr(W), ptr(b)))

    def get_weights(self, robot, layer):
        rows, cols = self.layer_shape(robot, layer)
        W, b = np.zeros((rows, cols)), np.zeros(rows)
        self._c(self.lib.cls_get_weights(self.h, robot, layer, ptr(W), ptr(b)))
        return W, b

    def get_grads(self, robot, layer):
        rows, cols = self.layer_shape(robot, layer)
        W, b = np.zeros((rows, cols)), np.zeros(rows)
        self._c(self.lib.cls_get_grads(self.h, robot, layer, ptr(W), ptr(b)))
        return W, b

    # ------------------------------------------------------------------ passes
    def forward(self, steps):
        self._c(self.lib.cls_forward(self.h, steps))

    def forward_eval(self, steps):
        self._c(self.lib.cls_forward_eval(self.h, steps))

    def loss(self):
        terms = np.zeros(8)
        env = np.zeros((8, self.n_envs))
        self._c(self.lib.cls_loss(self.h, ptr(terms), ptr(env)))
        return dict(zip(_capi.LOSS_SLOTS, terms.tolist())), env

    def set_loss(self, names):
        """Losses of the following rollouts, by name or CLS_LOSS_* mask
        (``cls_set_loss_mask``); the loss set passed to get_loss."""
        mask = names if isinstance(names, int) else sum(_capi.LOSS_BITS[n] for n in set(names))
        self._c(self.lib.cls_set_loss_mask(self.h, int(mask)))

    def set_loss_envs(self, robot, n_envs):
        """The env count robot type `robot`'s losses are divided by (default:
        this batch's count of the type; ``cls_set_loss_envs``)."""
        self._c(self.lib.cls_set_loss_envs(self.h, int(robot), int(n_envs)))

    def backward(self):
        self._c(self.lib.cls_backward(self.h))

    def simulate(self, steps, per_env=False):
        out = ctypes.c_double()
        fn = self.lib.cls_simulate_per_env if per_env else self.lib.cls_simulate
        self._c(fn(self.h, steps, ctypes.byref(out)))
        return out.value

    # ----------------------------------------------------------------- serving
    def serve_reset_env(self, env, x0, v0=None, target_v=None, target_h=None, target_c=None):
        """Restart env `env` with its own initial state and targets (one env's
        [T] columns); other envs are untouched."""
        n = self.robots[self.env_robot[env]].n_vertices
        x0 = self._f64(x0, (n, 3))
        v0 = None if v0 is None else self._f64(v0, (n, 3))
        tv = None if target_v is None else self._f64(target_v, (self.T, 3))
        th = None if target_h is None else self._f64(target_h, (self.T,))
        tc = None if target_c is None else self._f64(target_c, (self.T,))
        self._c(self.lib.cls_serve_reset_env(self.h, env, ptr(x0), ptr(v0), ptr(tv), ptr(th), ptr(tc)))

    @staticmethod
    def _i32(a, shape):
        return np.ascontiguousarray(np.asarray(a, dtype=np.int32).reshape(shape))

    def serve_forward(self, windows, steps):
        w, s = self._i32(windows, (self.n_envs, 4)), self._i32(steps, (self.n_envs,))
        self._c(self.lib.cls_serve_forward(self.h, ptr(w, _capi.P_I), ptr(s, _capi.P_I)))

    def serve_backward(self, windows, steps):
        w, s = self._i32(windows, (self.n_envs, 4)), self._i32(steps, (self.n_envs,))
        self._c(self.lib.cls_serve_backward(self.h, ptr(w, _capi.P_I), ptr(s, _capi.P_I)))

    def serve_loss(self, steps):
        s = self._i32(steps, (self.n_envs,))
        env = np.zeros((8, self.n_envs))
        self._c(self.lib.cls_serve_loss(self.h, ptr(s, _capi.P_I), ptr(env)))
        return env

    def serve_env_state(self, env):
        n = self.robots[self.env_robot[env]].n_vertices
        x, v = np.zeros((n, 3)), np.zeros((n, 3))
        self._c(self.lib.cls_serve_env_state(self.h, env, ptr(x), ptr(v)))
        return x, v

    # the library's own admission / poll loop over the envs as slots
    def serve_tick(self, tick_segments):
        self._c(self.lib.cls_serve_tick(self.h, int(tick_segments)))

    def admit(self, rid, robot, steps, grad=False, x0=None, target_v=None, target_h=None, target_c=None,
              budget=-1):
        """Admit request `rid` on a free slot of slot `robot`'s robot class;
        returns the slot, or -1 (no free slot, or its footprint does not fit
        `budget` bytes)."""
        slot = ctypes.c_int32(-1)
        n = self.robots[self.env_robot[robot]].n_vertices
        keep = [None if x0 is None else self._f64(x0, (n, 3)),
                None if target_v is None else self._f64(target_v, (self.T, 3)),
                None if target_h is None else self._f64(target_h, (self.T,)),
                None if target_c is None else self._f64(target_c, (self.T,))]
        req = _capi.Request(int(rid), int(robot), int(steps), 1 if grad else 0, *[ptr(a) for a in keep])
        self._c(self.lib.cls_admit(self.h, ctypes.byref(req), int(budget), ctypes.byref(slot)))
        return slot.value

    def poll(self, capacity=64):
        """Complete the tick in flight and issue the next; returns (ids of
        finished requests, slots still running)."""
        ids = (ctypes.c_uint64 * max(1, capacity))()
        n_done, n_active = ctypes.c_int32(), ctypes.c_int32()
        self._c(self.lib.cls_poll(self.h, ids, int(capacity), ctypes.byref(n_done), ctypes.byref(n_active)))
        return [int(ids[k]) for k in range(n_done.value)], n_active.value

    def serve_result(self, rid):
        """(slot, loss terms [8], final positions [n_v][3]) of a finished request."""
        slot = ctypes.c_int32()
        self._c(self.lib.cls_serve_result(self.h, int(rid), ctypes.byref(slot), None, None))
        n = self.robots[self.env_robot[slot.value]].n_vertices
        terms, x = np.zeros(8), np.zeros((n, 3))
        self._c(self.lib.cls_serve_result(self.h, int(rid), ctypes.byref(slot), ptr(terms), ptr(x)))
        return slot.value, terms, x

    def serve_release(self, rid):
        self._c(self.lib.cls_serve_release(self.h, int(rid)))

    def adam_step(self, it):
        tns = ctypes.c_double()
        self._c(self.lib.cls_adam_step(self.h, it, ctypes.byref(tns)))
        return tns.value

    def clear_adam(self):
        self._c(self.lib.cls_clear_adam(self.h))

    def weights_init(self, seed):
        self._c(self.lib.cls_weights_init(self.h, seed))

    def initialize_train(self, it, steps, seed, max_speed):
        self._c(self.lib.cls_initialize_train(self.h, it, steps, seed, max_speed))

    def profile(self, on=True):
        self._c(self.lib.cls_profile_enable(self.h, 1 if on else 0))

    def profile_read(self, reset=False):
        ms = np.zeros(len(_capi.PROFILE_KINDS))
        n = np.zeros(len(_capi.PROFILE_KINDS), dtype=np.int64)
        self._c(self.lib.cls_profile_read(self.h, ptr(ms), n.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                          1 if reset else 0))
        return dict(zip(_capi.PROFILE_KINDS, ms.tolist())), dict(zip(_capi.PROFILE_KINDS, n.tolist()))

    def synchronize(self):
        self._c(self.lib.cls_synchronize(self.h))

    def graph_capture(self, steps, with_adam=False):
        self._c(self.lib.cls_graph_capture(self.h, steps, 1 if with_adam else 0))

    def graph_launch(self, it=0):
        self._c(self.lib.cls_graph_launch(self.h, it))

    CONTROLLER_PATHS = {"auto": 0, "per_env": 1, "batched": 2}

    def set_controller_path(self, path):
        """'auto' (batched when every robot type has >= 256 envs), 'per_env'
        (the controller inside the fused segment kernels) or 'batched' (one
        tensor-core GEMM per layer over all envs of a type)."""
        self._c(self.lib.cls_set_controller_path(self.h, self.CONTROLLER_PATHS[path]))

    @property
    def controller_batched(self):
        on = np.zeros(1, dtype=np.int32)
        self._c(self.lib.cls_controller_batched(self.h, on.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        return bool(on[0])

    # ------------------------------------------------------------ launch shape
    def set_launch_shape(self, threads_per_block, ctas_per_sm=2, weights_shared=-1):
        """Threads per CTA of the fused segment kernels, the CTAs per SM the
        persistent grid is sized for, and whether each env's controller is
        kept in shared memory (1), read from global memory (0) or chosen by
        fit (-1) (``cls_set_launch_shape``)."""
        self._c(self.lib.cls_set_launch_shape(self.h, int(threads_per_block), int(ctas_per_sm),
                                              int(weights_shared)))

    @property
    def launch_shape(self):
        """(threads per CTA, CTAs per SM, controller in shared memory 0/1)."""
        t, c, w = (np.zeros(1, dtype=np.int32) for _ in range(3))
        self._c(self.lib.cls_get_launch_shape(self.h, ptr(t, _capi.P_I), ptr(c, _capi.P_I),
                                              ptr(w, _capi.P_I)))
        return int(t[0]), int(c[0]), int(w[0])

    def set_spring_tables(self, mode=-1):
        """Per-spring tables in shared memory: -1 when they fit (default), 0
        off (direct gathers from both endpoints), 1 on (``cls_set_spring_tables``)."""
        self._c(self.lib.cls_set_spring_tables(self.h, int(mode)))

    @property
    def spring_tables(self):
        on = np.zeros(1, dtype=np.int32)
        self._c(self.lib.cls_spring_tables(self.h, ptr(on, _capi.P_I)))
        return bool(on[0])

    def _tune_key(self, steps):
        import hashlib
        import json
        try:
            import torch
            device = torch.cuda.get_device_name(torch.cuda.current_device())
        except Exception:                                    # no torch: key on the rest
            device = "cuda"
        counts = np.bincount(self.env_robot, minlength=len(self.robots))
        sig = {"device": device, "precision": int(self.params.precision),
               "K": int(self.params.checkpoint_every), "T": int(self.T), "steps": int(steps),
               "types": [[r.n_vertices, r.n_springs, list(map(int, r.hidden)), int(r.n_outputs),
                          int(n)] for r, n in zip(self.robots, counts)]}
        return hashlib.sha1(json.dumps(sig, sort_keys=True).encode()).hexdigest()

    def autotune(self, steps=0, repeats=2, cache=None):
        """Time the fused kernels' launch shapes (threads per CTA x CTAs per SM)
        and, for robot types with many envs, the batched controller path on this
        batch's own workload, and apply the fastest (``cls_autotune``).  Needs
        the state, targets and weights set.  ``cache``: path of a JSON file; a
        workload tuned before (same device, robot shapes, env counts,
        precision, K, horizon) is applied from it without timing.  Returns
        ``{"threads_per_block", "ctas_per_sm", "weights_shared",
        "controller_path", "table", "cached"}``."""
        import json
        import os
        key = self._tune_key(steps)
        if cache and os.path.exists(cache):
            with open(cache) as f:
                hit = json.load(f).get(key)
            if hit:
                self.set_controller_path(hit["controller_path"])
                self.set_launch_shape(hit["threads_per_block"], hit["ctas_per_sm"], hit["weights_shared"])
                return dict(hit, cached=True)
        cap = 64
        table = (_capi.LaunchShape * cap)()
        n = np.zeros(1, dtype=np.int32)
        self._c(self.lib.cls_autotune(self.h, int(steps), int(repeats), table, cap, ptr(n, _capi.P_I)))
        names = {v: k for k, v in self.CONTROLLER_PATHS.items()}
        rows = [{"controller_path": names[e.controller_path], "threads_per_block": e.threads_per_block,
                 "ctas_per_sm": e.ctas_per_sm, "weights_shared": e.weights_shared, "ms": float(e.ms)}
                for e in table[:min(int(n[0]), cap)]]
        t, c, w = self.launch_shape
        out = {"threads_per_block": t, "ctas_per_sm": c, "weights_shared": w,
               "controller_path": "batched" if self.controller_batched else "per_env", "table": rows}
        if cache:
            data = {}
            if os.path.exists(cache):
                with open(cache) as f:
                    data = json.load(f)
            data[key] = out
            os.makedirs(os.path.dirname(os.path.abspath(cache)), exist_ok=True)
            tmp = cache + ".tmp"
            with open(tmp, "w") as f:
                json.dump(data, f, indent=1)
            os.replace(tmp, cache)
        return dict(out, cached=False)

    # ----------------------------------------------------------------- outputs
    def observables(self):
        T, E = self.T, self.n_envs
        c, h, u, r = np.zeros((T, E, 3)), np.zeros((T, E)), np.zeros((T, E)), np.zeros((T, E))
        self._c(self.lib.cls_get_observables(self.h, ptr(c), ptr(h), ptr(u), ptr(r)))
        return dict(center=c, height=h, upper_height=u, rotation=r)

    def targets(self):
        """(target_v [T][E][3], target_h [T][E], target_c [T][E]) as the
        device holds them (after set_targets or initialize_train)."""
        T, E = self.T, self.n_envs
        tv, th, tc = np.zeros((T, E, 3)), np.zeros((T, E)), np.zeros((T, E))
        self._c(self.lib.cls_get_targets(self.h, ptr(tv), ptr(th), ptr(tc)))
        return tv, th, tc

    def trajectory(self):
        x = np.zeros((self.T, self.n_vertices_total, 3))
        self._c(self.lib.cls_get_trajectory(self.h, ptr(x)))
        return x

    def final_state(self):
        x, v = np.zeros((self.n_vertices_total, 3)), np.zeros((self.n_vertices_total, 3))
        self._c(self.lib.cls_get_final_state(self.h, ptr(x), ptr(v)))
        return x, v

    def state_grads(self):
        gx, gv = np.zeros((self.n_vertices_total, 3)), np.zeros((self.n_vertices_total, 3))
        self._c(self.lib.cls_get_state_grads(self.h, ptr(gx), ptr(gv)))
        return gx, gv

    def env_slice(self, e):
        """Rows of the packed [n_vertices_total] arrays that belong to env e."""
        return slice(int(self.env_vertex_offset[e]), int(self.env_vertex_offset[e + 1]))
