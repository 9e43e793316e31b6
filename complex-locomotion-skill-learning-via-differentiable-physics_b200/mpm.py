"""Host front-end of the differentiable MLS-MPM solver (``cls_mpm_*`` C ABI).

Replaces the reference's SolverMPM (multitask/solver_mpm.py): a batch of
``n_envs`` copies of one particle body, stepped by advance_core (clear_grid,
p2g, grid_op, g2p) with a checkpointed reverse pass.
"""
import ctypes

import numpy as np

from . import _capi

_i32, _d = ctypes.c_int32, ctypes.c_double
P_D = _capi.P_D
MATERIAL = {"fixed_corotated": 0, "neo_hookean": 1}


class MPMBody(ctypes.Structure):
    _fields_ = [("dim", _i32), ("n_particles", _i32), ("positions", P_D),
                ("muscle", _capi.P_I), ("fibre", P_D), ("n_muscles", _i32)]


class MPMParams(ctypes.Structure):
    _fields_ = [("max_steps", _i32), ("n_grid", _i32), ("bound", _i32), ("material", _i32),
                ("precision", _i32), ("checkpoint_every", _i32), ("dt", _d), ("gravity", _d),
                ("p_vol", _d), ("mu", _d), ("la", _d), ("act_strength", _d), ("mass", _d),
                ("tile_nodes", _i32), ("particle_order", _i32)]
PARTICLE_ORDER = {"cells": 0, "base_runs": 1}


_SIGS = {
    "cls_mpm_default_params": (None, [ctypes.POINTER(MPMParams)]),
    "cls_mpm_create": (_i32, [ctypes.POINTER(MPMBody), ctypes.POINTER(MPMParams), _i32,
                              ctypes.POINTER(ctypes.c_void_p)]),
    "cls_mpm_destroy": (_i32, [ctypes.c_void_p]),
    "cls_mpm_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "cls_mpm_set_stream": (_i32, [ctypes.c_void_p, ctypes.c_void_p]),
    "cls_mpm_set_state": (_i32, [ctypes.c_void_p, P_D, P_D]),
    "cls_mpm_set_actuation": (_i32, [ctypes.c_void_p, P_D]),
    "cls_mpm_set_loss": (_i32, [ctypes.c_void_p, P_D, P_D, P_D]),
    "cls_mpm_forward": (_i32, [ctypes.c_void_p, _i32]),
    "cls_mpm_loss": (_i32, [ctypes.c_void_p, P_D]),
    "cls_mpm_backward": (_i32, [ctypes.c_void_p]),
    "cls_mpm_get_final_state": (_i32, [ctypes.c_void_p, P_D, P_D, P_D, P_D]),
    "cls_mpm_get_grads": (_i32, [ctypes.c_void_p, P_D, P_D, P_D, P_D, P_D]),
    "cls_mpm_get_centers": (_i32, [ctypes.c_void_p, P_D]),
    "cls_mpm_graph_capture": (_i32, [ctypes.c_void_p, _i32]),
    "cls_mpm_graph_launch": (_i32, [ctypes.c_void_p]),
    "cls_mpm_profile_enable": (_i32, [ctypes.c_void_p, _i32]),
    "cls_mpm_profile_read": (_i32, [ctypes.c_void_p, P_D, ctypes.POINTER(ctypes.c_int64), _i32]),
    "cls_mpm_reduction_peak": (_i32, [ctypes.c_int64, ctypes.c_int64, P_D]),
}

# categories of cls_mpm_profile_read
PROFILE_KINDS = ["particle", "particle_recompute", "grid", "particle_adj", "grid_adj", "other"]


def _lib():
    lib = _capi.load()
    if not getattr(lib, "_mpm_bound", False):
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        lib._mpm_bound = True
    return lib


def reduction_peak(n_nodes, n_ops=1 << 27):
    """Measured rate (operations/s) of 16-byte vector reductions into an
    n_nodes-node buffer (cls_mpm_reduction_peak)."""
    out = ctypes.c_double()
    rc = _lib().cls_mpm_reduction_peak(int(n_nodes), int(n_ops), ctypes.byref(out))
    if rc != 0:
        raise _capi.ClsError("cls_mpm_reduction_peak failed (%d)" % rc, rc)
    return out.value


def default_params(**over):
    p = MPMParams()
    _lib().cls_mpm_default_params(ctypes.byref(p))
    for k, v in over.items():
        if k == "material" and isinstance(v, str):
            v = MATERIAL[v]
        if k == "particle_order" and isinstance(v, str):
            v = PARTICLE_ORDER[v]
        setattr(p, k, v)
    return p


def _f64(a, shape):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(shape))


class MPMBatch:
    def __init__(self, positions, muscle, n_envs, *, dim, fibre=None, n_muscles=None,
                 params=None, **over):
        self.lib = _lib()
        self.dim = dim
        self.positions = _f64(positions, (-1, dim))
        self.P = self.positions.shape[0]
        self.muscle = np.ascontiguousarray(muscle, dtype=np.int32)
        self.M = int(n_muscles if n_muscles is not None else max(1, self.muscle.max() + 1))
        self.fibre = None if fibre is None else _f64(fibre, (self.P, dim))
        self.params = params if params is not None else default_params(**over)
        self.E = n_envs
        self.T = self.params.max_steps
        body = MPMBody(dim, self.P, _capi.ptr(self.positions), _capi.ptr(self.muscle, _capi.P_I),
                       _capi.ptr(self.fibre), self.M)
        h = ctypes.c_void_p()
        rc = self.lib.cls_mpm_create(ctypes.byref(body), ctypes.byref(self.params), n_envs,
                                     ctypes.byref(h))
        self._check(rc, None)
        self.h = h

    def _check(self, rc, h):
        if rc != 0:
            msg = self.lib.cls_mpm_last_error(h)
            raise _capi.ClsError("%s (%d): %s" % (_capi.ERRORS.get(rc, "error"), rc,
                                                   msg.decode() if msg else ""))

    def _c(self, rc):
        self._check(rc, self.h)

    def close(self):
        if getattr(self, "h", None):
            self.lib.cls_mpm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, s):
        self._c(self.lib.cls_mpm_set_stream(self.h, ctypes.c_void_p(s)))

    def set_state(self, x0, v0=None):
        x0 = _f64(x0, (self.E, self.P, self.dim))
        v0 = None if v0 is None else _f64(v0, (self.E, self.P, self.dim))
        self._c(self.lib.cls_mpm_set_state(self.h, _capi.ptr(x0), _capi.ptr(v0)))

    def set_actuation(self, act):
        self._c(self.lib.cls_mpm_set_actuation(self.h, _capi.ptr(_f64(act, (self.T, self.E, self.M)))))

    def set_loss(self, w=None, target=None, particle_weights=None):
        w = None if w is None else _f64(w, (self.T + 1,))
        t = None if target is None else _f64(target, (self.T + 1, self.E, self.dim))
        pw = None if particle_weights is None else _f64(particle_weights, (self.P,))
        self._c(self.lib.cls_mpm_set_loss(self.h, _capi.ptr(w), _capi.ptr(t), _capi.ptr(pw)))

    def forward(self, steps):
        self._c(self.lib.cls_mpm_forward(self.h, steps))

    def loss(self):
        out = ctypes.c_double()
        self._c(self.lib.cls_mpm_loss(self.h, ctypes.byref(out)))
        return out.value

    def backward(self):
        self._c(self.lib.cls_mpm_backward(self.h))

    def run(self, steps):
        self.forward(steps)
        L = self.loss()
        self.backward()
        return L

    def final_state(self):
        E, P, D = self.E, self.P, self.dim
        x, v = np.zeros((E, P, D)), np.zeros((E, P, D))
        C, F = np.zeros((E, P, D, D)), np.zeros((E, P, D, D))
        self._c(self.lib.cls_mpm_get_final_state(self.h, _capi.ptr(x), _capi.ptr(v),
                                                 _capi.ptr(C), _capi.ptr(F)))
        return x, v, C, F

    def grads(self):
        E, P, D = self.E, self.P, self.dim
        ga = np.zeros((self.T, E, self.M))
        gx, gv = np.zeros((E, P, D)), np.zeros((E, P, D))
        gC, gF = np.zeros((E, P, D, D)), np.zeros((E, P, D, D))
        self._c(self.lib.cls_mpm_get_grads(self.h, _capi.ptr(ga), _capi.ptr(gx), _capi.ptr(gv),
                                           _capi.ptr(gC), _capi.ptr(gF)))
        return dict(act=ga, x0=gx, v0=gv, C0=gC, F0=gF)

    def centers(self):
        c = np.zeros((self.T + 1, self.E, self.dim))
        self._c(self.lib.cls_mpm_get_centers(self.h, _capi.ptr(c)))
        return c

    def graph_capture(self, steps):
        self._c(self.lib.cls_mpm_graph_capture(self.h, steps))

    def graph_launch(self):
        self._c(self.lib.cls_mpm_graph_launch(self.h))

    def profile(self, on=True):
        self._c(self.lib.cls_mpm_profile_enable(self.h, 1 if on else 0))

    def profile_read(self, reset=False):
        """Per-category device milliseconds and launch counts since the last reset."""
        n = len(PROFILE_KINDS)
        ms = np.zeros(n)
        cnt = np.zeros(n, dtype=np.int64)
        self._c(self.lib.cls_mpm_profile_read(self.h, _capi.ptr(ms),
                                              cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                              1 if reset else 0))
        return dict(zip(PROFILE_KINDS, ms.tolist())), dict(zip(PROFILE_KINDS, cnt.tolist()))
