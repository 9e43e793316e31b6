"""ctypes front-end of the FP64 CPU oracle (``ms_oracle.c``).

TEST INFRASTRUCTURE ONLY: used by tests/, by ``__graft_entry__.smoke()`` as the
checker and by ``bench.py``'s CPU-baseline leg.  The product never imports it.

``MassSpringOracle`` owns full-trajectory NumPy fields laid out like the
reference's Taichi fields (``[t][env][i]``) and exposes the reference's
training rollout: ``forward`` (multitask/diffphy_trainer.py:231-255),
``loss`` (multitask/taichi_env.py:304-331) and ``backward`` (the
``ti.ad.Tape`` reverse pass, written by hand in ms_oracle.c).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
MAX_LAYERS = 5
ACT = {"sin": 0, "tanh": 1}
LOSS_BITS = {"velocity": 1, "height": 2, "pose": 4, "actuation": 8,
             "rotation": 16, "crawl": 32}
LOSS_SLOTS = ("total", "velocity", "height", "pose", "rotation", "weight",
              "actuation", "crawl")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


class _OrcMS(ctypes.Structure):
    _fields_ = [
        ("B", ctypes.c_int), ("N", ctypes.c_int), ("S", ctypes.c_int), ("T", ctypes.c_int),
        ("n_sin", ctypes.c_int), ("dup_v", ctypes.c_int), ("dup_h", ctypes.c_int),
        ("dup_c", ctypes.c_int), ("n_in", ctypes.c_int), ("n_out", ctypes.c_int),
        ("n_layers", ctypes.c_int), ("width", ctypes.c_int * (MAX_LAYERS + 1)),
        ("act_hidden", ctypes.c_int), ("act_out", ctypes.c_int),
        ("run_period", ctypes.c_int), ("turn_period", ctypes.c_int),
        ("jump_period", ctypes.c_int), ("robot_id", ctypes.c_int),
        ("loss_mask", ctypes.c_int), ("n_threads", ctypes.c_int), ("loss_envs", ctypes.c_int),
        ("dt", ctypes.c_double), ("gravity", ctypes.c_double), ("ground", ctypes.c_double),
        ("drag", ctypes.c_double), ("dashpot", ctypes.c_double), ("friction", ctypes.c_double),
        ("spring_omega", ctypes.c_double), ("max_speed", ctypes.c_double),
        ("max_height", ctypes.c_double),
        ("sa", _I), ("sb", _I), ("out_index", _I),
        ("len", _D), ("stiff", _D), ("coef", _D), ("init_obj", _D),
        ("W", _D * MAX_LAYERS), ("b", _D * MAX_LAYERS),
        ("gW", _D * MAX_LAYERS), ("gb", _D * MAX_LAYERS),
        ("x", _D), ("v", _D), ("v_inc", _D), ("center", _D),
        ("height", _D), ("upper", _D), ("rotation", _D), ("act", _D), ("input", _D),
        ("z", _D * MAX_LAYERS), ("tv", _D), ("th", _D), ("tc", _D),
        ("gx", _D), ("gv", _D), ("gv_inc", _D), ("gcenter", _D), ("gheight", _D),
        ("gupper", _D), ("gact", _D), ("ginput", _D), ("gz", _D * MAX_LAYERS),
        ("loss", _D), ("loss_batch", _D), ("current_max_height", _D),
    ]


_lib = None


def library():
    """Load (building on first use if needed) the oracle shared library."""
    global _lib
    if _lib is not None:
        return _lib
    path = os.path.join(HERE, "libms_oracle.so")
    src = os.path.join(HERE, "ms_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, path])
    lib = ctypes.CDLL(path)
    lib.orc_ms_forward.argtypes = [ctypes.POINTER(_OrcMS), ctypes.c_int]
    lib.orc_ms_forward_eval.argtypes = [ctypes.POINTER(_OrcMS), ctypes.c_int]
    lib.orc_ms_forward_eval.restype = ctypes.c_int
    lib.orc_ms_loss.argtypes = [ctypes.POINTER(_OrcMS), ctypes.c_int]
    lib.orc_ms_backward.argtypes = [ctypes.POINTER(_OrcMS), ctypes.c_int]
    for f in (lib.orc_ms_forward, lib.orc_ms_loss, lib.orc_ms_backward):
        f.restype = ctypes.c_int
    lib.orc_adam.argtypes = [_D, _D, _D, _D, ctypes.c_long, ctypes.c_double,
                             ctypes.c_double, ctypes.c_double, ctypes.c_int]
    lib.orc_adam.restype = None
    lib.orc_tns.argtypes = [_D, ctypes.c_long]
    lib.orc_tns.restype = ctypes.c_double
    _lib = lib
    return lib


_study = None


def study_library():
    """The oracle built with its precision-study hooks (``make study``:
    ``-DORC_STUDY``), for tests/study_fp32_state.py.  ``orc_study_set(bits,
    flags, flag_mode, x_exact)`` selects the FP32-stored fields (the ST_* bits
    of ms_oracle.c), the contact-decision array ([T][B][N] uint8; mode 1
    records, 2 forces) and the exact-position array of ST_X_EXACT.  Assign it
    to a MassSpringOracle's ``lib`` to run that oracle under the hooks."""
    global _study
    if _study is not None:
        return _study
    path = os.path.join(HERE, "libms_oracle_study.so")
    src = os.path.join(HERE, "ms_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, "study"])
    lib = ctypes.CDLL(path)
    for f in (lib.orc_ms_forward, lib.orc_ms_forward_eval, lib.orc_ms_loss, lib.orc_ms_backward):
        f.argtypes = [ctypes.POINTER(_OrcMS), ctypes.c_int]
        f.restype = ctypes.c_int
    lib.orc_study_set.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    lib.orc_study_set.restype = None
    _study = lib
    return lib


def _p(a, ptr=_D):
    return a.ctypes.data_as(ptr)


class MassSpringOracle:
    """One robot type, ``B`` environments, full ``[T][B][...]`` trajectory.

    ``springs`` rows are ``[a, b, rest_length, stiffness, actuation]`` as the
    reference's robot builder emits them (robot_design.py:344-349); stiffness is
    divided by ``stiffness_div`` (10 in the reference, solver_mass_spring.py:64).
    ``hidden`` lists the hidden-layer widths (reference: ``[n_hidden]``).
    ``out_index[s]`` is the MLP output driving spring ``s`` (reference: ``s``).
    """

    def __init__(self, objects, springs, B, T, *, n_sin, dup_v, dup_h, dup_c,
                 hidden, dt, gravity, ground, drag, dashpot, spring_omega,
                 run_period, turn_period, jump_period, robot_id=-1, friction=0.4,
                 act_hidden="sin", act_out="sin", out_index=None, n_out=None,
                 loss=("velocity", "rotation"), max_speed=0.1, max_height=0.1,
                 stiffness_div=10.0, n_threads=0, initial_objects=None, loss_envs=0):
        objects = np.asarray(objects, dtype=np.float64).reshape(-1, 3)
        springs = np.asarray(springs, dtype=np.float64).reshape(-1, 5)
        N, S = objects.shape[0], springs.shape[0]
        self.N, self.S, self.B, self.T = N, S, B, T
        n_in = n_sin + 6 * N + 2 * dup_v + dup_h + dup_c
        if out_index is None:
            out_index = np.arange(S, dtype=np.int32)
            n_out = S if n_out is None else n_out
        out_index = np.ascontiguousarray(out_index, dtype=np.int32)
        if n_out is None:
            n_out = int(out_index.max()) + 1
        self.widths = [n_in] + list(hidden) + [n_out]
        L = len(self.widths) - 1
        assert 1 <= L <= MAX_LAYERS
        self.n_in, self.n_out, self.L = n_in, n_out, L
        self.sa = np.ascontiguousarray(springs[:, 0], dtype=np.int32)
        self.sb = np.ascontiguousarray(springs[:, 1], dtype=np.int32)
        self.len = np.ascontiguousarray(springs[:, 2])
        self.stiff = np.ascontiguousarray(springs[:, 3] / stiffness_div)
        self.coef = np.ascontiguousarray(springs[:, 4])
        self.out_index = out_index
        init = objects.copy() if initial_objects is None else np.asarray(initial_objects, np.float64)
        self.init_obj = np.ascontiguousarray(init.reshape(-1))
        z = lambda *s: np.zeros(s, dtype=np.float64)  # noqa: E731
        self.W = [z(self.widths[l + 1], self.widths[l]) for l in range(L)]
        self.b = [z(self.widths[l + 1]) for l in range(L)]
        self.gW = [np.zeros_like(w) for w in self.W]
        self.gb = [np.zeros_like(b) for b in self.b]
        self.x, self.v, self.v_inc = z(T, B, N, 3), z(T, B, N, 3), z(T, B, N, 3)
        self.center = z(T, B, 3)
        self.height, self.upper, self.rotation = z(T, B), z(T, B), z(T, B)
        self.act = z(T, B, S)
        self.input = z(T, B, n_in)
        self.zs = [z(T, B, self.widths[l + 1]) for l in range(L)]
        self.tv, self.th, self.tc = z(T, B, 3), z(T, B), z(T, B)
        self.gx, self.gv, self.gv_inc = z(T, B, N, 3), z(T, B, N, 3), z(T, B, N, 3)
        self.gcenter, self.gheight, self.gupper = z(T, B, 3), z(T, B), z(T, B)
        self.gact, self.ginput = z(T, B, S), z(T, B, n_in)
        self.gzs = [z(T, B, self.widths[l + 1]) for l in range(L)]
        self.loss = z(len(LOSS_SLOTS))
        self.loss_batch = z(len(LOSS_SLOTS), B)
        self.cmh = z(1)
        s = _OrcMS()
        s.B, s.N, s.S, s.T = B, N, S, T
        s.n_sin, s.dup_v, s.dup_h, s.dup_c = n_sin, dup_v, dup_h, dup_c
        s.n_in, s.n_out, s.n_layers = n_in, n_out, L
        for l, w in enumerate(self.widths):
            s.width[l] = w
        s.act_hidden, s.act_out = ACT[act_hidden], ACT[act_out]
        s.run_period, s.turn_period, s.jump_period = run_period, turn_period, jump_period
        s.robot_id = robot_id
        s.loss_mask = sum(LOSS_BITS[n] for n in loss)
        s.n_threads = n_threads
        s.loss_envs = loss_envs
        s.dt, s.gravity, s.ground, s.drag, s.dashpot = dt, gravity, ground, drag, dashpot
        s.friction, s.spring_omega = friction, spring_omega
        s.max_speed, s.max_height = max_speed, max_height
        s.sa, s.sb, s.out_index = _p(self.sa, _I), _p(self.sb, _I), _p(self.out_index, _I)
        s.len, s.stiff, s.coef = _p(self.len), _p(self.stiff), _p(self.coef)
        s.init_obj = _p(self.init_obj)
        for l in range(L):
            s.W[l], s.b[l] = _p(self.W[l]), _p(self.b[l])
            s.gW[l], s.gb[l] = _p(self.gW[l]), _p(self.gb[l])
            s.z[l], s.gz[l] = _p(self.zs[l]), _p(self.gzs[l])
        for name in ("x", "v", "v_inc", "center", "height", "upper", "rotation", "act",
                     "input", "tv", "th", "tc", "gx", "gv", "gv_inc", "gcenter",
                     "gheight", "gupper", "gact", "ginput", "loss", "loss_batch"):
            setattr(s, name, _p(getattr(self, name)))
        s.current_max_height = _p(self.cmh)
        self._s = s
        self.lib = library()

    # -- inputs ---------------------------------------------------------------
    def set_weights(self, Ws, bs):
        for l in range(self.L):
            self.W[l][...] = Ws[l]
            self.b[l][...] = bs[l]

    def set_initial_state(self, x0, v0=None):
        self.x[0] = np.broadcast_to(np.asarray(x0, np.float64), (self.B, self.N, 3))
        self.v[0] = 0.0 if v0 is None else np.broadcast_to(v0, (self.B, self.N, 3))

    def set_targets(self, tv, th, tc=None):
        self.tv[...] = tv
        self.th[...] = th
        self.tc[...] = 0.0 if tc is None else tc

    # -- passes ---------------------------------------------------------------
    def forward(self, steps, train=True):
        """Training rollout (t in [0, steps-2]) or, with ``train=False``, the
        forward-only evaluation rollout (t in [0, steps])."""
        for a in (self.center, self.height, self.upper, self.rotation, self.act,
                  self.input, *self.zs):
            a[...] = 0.0
        self.x[1:] = 0.0
        self.v[1:] = 0.0
        fn = self.lib.orc_ms_forward if train else self.lib.orc_ms_forward_eval
        rc = fn(ctypes.byref(self._s), steps)
        if rc != 0:
            raise RuntimeError("oracle forward failed: %d" % rc)

    def compute_loss(self, steps):
        rc = self.lib.orc_ms_loss(ctypes.byref(self._s), steps)
        if rc != 0:
            raise RuntimeError("orc_ms_loss failed: %d" % rc)
        return dict(zip(LOSS_SLOTS, self.loss.tolist()))

    def backward(self, steps):
        for a in (self.gx, self.gv, self.gv_inc, self.gcenter, self.gheight, self.gupper,
                  self.gact, self.ginput, *self.gzs, *self.gW, *self.gb):
            a[...] = 0.0
        rc = self.lib.orc_ms_backward(ctypes.byref(self._s), steps)
        if rc != 0:
            raise RuntimeError("orc_ms_backward failed: %d" % rc)

    def run(self, steps):
        """forward + loss + backward; returns the total loss."""
        self.forward(steps)
        total = self.compute_loss(steps)["total"]
        self.backward(steps)
        return total

    def adam(self, m, v, lr, b1, b2, it):
        """Model.gradient_update (adam) over all weight tensors."""
        for l in range(self.L):
            for w, g, mm, vv in ((self.W[l], self.gW[l], m[2 * l], v[2 * l]),
                                 (self.b[l], self.gb[l], m[2 * l + 1], v[2 * l + 1])):
                self.lib.orc_adam(_p(w), _p(g), _p(mm), _p(vv), w.size, lr, b1, b2, it)

    def tns(self):
        return float(sum(self.lib.orc_tns(_p(g), g.size) for g in (*self.gW, *self.gb)))
