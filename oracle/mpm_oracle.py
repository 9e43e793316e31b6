"""ctypes front-end of the FP64 MLS-MPM oracle (``mpm_oracle.c``).

TEST INFRASTRUCTURE ONLY (tests/ and the bench's CPU leg); the product never
imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
MATERIAL = {"fixed_corotated": 0, "neo_hookean": 1}


class _OrcMPM(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("n_grid", ctypes.c_int), ("B", ctypes.c_int),
                ("P", ctypes.c_int), ("T", ctypes.c_int), ("M", ctypes.c_int),
                ("material", ctypes.c_int), ("bound", ctypes.c_int),
                ("dx", ctypes.c_double), ("inv_dx", ctypes.c_double), ("dt", ctypes.c_double),
                ("p_vol", ctypes.c_double), ("mu", ctypes.c_double), ("la", ctypes.c_double),
                ("act_strength", ctypes.c_double), ("gravity", ctypes.c_double),
                ("mass", ctypes.c_double),
                ("muscle", _I), ("fibre", _D), ("x", _D), ("v", _D), ("C", _D), ("F", _D),
                ("act", _D), ("loss_w", _D), ("loss_pw", _D), ("target", _D),
                ("gx0", _D), ("gv0", _D), ("gC0", _D), ("gF0", _D), ("gact", _D), ("loss", _D)]


_lib = None


def library():
    global _lib
    if _lib is not None:
        return _lib
    path = os.path.join(HERE, "libmpm_oracle.so")
    src = os.path.join(HERE, "mpm_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", HERE, path])
    lib = ctypes.CDLL(path)
    for f in ("orc_mpm_forward", "orc_mpm_backward"):
        getattr(lib, f).argtypes = [ctypes.POINTER(_OrcMPM), ctypes.c_int]
        getattr(lib, f).restype = ctypes.c_int
    lib.orc_mpm_loss.argtypes = [ctypes.POINTER(_OrcMPM), ctypes.c_int]
    lib.orc_mpm_loss.restype = ctypes.c_double
    _lib = lib
    return lib


def _p(a, t=_D):
    return a.ctypes.data_as(t)


class MPMOracle:
    """B envs of one particle body on a dim-D grid, full [T+1] trajectory."""

    def __init__(self, positions, muscle, B, T, *, dim, n_grid, dt, p_vol, mu, la,
                 act_strength, gravity, bound, material="fixed_corotated", fibre=None,
                 n_muscles=None, mass=1.0):
        pos = np.asarray(positions, np.float64).reshape(-1, dim)
        P = pos.shape[0]
        self.dim, self.P, self.B, self.T = dim, P, B, T
        self.muscle = np.ascontiguousarray(muscle, dtype=np.int32)
        self.M = int(n_muscles if n_muscles is not None else max(1, self.muscle.max() + 1))
        if fibre is None:
            fibre = np.zeros((P, dim))
            fibre[:, 1] = 1.0                  # the reference actuates along y
        self.fibre = np.ascontiguousarray(np.asarray(fibre, np.float64).reshape(P, dim))
        z = lambda *s: np.zeros(s)  # noqa: E731
        self.x, self.v = z(T + 1, B, P, dim), z(T + 1, B, P, dim)
        self.C = z(T + 1, B, P, dim, dim)
        self.F = z(T + 1, B, P, dim, dim)
        self.F[...] = np.eye(dim)
        self.x[0] = pos
        self.act = z(T, B, self.M)
        self.loss_w = z(T + 1)
        self.loss_pw = np.ones(P)
        self.target = z(T + 1, B, dim)
        self.gx0, self.gv0 = z(B, P, dim), z(B, P, dim)
        self.gC0, self.gF0 = z(B, P, dim, dim), z(B, P, dim, dim)
        self.gact = z(T, B, self.M)
        self.loss = z(1)
        s = _OrcMPM()
        s.dim, s.n_grid, s.B, s.P, s.T, s.M = dim, n_grid, B, P, T, self.M
        s.material, s.bound = MATERIAL[material], bound
        s.dx, s.inv_dx, s.dt, s.p_vol = 1.0 / n_grid, float(n_grid), dt, p_vol
        s.mu, s.la, s.act_strength, s.gravity, s.mass = mu, la, act_strength, gravity, mass
        s.muscle, s.fibre = _p(self.muscle, _I), _p(self.fibre)
        for n in ("x", "v", "C", "F", "act", "loss_w", "loss_pw", "target", "gx0", "gv0", "gC0", "gF0",
                  "gact", "loss"):
            setattr(s, n, _p(getattr(self, n)))
        self._s = s
        self.lib = library()

    def forward(self, steps):
        rc = self.lib.orc_mpm_forward(ctypes.byref(self._s), steps)
        if rc:
            raise RuntimeError("orc_mpm_forward: %d" % rc)

    def compute_loss(self, steps):
        return float(self.lib.orc_mpm_loss(ctypes.byref(self._s), steps))

    def backward(self, steps):
        self.gact[...] = 0
        rc = self.lib.orc_mpm_backward(ctypes.byref(self._s), steps)
        if rc:
            raise RuntimeError("orc_mpm_backward: %d" % rc)

    def run(self, steps):
        self.forward(steps)
        L = self.compute_loss(steps)
        self.backward(steps)
        return L
