"""ctypes binding of the C ABI declared in ``include/cls_b200.h``.

The product path has no fallback: if the CUDA library is missing or fails to
load, every entry point raises.
"""
import ctypes
import os

from . import build as _build

c_int32 = ctypes.c_int32
c_double = ctypes.c_double
P_D = ctypes.POINTER(ctypes.c_double)
P_I = ctypes.POINTER(ctypes.c_int32)
MAX_HIDDEN = 4

CLS_OK = 0
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of device memory",
          -4: "non-finite state", -5: "call out of order", -6: "bounded wait timed out"}

ACT = {"sin": 0, "tanh": 1}
LOSS_BITS = {"velocity": 1, "height": 2, "pose": 4, "actuation": 8,
             "rotation": 16, "crawl": 32}
PROFILE_KINDS = ("forward", "recompute", "reverse", "wgrad", "loss", "adam", "other", "ctrl_gemm",
                 "ctrl_gemm_adj")
LOSS_SLOTS = ("total", "velocity", "height", "pose", "rotation", "weight",
              "actuation", "crawl")


class RobotDesc(ctypes.Structure):
    _fields_ = [("n_vertices", c_int32), ("n_springs", c_int32),
                ("objects", P_D), ("springs", P_D), ("robot_id", c_int32),
                ("n_outputs", c_int32), ("spring_output", P_I),
                ("n_hidden_layers", c_int32), ("hidden", c_int32 * MAX_HIDDEN)]


class SimParams(ctypes.Structure):
    _fields_ = [("max_steps", c_int32), ("dt", c_double), ("gravity", c_double),
                ("ground_height", c_double), ("drag_damping", c_double),
                ("dashpot_damping", c_double), ("friction", c_double),
                ("stiffness_scale", c_double), ("run_period", c_int32),
                ("turn_period", c_int32), ("jump_period", c_int32),
                ("spring_omega", c_double), ("n_sin_waves", c_int32),
                ("duplicate_v", c_int32), ("duplicate_h", c_int32),
                ("duplicate_c", c_int32), ("activation_hidden", c_int32),
                ("activation_output", c_int32), ("loss_mask", c_int32),
                ("precision", c_int32), ("checkpoint_every", c_int32),
                ("max_speed", c_double), ("max_height", c_double),
                ("adam_b1", c_double), ("adam_b2", c_double),
                ("learning_rate", c_double), ("threads_per_block", c_int32),
                ("keep_trajectory", c_int32)]


class LaunchShape(ctypes.Structure):
    _fields_ = [("controller_path", c_int32), ("threads_per_block", c_int32),
                ("ctas_per_sm", c_int32), ("weights_shared", c_int32), ("ms", ctypes.c_float)]


class Request(ctypes.Structure):
    """cls_request: one rollout request for cls_admit."""
    _fields_ = [("id", ctypes.c_uint64), ("robot", c_int32), ("steps", c_int32), ("grad", c_int32),
                ("x0", P_D), ("target_v", P_D), ("target_h", P_D), ("target_c", P_D)]


class ClsError(RuntimeError):
    """A failed C-ABI call; ``code`` is the CLS_ERR_* value."""

    def __init__(self, msg, code=None):
        super().__init__(msg)
        self.code = code


_lib = None

_SIGS = {
    "cls_default_params": (None, [ctypes.POINTER(SimParams)]),
    "cls_create": (c_int32, [ctypes.POINTER(RobotDesc), c_int32, P_I, c_int32,
                             ctypes.POINTER(SimParams), ctypes.POINTER(ctypes.c_void_p)]),
    "cls_destroy": (c_int32, [ctypes.c_void_p]),
    "cls_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "cls_set_stream": (c_int32, [ctypes.c_void_p, ctypes.c_void_p]),
    "cls_get_sizes": (c_int32, [ctypes.c_void_p, P_I, P_I, P_I]),
    "cls_get_layer_shape": (c_int32, [ctypes.c_void_p, c_int32, c_int32, P_I, P_I]),
    "cls_set_state": (c_int32, [ctypes.c_void_p, P_D, P_D]),
    "cls_set_targets": (c_int32, [ctypes.c_void_p, P_D, P_D, P_D]),
    "cls_set_weights": (c_int32, [ctypes.c_void_p, c_int32, c_int32, P_D, P_D]),
    "cls_get_weights": (c_int32, [ctypes.c_void_p, c_int32, c_int32, P_D, P_D]),
    "cls_get_grads": (c_int32, [ctypes.c_void_p, c_int32, c_int32, P_D, P_D]),
    "cls_forward": (c_int32, [ctypes.c_void_p, c_int32]),
    "cls_forward_eval": (c_int32, [ctypes.c_void_p, c_int32]),
    "cls_loss": (c_int32, [ctypes.c_void_p, P_D, P_D]),
    "cls_backward": (c_int32, [ctypes.c_void_p]),
    "cls_simulate": (c_int32, [ctypes.c_void_p, c_int32, P_D]),
    "cls_simulate_per_env": (c_int32, [ctypes.c_void_p, c_int32, P_D]),
    "cls_adam_step": (c_int32, [ctypes.c_void_p, c_int32, P_D]),
    "cls_clear_adam": (c_int32, [ctypes.c_void_p]),
    "cls_get_observables": (c_int32, [ctypes.c_void_p, P_D, P_D, P_D, P_D]),
    "cls_get_trajectory": (c_int32, [ctypes.c_void_p, P_D]),
    "cls_get_targets": (c_int32, [ctypes.c_void_p, P_D, P_D, P_D]),
    "cls_set_loss_mask": (c_int32, [ctypes.c_void_p, c_int32]),
    "cls_set_loss_envs": (c_int32, [ctypes.c_void_p, c_int32, c_int32]),
    "cls_debug_gemm_starve": (c_int32, [ctypes.c_void_p, c_int32, ctypes.c_uint32]),
    "cls_env_step": (c_int32, [ctypes.c_void_p, c_int32, P_D, P_D, P_D]),
    "cls_serve_set_targets": (c_int32, [ctypes.c_void_p, c_int32, c_int32, P_D, P_D, P_D]),
    "cls_grad_buffers": (c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int64),
                                   ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int64), P_I]),
    "cls_get_final_state": (c_int32, [ctypes.c_void_p, P_D, P_D]),
    "cls_get_state_grads": (c_int32, [ctypes.c_void_p, P_D, P_D]),
    "cls_synchronize": (c_int32, [ctypes.c_void_p]),
    "cls_weights_init": (c_int32, [ctypes.c_void_p, ctypes.c_uint64]),
    "cls_initialize_train": (c_int32, [ctypes.c_void_p, c_int32, c_int32, ctypes.c_uint64,
                                       c_double]),
    "cls_profile_enable": (c_int32, [ctypes.c_void_p, c_int32]),
    "cls_profile_read": (c_int32, [ctypes.c_void_p, P_D, ctypes.POINTER(ctypes.c_int64), c_int32]),
    "cls_graph_capture": (c_int32, [ctypes.c_void_p, c_int32, c_int32]),
    "cls_graph_launch": (c_int32, [ctypes.c_void_p, c_int32]),
    "cls_set_controller_path": (c_int32, [ctypes.c_void_p, c_int32]),
    "cls_controller_batched": (c_int32, [ctypes.c_void_p, P_I]),
    "cls_phase_read": (c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]),
    "cls_set_spring_tables": (c_int32, [ctypes.c_void_p, c_int32]),
    "cls_spring_tables": (c_int32, [ctypes.c_void_p, P_I]),
    "cls_set_launch_shape": (c_int32, [ctypes.c_void_p, c_int32, c_int32, c_int32]),
    "cls_get_launch_shape": (c_int32, [ctypes.c_void_p, P_I, P_I, P_I]),
    "cls_autotune": (c_int32, [ctypes.c_void_p, c_int32, c_int32, ctypes.POINTER(LaunchShape),
                               c_int32, P_I]),
    "cls_serve_reset_env": (c_int32, [ctypes.c_void_p, c_int32, P_D, P_D, P_D, P_D, P_D]),
    "cls_serve_forward": (c_int32, [ctypes.c_void_p, P_I, P_I]),
    "cls_serve_backward": (c_int32, [ctypes.c_void_p, P_I, P_I]),
    "cls_serve_loss": (c_int32, [ctypes.c_void_p, P_I, P_D]),
    "cls_serve_env_state": (c_int32, [ctypes.c_void_p, c_int32, P_D, P_D]),
    "cls_serve_tick": (c_int32, [ctypes.c_void_p, c_int32]),
    "cls_admit": (c_int32, [ctypes.c_void_p, ctypes.POINTER(Request), ctypes.c_int64, P_I]),
    "cls_poll": (c_int32, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64), c_int32, P_I, P_I]),
    "cls_serve_result": (c_int32, [ctypes.c_void_p, ctypes.c_uint64, P_I, P_D, P_D]),
    "cls_serve_release": (c_int32, [ctypes.c_void_p, ctypes.c_uint64]),
}


def lib_path():
    return _build.LIB


def load(build_if_missing=True):
    """Load the CUDA library (building it first when sources are newer)."""
    global _lib
    if _lib is not None:
        return _lib
    path = os.environ.get("CLS_B200_LIBRARY")  # an alternative build of the same library
    if not path:
        if build_if_missing and _build.needs_build():
            _build.build()
        path = _build.LIB
    if not os.path.exists(path):
        raise ClsError("CUDA library %s is missing; run build.py" % path)
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc, handle=None):
    if rc != CLS_OK:
        lib = load()
        msg = lib.cls_last_error(handle)
        msg = msg.decode() if msg else ""
        raise ClsError("%s (%d): %s" % (ERRORS.get(rc, "error"), rc, msg), rc)


def ptr(a, kind=P_D):
    """ctypes pointer of a contiguous NumPy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(kind)
