"""cls_ms_advance_noalloc: the entry point for callers that may not allocate
device memory (they cannot create a cls_sim, whose buffers come from
cudaMalloc).  It must reproduce the regular entry point's trajectory while
allocating nothing, on two calls in a row that share its fixed scratch array.

The regular path is cls_forward with a controller whose weights are all zero,
so every spring's actuation is the constant sin(bias); the no-alloc call is
given exactly those actuations.  Tolerances: FP32 positions rel 1e-5 (the
spring sums are accumulated in a different order); velocities rel 1e-4 (the
same rounding, divided by the time step, weighs more against their size)."""
import ctypes

import numpy as np
import pytest

from helpers import batch_from_golden, load_golden, max_rel

pytestmark = pytest.mark.gpu


class NoallocAdvance(ctypes.Structure):
    _fields_ = [("n_envs", ctypes.c_int32), ("n_vertices", ctypes.c_int32),
                ("n_springs", ctypes.c_int32), ("n_substeps", ctypes.c_int32),
                ("spring_a", ctypes.c_void_p), ("spring_b", ctypes.c_void_p),
                ("rest_length", ctypes.c_void_p), ("stiffness", ctypes.c_void_p),
                ("actuation_coef", ctypes.c_void_p), ("actuation", ctypes.c_void_p),
                ("x", ctypes.c_void_p), ("v", ctypes.c_void_p),
                ("dt", ctypes.c_float), ("gravity", ctypes.c_float),
                ("ground_height", ctypes.c_float), ("drag_damping", ctypes.c_float),
                ("dashpot_damping", ctypes.c_float), ("friction", ctypes.c_float),
                ("error_message", ctypes.c_char_p), ("error_capacity", ctypes.c_int32)]


def _lib():
    import cls_b200
    lib = cls_b200._capi.load()
    fn = lib.cls_ms_advance_noalloc
    fn.argtypes = [ctypes.POINTER(NoallocAdvance), ctypes.c_void_p]
    fn.restype = ctypes.c_int32
    return fn


def _reference_final_states(g, n, biases):
    """(x, v) after n and 2n substeps through the regular entry point."""
    out = []
    for steps in (n, 2 * n):
        b = batch_from_golden(g, precision=32, K=8)
        W0, _ = b.get_weights(0, 0)
        W1, _ = b.get_weights(0, 1)
        b.set_weights(0, 0, np.zeros_like(W0), np.zeros(W0.shape[0]))
        b.set_weights(0, 1, np.zeros_like(W1), biases)
        b.forward(steps + 1)            # training rollout: steps substeps
        out.append(b.final_state())
        b.close()
    return out


def test_noalloc_matches_regular_entry_point_twice():
    import torch
    fn = _lib()
    g = load_golden("quad_ref")
    B, N = int(g["B"]), g["objects"].shape[0]
    springs = g["springs"]
    S = springs.shape[0]
    n = 20
    rng = np.random.default_rng(4)
    biases = rng.uniform(-1.0, 1.0, S)
    ref1, ref2 = _reference_final_states(g, n, biases)

    dev = torch.device("cuda:0")
    f32 = dict(dtype=torch.float32, device=dev)
    sa = torch.tensor(springs[:, 0].astype(np.int32), device=dev)
    sb = torch.tensor(springs[:, 1].astype(np.int32), device=dev)
    rest = torch.tensor(springs[:, 2], **f32)
    stiff = torch.tensor(springs[:, 3] * 0.1, **f32)      # the reference's /10
    coef = torch.tensor(springs[:, 4], **f32)
    act = torch.tensor(np.broadcast_to(np.sin(biases.astype(np.float32)), (B, S)).copy(), **f32)
    x = torch.tensor(g["x0"].reshape(B, N, 3), **f32).contiguous()
    v = torch.zeros((B, N, 3), **f32)
    msg = ctypes.create_string_buffer(256)
    a = NoallocAdvance(B, N, S, n, sa.data_ptr(), sb.data_ptr(), rest.data_ptr(), stiff.data_ptr(),
                       coef.data_ptr(), act.data_ptr(), x.data_ptr(), v.data_ptr(),
                       float(g["dt"]), float(g["gravity"]), float(g["ground"]), float(g["drag"]),
                       float(g["dashpot"]), 0.4, ctypes.cast(msg, ctypes.c_char_p), 256)
    stream = torch.cuda.current_stream().cuda_stream
    for call, (rx, rv) in enumerate((ref1, ref2)):   # two calls in a row, continuing the state
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = fn(ctypes.byref(a), ctypes.c_void_p(stream))
        assert rc == 0, msg.value
        torch.cuda.synchronize()
        if call == 1:
            # the first call may load the library's kernels (lazy module
            # loading takes device memory once); the second must take none
            assert torch.cuda.mem_get_info()[0] == free_before
        assert max_rel(x.cpu().numpy().reshape(-1, 3), rx) < 1e-5
        assert max_rel(v.cpu().numpy().reshape(-1, 3), rv) < 1e-4


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    fn = _lib()
    msg = ctypes.create_string_buffer(256)
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda:0")
    p = dummy.data_ptr()
    a = NoallocAdvance(4096, 1000, 0, 1, None, None, None, None, None, None, p, p,
                       1e-3, -9.8, 0.0, 0.0, 0.1, 0.4, ctypes.cast(msg, ctypes.c_char_p), 256)
    assert fn(ctypes.byref(a), None) == -1
    assert b"exceeds the fixed scratch" in msg.value
