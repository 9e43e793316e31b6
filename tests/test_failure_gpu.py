"""Failure detection on the GPU, in the forms that neither fault nor hang the
device: a non-finite state (NaN weights or a NaN initial state) is flagged by
the kernels and reported by cls_synchronize as CLS_ERR_NONFINITE; a
tensor-core tile whose bounded wait runs out (the starve self-test: no
operands are ever copied, nothing is in flight) reports CLS_ERR_TIMEOUT after
freeing its tensor memory.  After either, the handle keeps working and
reproduces a clean run.  The reference has no failure handling of its own
beyond Python exceptions (multitask/base_trainer.py:56-60)."""
import numpy as np
import pytest

from helpers import batch_from_golden, load_golden, many_env_batch

pytestmark = pytest.mark.gpu


def _expect(code, fn):
    import cls_b200
    with pytest.raises(cls_b200._capi.ClsError) as ei:
        fn()
    assert ei.value.code == code, str(ei.value)
    return str(ei.value)


@pytest.mark.parametrize("what", ["weights", "state"])
def test_non_finite_input_is_reported(what):
    g = load_golden("quad_ref")
    steps = 20
    b = batch_from_golden(g, precision=32, K=8)
    ref = b.simulate(steps)
    b.synchronize()
    if what == "weights":
        W = g["W1"].copy()
        W[3, 17] = np.nan
        b.set_weights(0, 0, W, g["b1"])
    else:
        x0 = g["x0"].reshape(-1, 3).copy()
        x0[5, 1] = np.nan
        b.set_state(x0)
    b.forward(steps)
    msg = _expect(-4, b.synchronize)
    assert "non-finite" in msg
    b.synchronize()                           # the status was cleared
    b.set_weights(0, 0, g["W1"], g["b1"])
    b.set_state(g["x0"].reshape(-1, 3))
    assert b.simulate(steps) == ref
    b.synchronize()
    b.close()


def test_tensor_core_wait_timeout_is_reported_and_recovers():
    b = many_env_batch(32, 64, [64], 8, 12, "batched")
    assert b.controller_batched
    ref = b.simulate(8)
    gref = b.get_grads(0, 0)[0]
    b.synchronize()
    b.lib.cls_debug_gemm_starve(b.h, 1, 1 << 14)
    b.forward(8)
    b.loss()
    b.backward()
    msg = _expect(-6, b.synchronize)
    assert "bounded wait" in msg
    b.lib.cls_debug_gemm_starve(b.h, 0, 0)
    assert b.simulate(8) == ref               # tensor memory was freed: the tiles run again
    np.testing.assert_array_equal(b.get_grads(0, 0)[0], gref)
    b.synchronize()
    b.close()
