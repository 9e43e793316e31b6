"""Launch shapes of the fused segment kernels and the autotuner over them
(cls_set_launch_shape / cls_get_launch_shape / cls_autotune).

The shape changes how envs are spread over CTAs (CTAs per SM: the persistent
grid's size) and where the controller is read from (shared or global memory),
both without changing a bit of the results, and the CTA size (threads per
CTA: block-wide reductions regroup, results equal within rounding).
"""
import json

import numpy as np
import pytest

from helpers import batch_from_golden, load_golden, many_env_batch, rel_err

pytestmark = pytest.mark.gpu


def _grads(b, n_layers=2):
    return [b.get_grads(0, l) for l in range(n_layers)]


def test_launch_shape_validation():
    import cls_b200
    g = load_golden("quad_ref")
    b = batch_from_golden(g, precision=32, K=7)
    for bad in ((100, 1), (32, 1), (2048, 1), (256, 0), (256, 33)):
        with pytest.raises(cls_b200._capi.ClsError):
            b.set_launch_shape(*bad)
    with pytest.raises(cls_b200._capi.ClsError):
        b.set_launch_shape(256, 1, 2)
    b.set_launch_shape(384, 3, 0)
    assert b.launch_shape == (384, 3, 0)
    with pytest.raises(cls_b200._capi.ClsError):
        b.set_launch_shape(100, 1)
    assert b.launch_shape == (384, 3, 0)   # a refused shape leaves the previous one
    b.set_launch_shape(256, 1, 1)           # the quadruped's controller fits in shared memory
    assert b.launch_shape == (256, 1, 1)
    b.close()


def test_spring_tables_switch():
    import cls_b200
    g = load_golden("quad_ref")
    b = batch_from_golden(g, precision=32, K=7)
    assert b.spring_tables                  # 272 springs: the tables fit
    with pytest.raises(cls_b200._capi.ClsError):
        b.set_spring_tables(2)
    b.set_spring_tables(0)
    assert not b.spring_tables
    b.set_spring_tables(-1)
    assert b.spring_tables
    b.close()
    from cls_b200 import workloads
    big, _, _ = workloads.uneven_batch(n_robots=2, steps=20, K=10, seed=5, vmin=1800, vmax=2000)
    assert not big.spring_tables            # > 3072 springs: direct gathers
    with pytest.raises(cls_b200._capi.ClsError, match="do not fit"):
        big.set_spring_tables(1)
    assert np.isfinite(big.simulate(20))
    big.close()


def test_controller_too_large_for_shared_memory():
    import cls_b200
    b = many_env_batch(32, 4, [1024], 10, 20, "per_env")   # 1024 x 176 weights: 720 KB
    with pytest.raises(cls_b200._capi.ClsError, match="does not fit"):
        b.set_launch_shape(256, 1, 1)
    b.set_launch_shape(256, 1, -1)          # automatic: global memory
    assert b.launch_shape == (256, 1, 0)
    assert np.isfinite(b.simulate(15))
    b.close()


@pytest.mark.parametrize("precision", [64, 32])
def test_controller_in_shared_memory_is_bit_identical(precision):
    """Weights and biases copied to shared memory once per work item give the
    same bits as reading them from global memory every substep."""
    b = many_env_batch(precision, 40, [32, 16], 9, 48, "per_env")   # FP64 controller ~80 KB
    runs = []
    for wsh in (0, 1):
        b.set_launch_shape(256, 2, wsh)
        loss = b.simulate(40)
        x, _ = b.final_state()
        runs.append((loss, _grads(b, 3), b.state_grads()[0], x))
    b.close()
    (l0, g0, s0, x0), (l1, g1, s1, x1) = runs
    assert l0 == l1 and np.array_equal(x0, x1) and np.array_equal(s0, s1)
    for (gW, gb), (rW, rb) in zip(g1, g0):
        assert np.array_equal(gW, rW) and np.array_equal(gb, rb)


@pytest.mark.parametrize("precision", [64, 32])
def test_ctas_per_sm_do_not_change_results(precision):
    """The grid only decides which CTA takes which env from the work queue."""
    b = many_env_batch(precision, 300, [70, 50], 9, 48, "per_env")
    runs = []
    for ctas in (1, 2, 4):
        b.set_launch_shape(256, ctas)
        loss = b.simulate(40)
        runs.append((loss, _grads(b, 3), b.state_grads()[0]))
    b.close()
    for loss, grads, gx in runs[1:]:
        assert loss == runs[0][0]
        for (gW, gb), (rW, rb) in zip(grads, runs[0][1]):
            assert np.array_equal(gW, rW) and np.array_equal(gb, rb)
        assert np.array_equal(gx, runs[0][2])


@pytest.mark.parametrize("precision", [64, 32])
def test_threads_per_block_change_only_rounding(precision):
    g = load_golden("quad_ref")
    steps = int(g["steps"])
    tol = 1e-12 if precision == 64 else 1e-5
    ref = None
    for threads in (64, 128, 256, 512, 1024):
        b = batch_from_golden(g, precision=precision, K=7)
        b.set_launch_shape(threads, 2)
        loss = b.simulate(steps)
        out = (loss, _grads(b), b.state_grads()[0])
        b.close()
        if ref is None:
            ref = out
            continue
        assert abs(out[0] - ref[0]) <= tol * abs(ref[0])
        for (gW, gb), (rW, rb) in zip(out[1], ref[1]):
            assert rel_err(gW, rW) < tol and rel_err(gb, rb) < tol
        assert rel_err(out[2], ref[2]) < tol


def test_autotune_applies_fastest_and_keeps_weights(tmp_path):
    from cls_b200 import workloads
    b, robots, _ = workloads.uneven_batch(n_robots=24, steps=120, K=20, seed=3, vmin=50, vmax=600)
    W0 = [b.get_weights(r, l) for r in range(len(robots)) for l in range(3)]
    ref_loss = b.simulate(120)
    ref_grads = [b.get_grads(r, 0) for r in range(len(robots))]
    cache = str(tmp_path / "shapes.json")
    res = b.autotune(repeats=1, cache=cache)
    assert not res["cached"]
    per_env = [e for e in res["table"] if e["controller_path"] == "per_env"]
    assert per_env and all(e["ms"] > 0 for e in per_env)
    assert {e["threads_per_block"] for e in per_env} <= {128, 256, 512, 1024}
    best = min(per_env, key=lambda e: e["ms"])
    shape = (best["threads_per_block"], best["ctas_per_sm"], best["weights_shared"])
    assert b.launch_shape == shape
    assert res["controller_path"] == "per_env"          # one env per type: no batched candidate
    assert all(e["controller_path"] == "per_env" for e in res["table"])
    for (W, bias), (W1, b1) in zip(W0, [b.get_weights(r, l) for r in range(len(robots)) for l in range(3)]):
        assert np.array_equal(W, W1) and np.array_equal(bias, b1)
    # the tuned shape computes the same rollout
    loss = b.simulate(120)
    assert abs(loss - ref_loss) <= 1e-5 * abs(ref_loss)
    for r in range(len(robots)):
        assert rel_err(b.get_grads(r, 0)[0], ref_grads[r][0]) < 1e-4
    # cached: applied without timing
    b.set_launch_shape(64, 1)
    hit = b.autotune(repeats=1, cache=cache)
    assert hit["cached"]
    assert b.launch_shape == shape
    with open(cache) as f:
        assert len(json.load(f)) == 1
    b.close()


def test_autotune_times_the_batched_path_for_many_envs():
    b = many_env_batch(32, 64, [64], 10, 40, "per_env")
    res = b.autotune(steps=30, repeats=1)
    batched = [e for e in res["table"] if e["controller_path"] == "batched"]
    assert len(batched) == 1
    per_env = min(e["ms"] for e in res["table"] if e["controller_path"] == "per_env")
    assert b.controller_batched == (batched[0]["ms"] < per_env)
    loss = b.simulate(30)
    assert np.isfinite(loss)
    b.close()
