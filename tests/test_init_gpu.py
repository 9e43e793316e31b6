"""Task sampling (cls_initialize_train) and weight initialisation
(cls_weights_init) on the device, checked by range and by their statistics
over seeded batches.

The reference draws both from ti.random (time-seeded, so no run of it can be
reproduced); the properties checked here are the ones its kernels define:

* TaichiEnv.initialize_train, 3D branch (multitask/taichi_env.py:385-447): one
  pool of uniforms per (turn period, env); with p0 the first of them, 25 % of
  the (period, env) pairs turn -1 (target_h = -1, target_v = 0), 25 % turn +1
  (target_h = 1), 25 % run along z (target_v.z = (2 p1 - 1) max_velocity) and
  25 % along x; target_c is not written; every t < steps of a period holds
  the same task.
* Model.weights_init (multitask/nn.py:59-67): W = (2 u - 1) sqrt(6 / fan_in)
  with u ~ U(0, 1); biases untouched.

Statistical bounds: chi-square (3 degrees of freedom) and Kolmogorov-Smirnov
p-values above 1e-4 for the fixed seeds used.
"""
import numpy as np
import pytest

from helpers import load_golden, params_from_golden

pytestmark = pytest.mark.gpu


def _quad_batch(n_envs, T, hidden=(64,), **over):
    import cls_b200
    g = load_golden("quad_ref")
    robot = cls_b200.Robot(g["objects"], g["springs"], robot_id=int(g["robot_id"]),
                           hidden=list(hidden))
    p = params_from_golden(g, precision=32, K=50, max_steps=T, **over)
    return cls_b200.MassSpringBatch([robot], [0] * n_envs, p)


def _classify(tv, th):
    """Task index per entry: 0 turn -1, 1 turn +1, 2 along z, 3 along x; -1
    for anything that is none of the four."""
    zero_v = (tv[..., 0] == 0) & (tv[..., 2] == 0)
    cls = np.full(th.shape, -1)
    cls[(th == -1) & zero_v] = 0
    cls[(th == 1) & zero_v] = 1
    cls[(th == 0) & (tv[..., 0] == 0)] = 2
    cls[(th == 0) & (tv[..., 2] == 0) & (tv[..., 0] != 0)] = 3
    return cls


def test_initialize_train_task_mix():
    from scipy import stats
    n_envs, T, period, vmax = 1024, 1000, 100, 0.08
    b = _quad_batch(n_envs, T, turn_period=period)
    rng = np.random.default_rng(0)
    tc0 = rng.uniform(0, 1, (T, n_envs))
    b.set_targets(np.full((T, n_envs, 3), 7.0), np.full((T, n_envs), 7.0), tc0)
    steps = T - 150                  # rows t >= steps keep what they held
    b.initialize_train(3, steps, 11, vmax)
    tv, th, tc = b.targets()
    np.testing.assert_array_equal(tc, tc0.astype(np.float32))     # target_c untouched
    assert np.all(tv[steps:] == 7.0) and np.all(th[steps:] == 7.0)
    tv, th = tv[:steps], th[:steps]
    assert np.all(tv[..., 1] == 0)
    assert np.abs(tv).max() <= vmax * (1 + 1e-6)
    # one task per (period, env), held for the whole period
    blocks = np.arange(steps) // period
    first = np.searchsorted(blocks, np.unique(blocks))
    for b0, t0 in zip(np.unique(blocks), first):
        rows = blocks == b0
        assert np.all(tv[rows] == tv[t0][None]) and np.all(th[rows] == th[t0][None])
    task = _classify(tv[first], th[first])
    assert np.all(task >= 0), "an entry outside the four tasks"
    counts = np.bincount(task.ravel(), minlength=4)
    chi2 = stats.chisquare(counts)
    assert chi2.pvalue > 1e-4, counts
    # the running speed r = 2 p1 - 1 is uniform on [-1, 1]
    r = np.concatenate([tv[first][..., 2][task == 2], tv[first][..., 0][task == 3]]) / vmax
    assert stats.kstest(r, "uniform", args=(-1, 2)).pvalue > 1e-4
    b.close()


def test_initialize_train_is_a_function_of_seed_and_iteration():
    n_envs, T = 64, 600
    b = _quad_batch(n_envs, T, turn_period=100)
    draws = {}
    for key in ((5, 1), (5, 1), (5, 2), (6, 1)):
        b.initialize_train(key[1], T, key[0], 0.1)
        draws.setdefault(key, []).append(b.targets()[:2])
    (a_v, a_h), (b_v, b_h) = draws[(5, 1)]
    np.testing.assert_array_equal(a_v, b_v)
    np.testing.assert_array_equal(a_h, b_h)
    for other in ((5, 2), (6, 1)):
        o_v, o_h = draws[other][0]
        assert not (np.array_equal(o_v, a_v) and np.array_equal(o_h, a_h))
    b.close()


def test_weights_init_range_and_distribution():
    from scipy import stats
    b = _quad_batch(4, 20, hidden=(96, 80))
    biases = []
    for l in range(3):
        rows, cols = b.layer_shape(0, l)
        bb = np.linspace(-0.5, 0.5, rows)
        b.set_weights(0, l, np.zeros((rows, cols)), bb)
        biases.append(bb)
    b.weights_init(123)
    first = []
    for l in range(3):
        W, bb = b.get_weights(0, l)
        rows, cols = W.shape
        q = np.sqrt(6.0 / cols)
        np.testing.assert_allclose(bb, biases[l], rtol=1e-6, atol=1e-7)   # biases untouched
        assert np.abs(W).max() <= q * (1 + 1e-6)
        u = W.ravel() / q                                                  # 2 u - 1 ~ U(-1, 1)
        assert stats.kstest(u, "uniform", args=(-1, 2)).pvalue > 1e-4, l
        assert abs(u.mean()) < 5 * np.sqrt(1 / 3 / u.size)
        first.append(W)
    b.weights_init(123)
    for l in range(3):
        np.testing.assert_array_equal(b.get_weights(0, l)[0], first[l])
    b.weights_init(124)
    assert not np.array_equal(b.get_weights(0, 0)[0], first[0])
    b.close()
