"""The FP64 CPU oracle against the reference's own kernels (golden vectors made
by tests/golden/make_golden.py) and against central finite differences."""
import numpy as np
import pytest

from helpers import TRAIN_CASES, load_golden, max_rel, oracle_from_golden


@pytest.mark.parametrize("case", TRAIN_CASES)
def test_forward_matches_reference_golden(case):
    g = load_golden(case)
    o = oracle_from_golden(g)
    steps = int(g["steps"])
    o.forward(steps)
    L = o.compute_loss(steps)
    assert max_rel(o.x, g["x"]) < 1e-12
    assert max_rel(o.v, g["v"]) < 1e-12
    assert max_rel(o.center, g["center"]) < 1e-12
    np.testing.assert_allclose(o.height, g["height"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(o.upper, g["upper_height"], rtol=0, atol=1e-14)
    assert max_rel(o.rotation, g["rotation"]) < 1e-11
    assert max_rel(o.act, g["actuation"]) < 1e-12
    assert max_rel(o.input, g["input_state"]) < 1e-12
    assert max_rel(o.zs[0], g["hidden"]) < 1e-12
    assert max_rel(o.zs[1], g["output"]) < 1e-12
    assert abs(L["total"] - float(g["loss"])) <= 1e-12 * abs(float(g["loss"]))
    np.testing.assert_allclose(o.loss[1:], g["loss_terms"], rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(o.loss_batch[0], g["loss_batch"], rtol=1e-12)
    np.testing.assert_allclose(o.loss_batch[1:], g["loss_terms_batch"], rtol=1e-12, atol=1e-300)


def test_eval_rollout_matches_reference_golden():
    g = load_golden("snake_eval")
    o = oracle_from_golden(g)
    steps = int(g["steps"])
    o.forward(steps, train=False)
    L = o.compute_loss(steps)
    assert max_rel(o.x, g["x"]) < 1e-12
    assert max_rel(o.center, g["center"]) < 1e-12
    assert max_rel(o.act, g["actuation"]) < 1e-12
    assert abs(L["total"] - float(g["loss"])) <= 1e-12 * abs(float(g["loss"]))


def test_all_losses_case_exercises_every_loss():
    g = load_golden("x_all_losses")
    terms = dict(zip(("velocity", "height", "pose", "rotation", "weight", "actuation", "crawl"),
                     g["loss_terms"]))
    for k in ("velocity", "pose", "rotation", "actuation", "crawl"):
        assert terms[k] > 0, k


def _fd_check(o, steps, arrays, n=5, h=1e-6, rtol=2e-5, seed=0):
    o.run(steps)
    grads = {name: garr.copy() for name, (arr, garr) in arrays.items()}
    rng = np.random.default_rng(seed)
    for name, (arr, _) in arrays.items():
        for _ in range(n):
            idx = tuple(int(rng.integers(0, s)) for s in arr.shape)
            old = arr[idx]
            arr[idx] = old + h
            o.forward(steps)
            lp = o.compute_loss(steps)["total"]
            arr[idx] = old - h
            o.forward(steps)
            lm = o.compute_loss(steps)["total"]
            arr[idx] = old
            fd = (lp - lm) / (2 * h)
            an = grads[name][idx]
            assert abs(fd - an) <= rtol * max(abs(fd), abs(an)) + 1e-9, (name, idx, fd, an)


@pytest.mark.parametrize("case", TRAIN_CASES)
def test_oracle_gradients_match_finite_differences(case):
    g = load_golden(case)
    o = oracle_from_golden(g)
    # the symmetric rest pose puts several vertices at exactly the same
    # height, where min/max are not differentiable; move off the ties
    o.x[0] += np.random.default_rng(7).uniform(-1e-5, 1e-5, o.x[0].shape)
    th = o.th.copy()
    if case == "x_all_losses":
        th[:, 2] = 1.0      # switch the height loss on for one env
        o.th[...] = th
    steps = int(g["steps"])
    arrays = {"W0": (o.W[0], o.gW[0]), "W1": (o.W[1], o.gW[1]),
              "b0": (o.b[0], o.gb[0]), "b1": (o.b[1], o.gb[1])}
    _fd_check(o, steps, arrays)
    # initial state: only t = 0 entries are inputs
    o.run(steps)
    gx0, gv0 = o.gx[0].copy(), o.gv[0].copy()
    rng = np.random.default_rng(1)
    for arr, gref in ((o.x, gx0), (o.v, gv0)):
        for _ in range(4):
            k, i, d = (int(rng.integers(0, s)) for s in arr.shape[1:])
            old = arr[0, k, i, d]
            h = 1e-6
            arr[0, k, i, d] = old + h
            o.forward(steps)
            lp = o.compute_loss(steps)["total"]
            arr[0, k, i, d] = old - h
            o.forward(steps)
            lm = o.compute_loss(steps)["total"]
            arr[0, k, i, d] = old
            fd = (lp - lm) / (2 * h)
            an = gref[k, i, d]
            assert abs(fd - an) <= 2e-5 * max(abs(fd), abs(an)) + 5e-8  # FD round-off


def test_oracle_two_hidden_tanh_actuated_outputs_fd():
    """The generalised controller (2 hidden tanh layers, outputs only for
    actuated springs) that the batched configurations use."""
    g = load_golden("x_all_losses")
    springs = g["springs"]
    act = springs[:, 4] > 0
    out_index = np.full(len(springs), -1, dtype=np.int32)
    out_index[act] = np.arange(int(act.sum()), dtype=np.int32)
    o = oracle_from_golden(g, hidden=[16, 12], act_hidden="tanh", act_out="tanh",
                           out_index=out_index, n_out=int(act.sum()))
    rng = np.random.default_rng(5)
    for l in range(o.L):
        o.W[l][...] = rng.uniform(-1, 1, o.W[l].shape) * np.sqrt(6 / o.W[l].shape[1])
        o.b[l][...] = rng.uniform(-0.1, 0.1, o.b[l].shape)
    steps = int(g["steps"])
    arrays = {"W%d" % l: (o.W[l], o.gW[l]) for l in range(o.L)}
    arrays.update({"b%d" % l: (o.b[l], o.gb[l]) for l in range(o.L)})
    _fd_check(o, steps, arrays, n=4)


def test_oracle_adam_matches_reference_formula():
    rng = np.random.default_rng(0)
    from oracle.ms_oracle import library, _p
    lib = library()
    w = rng.normal(size=50)
    g = rng.normal(size=50)
    m = np.zeros(50)
    v = np.zeros(50)
    w_ref = w.copy()
    m_ref = np.zeros(50)
    v_ref = np.zeros(50)
    for it in range(3):
        lib.orc_adam(_p(w), _p(g), _p(m), _p(v), 50, 3e-4, 0.9, 0.9, it)
        m_ref = 0.9 * m_ref + 0.1 * g
        v_ref = 0.9 * v_ref + 0.1 * g * g
        w_ref -= 3e-4 * (m_ref / (1 - 0.9 ** (it + 1))) / (np.sqrt(v_ref / (1 - 0.9 ** (it + 1))) + 1e-8)
    np.testing.assert_allclose(w, w_ref, rtol=1e-14)


def test_study_hooks_off_reproduce_the_oracle_and_round_when_on():
    """The precision-study build of the oracle (tests/study_fp32_state.py) is
    the plain oracle when its hooks are off, replays recorded contact
    decisions exactly, and stores FP32-representable positions under ST_X."""
    from oracle.ms_oracle import study_library
    g = load_golden("quad_ref")
    steps = int(g["steps"])
    plain = oracle_from_golden(g)
    plain.run(steps)
    lib = study_library()
    o = oracle_from_golden(g)
    o.lib = lib
    flags = np.zeros((o.T, o.B, o.N), np.uint8)
    lib.orc_study_set(0, flags.ctypes.data, 1, None)
    o.run(steps)
    assert np.array_equal(o.x, plain.x) and np.array_equal(o.gW[0], plain.gW[0])
    assert flags.any()
    lib.orc_study_set(0, flags.ctypes.data, 2, None)  # force the recorded decisions
    o.run(steps)
    assert np.array_equal(o.x, plain.x) and np.array_equal(o.gW[0], plain.gW[0])
    lib.orc_study_set(1, None, 0, None)  # ST_X
    o.run(steps)
    lib.orc_study_set(0, None, 0, None)
    xs = o.x[1:steps]  # x[0] is the caller's input
    assert np.array_equal(xs, xs.astype(np.float32).astype(np.float64))
    assert not np.array_equal(xs, plain.x[1:steps])
    assert max_rel(o.x[:steps], plain.x[:steps]) < 1e-6
