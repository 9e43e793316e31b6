"""CUDA mass-spring path (through the C ABI) against the FP64 oracle and the
reference-generated golden vectors.

Tolerances: the FP64 build must agree with the oracle to rounding (1e-9
relative); the FP32 build to rel 1e-5 on trajectories over these <= 48-substep
rollouts and rel 1e-4 on losses and gradients.
"""
import numpy as np
import pytest

from helpers import (TRAIN_CASES, batch_from_golden, load_golden, max_rel,
                     oracle_from_golden, rel_err)

pytestmark = pytest.mark.gpu

TOL = {64: dict(traj=1e-9, loss=1e-9, grad=1e-8), 32: dict(traj=1e-5, loss=1e-4, grad=1e-4)}


def _oracle_run(g):
    o = oracle_from_golden(g)
    steps = int(g["steps"])
    o.run(steps)
    return o


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("case", TRAIN_CASES)
def test_forward_matches_golden(case, precision):
    g = load_golden(case)
    steps = int(g["steps"])
    b = batch_from_golden(g, precision=precision, K=7)
    b.forward(steps)
    terms, env = b.loss()
    obs = b.observables()
    tol = TOL[precision]
    assert max_rel(obs["center"], g["center"]) < tol["traj"]
    assert max_rel(obs["height"], g["height"]) < tol["traj"]
    assert max_rel(obs["upper_height"], g["upper_height"]) < tol["traj"]
    x = b.trajectory()
    B, N = int(g["B"]), g["objects"].shape[0]
    gx = g["x"].reshape(g["x"].shape[0], B * N, 3)
    assert max_rel(x[:steps], gx[:steps]) < tol["traj"]
    xf, vf = b.final_state()
    assert max_rel(xf, gx[steps - 1]) < tol["traj"]
    assert abs(terms["total"] - float(g["loss"])) <= tol["loss"] * abs(float(g["loss"]))
    np.testing.assert_allclose(env[0], g["loss_batch"], rtol=tol["loss"] * 10, atol=1e-12)
    b.close()


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("case", TRAIN_CASES)
def test_gradients_match_oracle(case, precision):
    g = load_golden(case)
    steps = int(g["steps"])
    o = _oracle_run(g)
    b = batch_from_golden(g, precision=precision, K=9)
    loss = b.simulate(steps)
    tol = TOL[precision]
    assert abs(loss - o.loss[0]) <= tol["loss"] * abs(o.loss[0])
    for l in range(2):
        gW, gb = b.get_grads(0, l)
        assert rel_err(gW, o.gW[l]) < tol["grad"], (l, rel_err(gW, o.gW[l]))
        assert rel_err(gb, o.gb[l]) < tol["grad"], (l, rel_err(gb, o.gb[l]))
    gx0, gv0 = b.state_grads()
    B, N = int(g["B"]), g["objects"].shape[0]
    assert rel_err(gx0, o.gx[0].reshape(B * N, 3)) < tol["grad"]
    assert rel_err(gv0, o.gv[0].reshape(B * N, 3)) < tol["grad"]
    b.close()


@pytest.mark.parametrize("K", [1, 5, 47])
def test_checkpoint_interval_does_not_change_gradients(K):
    g = load_golden("quad_ref")
    steps = int(g["steps"])
    ref = batch_from_golden(g, precision=64, K=10)
    ref.simulate(steps)
    gw_ref = ref.get_grads(0, 0)[0]
    gx_ref = ref.state_grads()[0]
    b = batch_from_golden(g, precision=64, K=K)
    b.simulate(steps)
    gw = b.get_grads(0, 0)[0]
    # the forward kernels are deterministic, so the recompute reproduces the
    # first pass bit for bit; K only regroups the per-segment weight-gradient
    # sums and the atomic adds of the actuation gradients
    assert rel_err(b.state_grads()[0], gx_ref) < 1e-12
    assert rel_err(gw, gw_ref) < 1e-12


@pytest.mark.parametrize("precision", [64, 32])
def test_single_segment_records_in_first_pass(precision):
    """An episode of one checkpoint segment (steps - 1 <= K) takes its records
    from the first pass and skips the recompute: the same gradients as a
    multi-segment schedule (FP64 to rounding of the regrouped weight-gradient
    sums; FP32 within its atomic-add rounding) and one forward launch fewer
    per segment."""
    g = load_golden("quad_ref")
    steps = int(g["steps"])
    ref = batch_from_golden(g, precision=precision, K=7)
    ref.simulate(steps)
    one = batch_from_golden(g, precision=precision, K=int(g["x"].shape[0]))
    one.profile(True)
    one.simulate(steps)
    _, n = one.profile_read(reset=True)
    assert n["recompute"] == 0
    tol = 1e-12 if precision == 64 else 1e-5
    for l in range(2):
        assert rel_err(one.get_grads(0, l)[0], ref.get_grads(0, l)[0]) < tol
    assert rel_err(one.state_grads()[0], ref.state_grads()[0]) < tol
    ref.close()
    one.close()


def test_per_env_launch_equals_batched():
    g = load_golden("spider_ref")
    steps = int(g["steps"])
    b = batch_from_golden(g, precision=32, K=8)
    l1 = b.simulate(steps)
    g1 = b.get_grads(0, 0)[0]
    l2 = b.simulate(steps, per_env=True)
    g2 = b.get_grads(0, 0)[0]
    assert l1 == l2          # deterministic forward: identical losses
    assert rel_err(g2, g1) < 1e-5   # atomic adds (actuation, weight gradients) only change rounding


def test_eval_rollout_matches_golden():
    g = load_golden("snake_eval")
    steps = int(g["steps"])
    b = batch_from_golden(g, precision=64, K=10)
    b.forward_eval(steps)
    terms, _ = b.loss()
    obs = b.observables()
    assert max_rel(obs["center"][:steps + 1], g["center"][:steps + 1]) < 1e-9
    assert abs(terms["total"] - float(g["loss"])) <= 1e-9 * abs(float(g["loss"]))


def test_graph_replay_matches_eager():
    import torch
    g = load_golden("quad_ref")
    steps = int(g["steps"])
    b = batch_from_golden(g, precision=32, K=12)
    l_eager = b.simulate(steps)
    g_eager = b.get_grads(0, 1)[0]
    s = torch.cuda.Stream()
    b.set_stream(s.cuda_stream)
    b.graph_capture(steps)
    for _ in range(2):
        b.graph_launch()
    b.synchronize()
    terms, _ = b.loss()
    g_graph = b.get_grads(0, 1)[0]
    assert terms["total"] == pytest.approx(l_eager, rel=1e-6)
    np.testing.assert_allclose(g_graph, g_eager, rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("case", TRAIN_CASES)
def test_direct_spring_gathers_match_oracle_and_tables(case, precision):
    """The direct gathers -- each spring evaluated from both endpoints, the
    path of robots whose spring tables do not fit in shared memory (the
    uneven benchmark's) -- against the oracle, and against the table path."""
    g = load_golden(case)
    steps = int(g["steps"])
    o = oracle_from_golden(g)
    o.run(steps)
    runs = {}
    for mode in (0, 1):
        b = batch_from_golden(g, precision=precision, K=7)
        b.set_spring_tables(mode)
        assert b.spring_tables == bool(mode)
        loss = b.simulate(steps)
        runs[mode] = (loss, [b.get_grads(0, l) for l in range(2)], b.state_grads()[0],
                      b.trajectory()[:steps])
        b.close()
    tol = TOL[precision]
    loss0, grads0, gx0, traj0 = runs[0]
    assert abs(loss0 - o.loss[0]) <= tol["loss"] * abs(o.loss[0])
    for l in range(2):
        assert rel_err(grads0[l][0], o.gW[l]) < tol["grad"]
        assert rel_err(grads0[l][1], o.gb[l]) < tol["grad"]
    B, N = int(g["B"]), g["objects"].shape[0]
    assert rel_err(gx0, o.gx[0].reshape(B * N, 3)) < tol["grad"]
    same = 1e-12 if precision == 64 else 1e-6   # the same arithmetic either way
    loss1, grads1, gx1, traj1 = runs[1]
    assert abs(loss1 - loss0) <= same * abs(loss0)
    assert max_rel(traj1, traj0) < same
    for (gW, gb), (rW, rb) in zip(grads1, grads0):
        assert rel_err(gW, rW) < same and rel_err(gb, rb) < same
    assert rel_err(gx1, gx0) < same


def test_adam_step_matches_oracle():
    g = load_golden("x_all_losses")
    steps = int(g["steps"])
    o = _oracle_run(g)
    b = batch_from_golden(g, precision=64, K=10)
    b.simulate(steps)
    tns = b.adam_step(0)
    assert tns == pytest.approx(o.tns(), rel=1e-9)
    m = [np.zeros_like(a) for l in range(2) for a in (o.W[l], o.b[l])]
    v = [np.zeros_like(a) for a in m]
    o.adam(m, v, 3e-4, 0.9, 0.9, 0)
    for l in range(2):
        W, bb = b.get_weights(0, l)
        np.testing.assert_allclose(W, o.W[l], rtol=1e-12, atol=1e-15)
        np.testing.assert_allclose(bb, o.b[l], rtol=1e-12, atol=1e-15)


def test_batched_uneven_robots_match_per_robot_oracles():
    """Three robot types with different sizes and env counts in one batch; each
    type's gradient must equal its own oracle's (losses are per type)."""
    import cls_b200
    from helpers import params_from_golden
    cases = ["quad_ref", "spider_ref", "x_all_losses"]
    gs = [load_golden(c) for c in cases]
    base = gs[1]
    steps = 30
    rng = np.random.default_rng(3)
    robots, env_robot, oracles = [], [], []
    counts = [2, 1, 3]
    for r, (g, cnt) in enumerate(zip(gs, counts)):
        robots.append(cls_b200.Robot(g["objects"], g["springs"], robot_id=int(g["robot_id"]),
                                     hidden=[20], n_outputs=0))
        env_robot += [r] * cnt
    order = [2, 0, 1, 0, 2, 2]           # interleaved on purpose
    env_robot = [order[i] for i in range(6)]
    p = params_from_golden(base, precision=64, K=7, max_steps=40, loss=["velocity", "rotation"])
    b = cls_b200.MassSpringBatch(robots, env_robot, p)
    x0 = []
    for r in env_robot:
        x0.append(gs[r]["x0"][0])
    b.set_state(np.concatenate(x0))
    tv = rng.uniform(-0.1, 0.1, (40, 6, 3))
    th = rng.choice([-1.0, 0.0, 1.0], size=(40, 6))
    b.set_targets(tv, th)
    Ws = []
    for r, g in enumerate(gs):
        rows0, cols0 = b.layer_shape(r, 0)
        rows1, cols1 = b.layer_shape(r, 1)
        W0 = rng.uniform(-1, 1, (rows0, cols0)) * np.sqrt(6 / cols0)
        W1 = rng.uniform(-1, 1, (rows1, cols1)) * np.sqrt(6 / cols1)
        b0, b1 = rng.uniform(-0.1, 0.1, rows0), rng.uniform(-0.1, 0.1, rows1)
        b.set_weights(r, 0, W0, b0)
        b.set_weights(r, 1, W1, b1)
        Ws.append((W0, W1, b0, b1))
    total = b.simulate(steps)
    ref_total = 0.0
    for r, g in enumerate(gs):
        envs = [e for e, rr in enumerate(env_robot) if rr == r]
        from oracle.ms_oracle import MassSpringOracle
        from helpers import golden_kwargs
        kw = golden_kwargs(base)
        kw.update(robot_id=int(g["robot_id"]), loss=["velocity", "rotation"])
        o = MassSpringOracle(g["objects"], g["springs"], len(envs), 40, hidden=[20],
                             initial_objects=g["x0"][0], **kw)
        W0, W1, b0, b1 = Ws[r]
        o.set_weights([W0, W1], [b0, b1])
        o.x[0] = g["x0"][0][None]
        o.set_targets(tv[:, envs], th[:, envs])
        ref_total += o.run(steps)
        gW0, gb0 = b.get_grads(r, 0)
        gW1, gb1 = b.get_grads(r, 1)
        assert rel_err(gW0, o.gW[0]) < 1e-8
        assert rel_err(gW1, o.gW[1]) < 1e-8
        assert rel_err(gb0, o.gb[0]) < 1e-8
        gx0, _ = b.state_grads()
        for j, e in enumerate(envs):
            assert rel_err(gx0[b.env_slice(e)], o.gx[0, j]) < 1e-8
    assert total == pytest.approx(ref_total, rel=1e-9)
