"""Served requests on the GPU: a request's result is the same alone and in a
mix that folds other requests into the running launches, and both equal the
plain one-env batch (cls_forward + cls_loss + cls_backward) of the same robot,
weights and targets.  Losses within rel 1e-6 (the first pass is
deterministic), weight gradients within rel 1e-5 (the reverse pass adds
actuation gradients and weight-gradient splits with atomic adds); FP64 at 1e-10."""
import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu


def _types(precision):
    from cls_b200 import robot_design
    from cls_b200.batch import Robot
    from cls_b200.serving import RobotType
    obj, spr = robot_design.quadruped_lattice()
    types = {"quad": RobotType(Robot.actuated_outputs(obj, spr, hidden=[64]))}
    rng = np.random.default_rng(5)
    for name, n in (("lat120", 120), ("lat300", 300)):
        o2, s2 = robot_design.random_lattice(rng, n)
        types[name] = RobotType(Robot.actuated_outputs(o2, s2, hidden=[64, 64]))
    return types


def _params(T, precision):
    from cls_b200 import workloads
    from cls_b200.batch import default_params
    return default_params(**workloads._params(T, 50, precision=precision))


def _requests():
    from cls_b200.serving import Request
    return [Request("quad", 300, grad=True, seed=11), Request("lat120", 260, grad=False, seed=12),
            Request("lat300", 400, grad=True, seed=13), Request("quad", 120, grad=False, seed=14),
            Request("lat120", 333, grad=True, seed=15), Request("lat300", 75, grad=False, seed=16)]


def _serve(types, params, reqs, slots, stagger, rounds=1):
    from cls_b200.serving import Server
    srv = Server(types, slots, params, tick_segments=rounds)
    try:
        ids = []
        for k, r in enumerate(reqs):
            ids.append(srv.submit(r))
            if stagger and k % 2 == 1:
                srv.tick()
                srv.tick()
        res = {r.rid: r for r in srv.drain()}
        return [res[i] for i in ids]
    finally:
        srv.close()


def _plain(types, params, req):
    from cls_b200.batch import MassSpringBatch
    from cls_b200.serving import request_targets
    rt = types[req.kind]
    b = MassSpringBatch([rt.robot], [0], params)
    try:
        for l, (W, bias) in enumerate(rt.weights):
            b.set_weights(0, l, W, bias)
        tv, th = request_targets(req.seed, b.T, req.steps, params.turn_period)
        b.set_targets(tv[:, None, :], th[:, None])
        b.forward(req.steps)
        terms, _ = b.loss()
        grads = None
        if req.grad:
            b.backward()
            grads = [b.get_grads(0, l) for l in range(b.n_layers(0))]
        x, _ = b.final_state()
        return terms["total"], grads, x
    finally:
        b.close()


@pytest.mark.parametrize("precision,rounds", [(32, 1), (64, 1), (32, 3)])
def test_served_results_same_alone_in_mix_and_as_plain_batch(precision, rounds):
    """rounds: checkpoint segments per tick (forward windows of rounds * K
    substeps, rounds reverse segments per tick)."""
    import copy
    types = _types(precision)
    params = _params(400, precision)
    tl, tg = (1e-6, 1e-5) if precision == 32 else (1e-10, 1e-10)
    mix = _serve(types, params, _requests(), {"quad": 2, "lat120": 2, "lat300": 2}, stagger=True,
                 rounds=rounds)
    # the mix made the types' controllers; alone-runs reuse them
    for req, got in zip(_requests(), mix):
        alone = _serve(types, params, [copy.copy(req)], {req.kind: 1}, stagger=False)[0]
        ref_loss, ref_grads, ref_x = _plain(types, params, req)
        assert got.loss == pytest.approx(alone.loss, rel=tl, abs=1e-12)
        assert got.loss == pytest.approx(ref_loss, rel=tl, abs=1e-12)
        assert rel_err(got.final_x, ref_x) < tl
        if req.grad:
            for (gW, gb), (aW, ab), (rW, rb) in zip(got.grads, alone.grads, ref_grads):
                assert rel_err(gW, aW) < tg and rel_err(gW, rW) < tg
                assert rel_err(gb, ab) < tg and rel_err(gb, rb) < tg
        else:
            assert got.grads is None


def test_open_loop_run_reports_latency():
    from cls_b200.serving import Server, poisson_requests
    types = _types(32)
    params = _params(400, 32)
    rng = np.random.default_rng(3)
    reqs = poisson_requests(rng, 100.0, 0.2, list(types), [0.4, 0.3, 0.3], steps_lo=50, steps_hi=400)
    srv = Server(types, {"quad": 4, "lat120": 4, "lat300": 4}, params)
    try:
        res, st = srv.run(reqs)
    finally:
        srv.close()
    assert len(res) == len(reqs) and st["requests"] == len(reqs)
    assert 0 < st["p50_ms"] <= st["p99_ms"]
    assert all(np.isfinite(r.loss) for r in res)


def _mpm_type():
    from cls_b200 import workloads
    from cls_b200.serving import MpmType
    pos, mus, fib = workloads.legged_body(n_grid=32, ppc=2, torso=(12, 4, 7), leg=(3, 5, 3),
                                          origin_cells=(9, 4, 12))
    E, nu = 1e4, 0.3
    solver = dict(n_grid=32, bound=3, material="neo_hookean", precision=64, dt=1e-4, gravity=-10.0,
                  p_vol=1.0, mu=E / (2 * (1 + nu)), la=E * nu / ((1 + nu) * (1 - 2 * nu)), act_strength=1e3,
                  mass=1.0)
    return MpmType(pos, mus, fib, n_muscles=16, solver=solver)


def _mpm_plain(mt, T, K, req):
    from cls_b200.mpm import MPMBatch
    from cls_b200.serving import mpm_request_inputs
    b = MPMBatch(mt.positions, mt.muscle, 1, dim=3, fibre=mt.fibre, n_muscles=mt.n_muscles, max_steps=T,
                 checkpoint_every=K, **mt.solver)
    try:
        b.set_state(mt.positions[None])
        b.set_actuation(mpm_request_inputs(req.seed, T, req.steps, 16, 1e-4)[:, None, :])
        w = np.zeros(T + 1)
        w[req.steps] = 1.0
        c0 = mt.positions.mean(axis=0)
        b.set_loss(w, np.broadcast_to(c0 + np.array([0.05, 0, 0]), (T + 1, 1, 3)).copy())
        loss = b.run(req.steps)
        g = b.grads()
        return loss, b.final_state()[0][0], (g["act"][:req.steps, 0], g["x0"][0])
    finally:
        b.close()


def test_mpm_requests_same_alone_in_mix_and_as_plain_batch():
    """MPM rollout requests (configs[2]-style bodies) served in whole-rollout
    slots beside mass-spring pools: each result equals its alone run and a
    plain one-env MPMBatch.  FP64 (the P2G reductions are atomic, so only
    rounding separates the runs): loss, positions and the gradients with
    respect to the initial positions rel 1e-10; the actuation gradients of
    this short horizon are tiny (~1e-15, sums of cancelling terms) and
    compared at rel 1e-5."""
    import copy
    from cls_b200.serving import Request
    types = _types(32)
    types["blob"] = _mpm_type()
    T, K = 160, 40
    params = _params(T, 32)
    params.checkpoint_every = K
    reqs = [Request("blob", 120, grad=True, seed=21), Request("quad", 150, grad=False, seed=22),
            Request("blob", 80, grad=False, seed=23), Request("blob", 100, grad=True, seed=24),
            Request("lat120", 90, grad=True, seed=25)]
    mix = _serve(types, params, reqs, {"quad": 1, "lat120": 1, "blob": 2}, stagger=True)
    mt = types["blob"]
    for req, got in zip(reqs, mix):
        if req.kind != "blob":
            continue
        alone = _serve(types, params, [copy.copy(req)], {"blob": 1}, stagger=False)[0]
        ref_loss, ref_x, ref_g = _mpm_plain(mt, T, K, req)
        for r in (got, alone):
            assert r.loss == pytest.approx(ref_loss, rel=1e-10)
            assert rel_err(r.final_x, ref_x) < 1e-10
            if req.grad:
                assert rel_err(r.grads["x0"], ref_g[1]) < 1e-10
                assert rel_err(r.grads["act"], ref_g[0]) < 1e-5
            else:
                assert r.grads is None


@pytest.mark.parametrize("precision,rounds", [(32, 1), (64, 2)])
def test_library_admission_and_poll_match_plain_batch(precision, rounds):
    """The library's own scheduler (cls_admit / cls_poll over one handle whose
    envs are the slots): requests admitted two per poll while earlier ones run
    give the plain one-env batch's loss, final positions and gradients."""
    from cls_b200.batch import MassSpringBatch
    from cls_b200.serving import Request, request_targets
    types = _types(precision)
    del types["quad"]              # one handle: every robot of it has the same MLP depth
    params = _params(400, precision)
    kinds = ["lat120", "lat120", "lat300", "lat300", "lat120"]
    b = MassSpringBatch([types[k].robot for k in kinds], list(range(len(kinds))), params)
    try:
        rng = np.random.default_rng(9)
        for k in types:
            s0 = kinds.index(k)
            types[k].weights = []
            for l in range(b.n_layers(s0)):
                rows, cols = b.layer_shape(s0, l)
                types[k].weights.append(((rng.random((rows, cols)) * 2 - 1) * np.sqrt(6.0 / cols),
                                         rng.uniform(-0.1, 0.1, rows)))
        for slot, k in enumerate(kinds):
            for l, (W, bias) in enumerate(types[k].weights):
                b.set_weights(slot, l, W, bias)
        b.serve_tick(rounds)
        reqs = [Request("lat120", 260, grad=False, seed=12), Request("lat300", 400, grad=True, seed=13),
                Request("lat120", 333, grad=True, seed=15), Request("lat300", 75, grad=False, seed=16),
                Request("lat120", 150, grad=True, seed=17), Request("lat300", 220, grad=True, seed=18),
                Request("lat120", 2, grad=True, seed=19)]
        pending = list(range(len(reqs)))
        results = {}
        for _ in range(400):
            for rid in list(pending[:2]):
                req = reqs[rid]
                tv, th = request_targets(req.seed, b.T, req.steps, params.turn_period)
                slot = b.admit(rid, kinds.index(req.kind), req.steps, req.grad, target_v=tv, target_h=th)
                if slot >= 0:
                    assert kinds[slot] == req.kind
                    pending.remove(rid)
            done, active = b.poll()
            for rid in done:
                slot, terms, x = b.serve_result(rid)
                grads = [b.get_grads(slot, l) for l in range(b.n_layers(slot))] if reqs[rid].grad else None
                results[rid] = (terms[0], grads, x)
                b.serve_release(rid)
            if not pending and active == 0:
                break
    finally:
        b.close()
    assert sorted(results) == list(range(len(reqs)))
    tl, tg = (1e-6, 1e-5) if precision == 32 else (1e-10, 1e-10)
    for rid, req in enumerate(reqs):
        loss, grads, x = results[rid]
        ref_loss, ref_grads, ref_x = _plain(types, params, req)
        assert loss == pytest.approx(ref_loss, rel=tl, abs=1e-12)
        assert rel_err(x, ref_x) < tl
        if req.grad:
            for (gW, gb), (rW, rb) in zip(grads, ref_grads):
                assert rel_err(gW, rW) < tg and rel_err(gb, rb) < tg
