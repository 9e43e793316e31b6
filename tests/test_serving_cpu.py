"""Request-loop scheduling on the CPU with a fake backend: window tables per
tick (they must reproduce the windows of cls_forward / cls_backward),
folding of late requests into running launches, admission by slots and by
HBM footprint, and the open-loop arrival generator."""
import itertools
from types import SimpleNamespace

import numpy as np
import pytest

from cls_b200 import robot_design
from cls_b200.batch import Robot
from cls_b200.serving import (Request, RobotType, Server, footprint_bytes, poisson_requests)


class FakeBackend:
    """Records every launch; losses and gradients are functions of the request."""

    def __init__(self, slot_types, types, params):
        self.slot_types = list(slot_types)
        self.loaded = [k for k in slot_types]
        self.req = [None] * len(slot_types)
        self.calls = []

    def load_weights(self, slot, kind, weights):
        self.loaded[slot] = kind

    def reset(self, slot, req, robot):
        self.req[slot] = req
        self.calls.append(("reset", slot, req.rid))

    def forward(self, windows, steps):
        self.calls.append(("forward", windows.copy(), steps.copy()))

    def backward(self, windows, steps):
        self.calls.append(("backward", windows.copy(), steps.copy()))

    def loss(self, steps):
        env = np.zeros((8, len(self.slot_types)))
        for i, r in enumerate(self.req):
            if r is not None and steps[i] > 0:
                env[0, i] = r.seed + 0.5 * steps[i]
        return env

    def final_x(self, slot):
        return np.zeros((1, 3))

    def grads(self, slot):
        return [("grad-of", self.req[slot].rid)]

    def sync(self):
        pass

    def query(self):
        return True

    def close(self):
        pass


def _robots():
    obj, spr = robot_design.quadruped_lattice()
    quad = Robot.actuated_outputs(obj, spr, hidden=[64])
    rng = np.random.default_rng(0)
    o2, s2 = robot_design.random_lattice(rng, 120)
    lat = Robot.actuated_outputs(o2, s2, hidden=[128, 128])
    return {"quad": RobotType(quad), "lattice": RobotType(lat)}


def _server(slots, K=50, T=2000, budget=None, rounds=1):
    params = SimpleNamespace(checkpoint_every=K, max_steps=T, turn_period=500)
    ticks = itertools.count()
    clock = lambda: next(ticks) * 1e-3  # noqa: E731
    return Server(_robots(), slots, params, hbm_budget=budget, tick_segments=rounds,
                  backend_factory=lambda st, types, p: FakeBackend(st, types, p), clock=clock)


def _windows_of(backend, slot, kind):
    return [tuple(c[1][slot]) for c in backend.calls if c[0] == kind and c[1][slot][0] < c[1][slot][1]]


@pytest.mark.parametrize("steps,K,rounds", [(1000, 50, 1), (137, 50, 1), (2, 50, 1), (51, 50, 1),
                                            (52, 50, 1), (300, 7, 1), (1000, 50, 4), (333, 7, 3)])
def test_windows_reproduce_forward_and_backward_segments(steps, K, rounds):
    srv = _server({"quad": 1}, K=K, rounds=rounds)
    srv.submit(Request(kind="quad", steps=steps, grad=True, seed=3))
    res = srv.drain()
    assert len(res) == 1 and res[0].grads == [("grad-of", 0)]
    be = srv.pools[0].backend
    t_last = steps - 1
    fwd = _windows_of(be, 0, "forward")
    exp_f = [(t, min(t + rounds * K, t_last), t // K, 0) for t in range(0, t_last, rounds * K)]
    assert fwd == exp_f
    n_seg = (t_last + K - 1) // K
    exp_b = [(s * K, min(s * K + K, t_last), s, int(s == n_seg - 1)) for s in range(n_seg - 1, -1, -1)]
    assert _windows_of(be, 0, "backward") == exp_b
    assert res[0].loss == pytest.approx(3 + 0.5 * steps)


def test_late_request_is_folded_into_running_launches():
    srv = _server({"quad": 2, "lattice": 1})
    srv.submit(Request(kind="quad", steps=1000, seed=1))
    for _ in range(4):
        srv.tick()
    srv.submit(Request(kind="quad", steps=400, seed=2))
    srv.submit(Request(kind="lattice", steps=300, seed=3))
    srv.tick()
    # the quad pool's next launch advances the first request at t = 200 and
    # starts the second at t = 0 in the same launch
    quad_pool = [p for p in srv.pools if p.slots[0].kind == "quad"][0]
    last = [c for c in quad_pool.backend.calls if c[0] == "forward"][-1][1]
    assert tuple(last[0][:2]) == (200, 250) and tuple(last[1][:2]) == (0, 50)
    res = {r.rid: r for r in srv.drain()}
    assert sorted(res) == [0, 1, 2]
    assert res[1].done < res[0].done      # the short late request finishes first


def test_admission_waits_for_slots_and_lets_other_types_pass():
    srv = _server({"quad": 1, "lattice": 1})
    a = srv.submit(Request(kind="quad", steps=500))
    b = srv.submit(Request(kind="quad", steps=200))
    c = srv.submit(Request(kind="lattice", steps=200))
    srv.tick()
    active = {s.req.rid for p in srv.pools for s in p.slots if s.req is not None}
    assert active == {a, c} and [r.rid for r in srv.queue] == [b]
    res = srv.drain()
    order = [r.rid for r in sorted(res, key=lambda r: r.done)]
    assert order.index(a) < order.index(b)


def test_admission_by_hbm_footprint():
    types = _robots()
    fp = footprint_bytes(types["quad"].robot, 1000, False, 50)
    srv = _server({"quad": 4}, budget=int(1.5 * fp))
    ids = [srv.submit(Request(kind="quad", steps=1000)) for _ in range(3)]
    srv.tick()
    active = [s.req.rid for s in srv.pools[0].slots if s.req is not None]
    assert active == [ids[0]] and srv.used_bytes == fp
    res = srv.drain()
    assert len(res) == 3 and srv.used_bytes == 0
    done = sorted(res, key=lambda r: r.done)
    assert [r.rid for r in done] == ids           # one at a time, in order
    with pytest.raises(ValueError):
        srv.submit(Request(kind="quad", steps=5000))


def test_poisson_requests_statistics():
    rng = np.random.default_rng(7)
    reqs = poisson_requests(rng, 200.0, 50.0, ["a", "b"], [0.25, 0.75])
    assert abs(len(reqs) / 50.0 - 200.0) < 200.0 * 0.05
    gaps = np.diff([r.arrival for r in reqs])
    assert abs(gaps.mean() - 1 / 200.0) < 0.05 / 200.0
    steps = np.array([r.steps for r in reqs])
    assert steps.min() >= 100 and steps.max() <= 2000
    assert abs(np.mean([r.grad for r in reqs]) - 0.2) < 0.03
    assert abs(np.mean([r.kind == "a" for r in reqs]) - 0.25) < 0.03


def test_stats_report_percentiles():
    srv = _server({"quad": 2})
    for k in range(6):
        srv.submit(Request(kind="quad", steps=60 + 40 * k))
    srv.drain()
    st = srv.stats()
    lat = sorted(r.latency for r in srv.results)
    assert st["requests"] == 6
    assert st["p50_ms"] == pytest.approx(np.percentile(lat, 50) * 1e3)
    assert st["p99_ms"] == pytest.approx(np.percentile(lat, 99) * 1e3)
    assert st["env_substeps_per_s"] > 0


def test_open_loop_run_serves_every_request_with_independent_pools():
    srv = _server({"quad": 2, "lattice": 2}, rounds=2)
    rng = np.random.default_rng(4)
    reqs = poisson_requests(rng, 2000.0, 0.02, ["quad", "lattice"], [0.5, 0.5], steps_lo=50, steps_hi=500)
    res, st = srv.run(reqs)
    assert sorted(r.rid for r in res) == list(range(len(reqs)))
    assert st["requests"] == len(reqs) and all(r.latency >= 0 for r in res)
    assert all(r.done >= r.admitted >= r.arrival - 1e-9 for r in res)
    # the pools ticked independently: both launched
    for p in srv.pools:
        assert any(c[0] == "forward" for c in p.backend.calls)


class FakeMpmBackend:
    """Whole-rollout MPM slots: a request finishes `lag` done() polls after it
    starts; its loss is a function of the request."""

    def __init__(self, mt, n, T, K, lag=2):
        self.started = []
        self.polls = [0] * n
        self.lag = lag

    def start(self, slot, req):
        self.started.append((slot, req.rid))
        self.polls[slot] = 0

    def done(self, slot):
        self.polls[slot] += 1
        return self.polls[slot] > self.lag

    def result(self, slot, req):
        return float(req.seed), np.zeros((2, 3)), ({"act": req.rid} if req.grad else None)

    def close(self):
        pass


def test_mpm_requests_are_served_by_whole_rollout_slots():
    """MPM requests take a free slot of their type at once (no ticks), run
    while other slots start and finish, and mix with mass-spring pools."""
    from cls_b200.serving import MpmType
    obj, spr = robot_design.quadruped_lattice()
    types = {"quad": RobotType(Robot.actuated_outputs(obj, spr, hidden=[8])),
             "blob": MpmType(np.zeros((4, 3)), np.zeros(4, dtype=np.int32), n_muscles=1)}
    params = SimpleNamespace(checkpoint_every=10, max_steps=100, turn_period=50)
    srv = Server(types, {"quad": 1, "blob": 2}, params, backend_factory=FakeBackend, streams=False,
                 mpm_backend_factory=FakeMpmBackend)
    reqs = [Request("blob", 50, grad=True, seed=3), Request("blob", 60, seed=4), Request("blob", 70, seed=5),
            Request("quad", 30, seed=6)]
    for r in reqs:
        srv.submit(r)
    res = {r.rid: r for r in srv.drain()}
    assert sorted(res) == [0, 1, 2, 3]
    mpm_pool = [p for p in srv.pools if getattr(p, "kind", None) == "blob"][0]
    # two slots: the third request waited for a slot, then reused one
    assert [rid for _, rid in mpm_pool.backend.started] == [0, 1, 2]
    assert res[0].loss == 3.0 and res[0].grads == {"act": 0}
    assert res[1].grads is None and res[2].loss == 5.0
    assert srv.used_bytes == 0
