"""The library's slot scheduler (csrc/ms_sched.h, behind cls_admit /
cls_poll) on the CPU: a g++ build of it over a recording fake handle
(tests/sched_driver.cpp) must issue, request by request and tick by tick,
the launches of the Python scheduler (serving.Server / Pool) for the same
requests, and keep its admission rules (robot class, footprint budget,
unique ids, results held until release)."""
import json
import os
import shutil
import subprocess
from types import SimpleNamespace

import numpy as np
import pytest

from cls_b200.serving import Request, Server
from test_serving_cpu import FakeBackend, _robots

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "..", "complex-locomotion-skill-learning-via-differentiable-physics_b200", "csrc")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path_factory.mktemp("sched") / "sched_driver")
    subprocess.check_call([gxx, "-std=c++17", "-O1", "-Wall", "-Werror", "-I", CSRC, "-o", exe,
                           os.path.join(HERE, "sched_driver.cpp")])
    return exe


def run(exe, classes, T, K, rounds, commands):
    args = [exe, str(len(classes)), str(T), str(K), str(rounds)] + [str(c) for c in classes]
    out = subprocess.run(args, input="\n".join(commands) + "\n", capture_output=True, text=True, check=True)
    return [json.loads(line) for line in out.stdout.splitlines()]


class RecBackend(FakeBackend):
    """FakeBackend that logs each launch as {request id: window}."""

    def __init__(self, *a):
        super().__init__(*a)
        self.log = []

    def _log(self, kind, windows):
        self.log.append((kind, {self.req[i].rid: tuple(int(v) for v in windows[i])
                                for i in range(len(self.req)) if windows[i][0] < windows[i][1]}))

    def forward(self, windows, steps):
        super().forward(windows, steps)
        self._log("forward", windows)

    def backward(self, windows, steps):
        super().backward(windows, steps)
        self._log("backward", windows)


def python_plan(reqs, arrivals, n_slots, T, K, rounds, n_ticks):
    params = SimpleNamespace(checkpoint_every=K, max_steps=T, turn_period=500)
    backends = []

    def factory(st, types, p):
        backends.append(RecBackend(st, types, p))
        return backends[-1]

    srv = Server(_robots(), {"lattice": n_slots}, params, tick_segments=rounds, backend_factory=factory,
                 clock=lambda: 0.0)
    done = []
    for k in range(n_ticks):
        for (steps, grad), a in zip(reqs, arrivals):
            if a == k:
                srv.submit(Request("lattice", steps, grad=grad))
        done.append(sorted(r.rid for r in srv.tick()))
    return backends[0].log, done


def native_plan(exe, reqs, arrivals, n_slots, T, K, rounds, n_ticks):
    cmds = []
    for k in range(n_ticks + 1):
        for rid, ((steps, grad), a) in enumerate(zip(reqs, arrivals)):
            if a == k:
                cmds.append("admit %d 0 %d %d -1" % (rid, steps, int(grad)))
        cmds.append("poll")
    out = run(exe, [0] * n_slots, T, K, rounds, cmds)
    log, done, slot_of = [], [], {}
    for o in out:
        if "admit" in o:
            assert o["slot"] >= 0
            slot_of[o["slot"]] = o["admit"]
        elif "forward" in o or "backward" in o:
            kind = "forward" if "forward" in o else "backward"
            log.append((kind, {slot_of[w[0]]: tuple(w[1:5]) for w in o[kind]}))
        elif "done" in o:
            done.append(sorted(o["done"]))
    return log, done[1:]   # poll k + 1 completes the tick that poll k issued


REQS = [(120, True), (260, False), (51, True), (2, True), (300, True), (175, False), (101, True)]


@pytest.mark.parametrize("rounds", [1, 3])
@pytest.mark.parametrize("staggered", [False, True])
def test_native_scheduler_issues_the_python_schedulers_launches(driver, rounds, staggered):
    arrivals = [0, 0, 1, 3, 3, 5, 6] if staggered else [0] * len(REQS)
    n_ticks = 40
    py_log, py_done = python_plan(REQS, arrivals, 8, 400, 50, rounds, n_ticks)
    nat_log, nat_done = native_plan(driver, REQS, arrivals, 8, 400, 50, rounds, n_ticks)
    assert nat_log == py_log
    assert nat_done == py_done
    assert sorted(sum(nat_done, [])) == list(range(len(REQS)))   # every request finished once


def test_admission_by_class_and_budget(driver):
    out = run(driver, [0, 0, 1], 200, 50, 1, [
        "admit 1 2 100 0 -1",     # class of slot 2 (its only slot)
        "admit 2 2 100 0 -1",     # no free slot of that class
        "admit 3 0 100 1 1300",   # footprint 300 (gradients: x3): 1100 + 300 > 1300, refused
        "admit 3 0 100 1 1400",   # fits exactly
        "admit 4 1 150 0 1500",   # 1400 + 150 > 1500: refused
        "admit 5 1 100 0 1500",   # 1400 + 100 = 1500 fits
    ])
    slots = [o["slot"] for o in out if "admit" in o]
    assert slots == [2, -1, -1, 0, -1, 1]
    used = [o["used"] for o in out if "admit" in o]
    assert used == [1100, 1100, 1100, 1400, 1400, 1500]


def test_errors_results_and_release(driver):
    out = run(driver, [0, 0], 100, 50, 1, [
        "admit 7 0 60 0 -1",
        "admit 7 1 60 0 -1",      # duplicate id
        "admit 8 0 1 0 -1",       # steps < 2
        "admit 9 0 101 0 -1",     # steps > max_steps
        "admit 10 5 60 0 -1",     # no such slot
        "result 7",               # not finished
        "release 7",
        "poll", "rounds 2",       # tick in flight
        "poll", "poll",
        "result 7", "release 7", "release 7",
    ])
    errors = [o["error"] for o in out if "error" in o]
    assert errors[:4] == ["request id already admitted", "steps must be in [2, max_steps]",
                          "steps must be in [2, max_steps]", "robot slot out of range"]
    assert errors[4] == "the request has not finished"
    assert errors[5] == "only finished requests are released"
    assert errors[6] == "the tick length changes only with no tick in flight"
    assert errors[7] == "unknown request id"
    res = [o for o in out if "result" in o][0]
    assert res["slot"] == 0
    np.testing.assert_allclose(res["terms"], [k + 0.001 * 60 for k in range(8)])
    np.testing.assert_allclose(res["x"], [0, 7, 2, 0, 7, 5])
    # 60 steps: first pass of 59 substeps = windows [0, 50) and [50, 59), then done
    fw = [o["forward"] for o in out if "forward" in o]
    assert fw == [[[0, 0, 50, 0, 0, 60]], [[0, 50, 59, 1, 0, 60]]]
    assert [o for o in out if "loss" in o] == [{"loss": [[0, 60]]}]


def test_gradient_queries_need_a_controller_of_their_own(driver):
    # slots 0 and 1 share one robot entry (class -1 in the fake), slot 2 does not
    out = run(driver, [-1, -1, 0], 200, 50, 1, [
        "admit 1 0 100 1 -1",     # gradient query on a shared controller: refused
        "admit 2 0 100 0 -1",     # forward-only: fine
        "admit 3 2 100 1 -1",     # own controller: fine
    ])
    assert [o for o in out if "error" in o] == [
        {"error": "gradient queries need a slot whose robot entry (controller) no other env shares"}]
    assert [o["slot"] for o in out if "admit" in o] == [0, 2]
