"""bench.py's configuration blocks: every configuration names its workload
with the keys the driver compares (no model keys), and the checkpoint default
of each configuration (50; the quadruped and spider episodes as one segment)."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _args(argv):
    sys.path.insert(0, ROOT)
    import bench
    old = sys.argv
    sys.argv = ["bench.py"] + argv
    try:
        return bench, bench.parse()
    finally:
        sys.argv = old


@pytest.mark.parametrize("config", ["uneven", "quadruped", "spider", "mpm", "serve"])
def test_config_block(config):
    bench, a = _args(["--config", config])
    c = bench.config_dict(a, 1)
    assert isinstance(c["workload"], str) and c["workload"]
    assert "model" not in c and "checkpoint_every" in c and "l2" in c
    assert c["parallelism"].endswith("x1 (no data-path collective)")
    assert bench.METRICS[config] and bench.UNIT == "env-substeps/s"
    # the reference arm reports the same block for the same arguments
    assert bench.config_dict(a, 1) == c


def test_checkpoint_defaults():
    _, a = _args([])
    assert (a.config, a.substeps, a.checkpoint, a.robots) == ("uneven", 2000, 50, 512)
    for config, subs in (("quadruped", 1000), ("spider", 1000)):
        _, a = _args(["--config", config])
        assert a.checkpoint == a.substeps == subs
    _, a = _args(["--config", "spider", "--checkpoint", "50"])
    assert a.checkpoint == 50
    _, a = _args(["--config", "mpm"])
    assert a.checkpoint == 50


def test_algorithmic_bytes_of_the_replaying_recompute():
    """With the controller replayed from the first pass's records, the
    recompute moves no controller weights and the first pass writes every
    substep's controller records on top of its weight stream."""
    sys.path.insert(0, ROOT)
    import numpy as np
    from cls_b200 import robot_design
    from cls_b200.batch import Robot
    from cls_b200 import workloads
    rng = np.random.default_rng(0)
    robots = []
    for n in (60, 300):
        obj, spr = robot_design.random_lattice(rng, n)
        robots.append(Robot.actuated_outputs(obj, spr, hidden=[128, 128]))
    env_robot = [0, 1]
    base = workloads.algorithmic_bytes(robots, env_robot)
    rep = workloads.algorithmic_bytes(robots, env_robot, replay=True)
    widths = [workloads._widths(r) for r in robots]
    wbytes = sum(sum(w[l + 1] * (-(-w[l] // 4) * 4) for l in range(len(w) - 1)) * 4 for w in widths)
    rows = sum(sum(w[1:]) * 4 for w in widths)
    inputs = sum(w[0] * 4 for w in widths)
    outputs = sum(w[-1] * 4 for w in widths)
    assert rep["reverse"] == base["reverse"]
    assert rep["forward"] == pytest.approx(base["forward"] + inputs + rows)
    assert rep["recompute"] == pytest.approx(base["recompute"] - wbytes - inputs - rows + outputs)
    assert rep["recompute"] < 0.2 * base["recompute"]
