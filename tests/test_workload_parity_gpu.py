"""The benchmarked configurations' arithmetic against the FP64 oracle.

Each case runs the CUDA path through the C ABI and one FP64 oracle per robot
type (oracle/ms_oracle.c, pinned to the reference's own kernels by the golden
vectors) on the same seeded inputs: the robots' rest poses plus noise,
targets held per turn period, Xavier-uniform weights.  Physics and controller
are the configurations': dt 2e-3, gravity -9.8, ground at 0 with friction 0.5,
damping 0.99 per substep, tanh controllers, 8 sinusoid inputs
(multitask/solver_mass_spring.py:86-148, multitask/nn.py:130-150).  The
velocity and rotation loss windows open after run_period = 30 substeps so that
100-substep rollouts carry loss and gradients.

Tolerances (the configuration's bar): FP64 build rel 1e-9 on trajectories
and losses, 1e-8 on gradients; FP32 build rel 1e-5 on trajectories, rel 1e-4
on the loss and on the weight, bias, initial-position and initial-velocity
gradients (2-norm relative, worst layer / robot / env).
"""
import numpy as np
import pytest

from helpers import WorkloadCase

pytestmark = pytest.mark.gpu

TOL = {64: dict(traj=1e-9, loss=1e-9, grad=1e-8), 32: dict(traj=1e-5, loss=1e-4, grad=1e-4)}


def _params(steps, K, precision, **over):
    import cls_b200
    from cls_b200 import workloads
    kw = workloads._params(steps, K, precision=precision)
    kw.update(over)
    return cls_b200.default_params(**kw)


def _lattices(sizes=(60, 250, 700), hidden=(128, 128)):
    from cls_b200 import robot_design
    from cls_b200.batch import Robot
    rng = np.random.default_rng(0)
    out = []
    for n in sizes:
        o, s = robot_design.random_lattice(rng, n)
        out.append(Robot.actuated_outputs(o, s, hidden=list(hidden)))
    return out


def _check(robots, env_robot, steps, K, precision, path="per_env", traj_steps=100, **over):
    case = WorkloadCase(robots, env_robot, _params(steps, K, precision, **over), seed=5, path=path)
    try:
        if path == "batched":
            assert case.b.controller_batched
        case.run_oracles(steps)
        _, err = case.errors(steps, traj_steps=min(traj_steps, steps))
    finally:
        case.close()
    tol = TOL[precision]
    assert err["traj"] < tol["traj"], err
    assert err["loss"] < tol["loss"], err
    for k in ("gW", "gb", "gx0", "gv0"):
        assert err[k] < tol["grad"], (k, err)
    return err


@pytest.mark.parametrize("precision", [64, 32])
def test_uneven_lattices_2x128_tanh_100_substeps(precision):
    """Three random lattices of different sizes (60, 250, 700 vertices) in one
    batch, each its own robot type and controller (the uneven batch's form)."""
    _check(_lattices(), [0, 1, 2], 100, 50, precision, run_period=30)


@pytest.mark.parametrize("precision", [64, 32])
def test_uneven_lattices_300_substeps_six_segments(precision):
    """The same batch over six checkpoint segments of 50 (the uneven
    benchmark's interval), with the benchmark's run period."""
    _check(_lattices(), [0, 1, 2], 300, 50, precision, run_period=100)


@pytest.mark.parametrize("precision", [64, 32])
def test_quadruped_1x64_tanh_32_envs(precision):
    from cls_b200 import robot_design
    from cls_b200.batch import Robot
    obj, spr = robot_design.quadruped_lattice()
    _check([Robot.actuated_outputs(obj, spr, hidden=[64])], [0] * 32, 100, 50, precision, run_period=30)


@pytest.mark.parametrize("path", ["per_env", "batched"])
@pytest.mark.parametrize("precision", [64, 32])
def test_spider_2x256_tanh_both_controller_paths(precision, path):
    from cls_b200 import robot_design
    from cls_b200.batch import Robot
    obj, spr = robot_design.spider_lattice()
    _check([Robot.actuated_outputs(obj, spr, hidden=[256, 256])], [0] * 64, 100, 100, precision, path=path,
           run_period=30)


@pytest.mark.parametrize("precision", [64, 32])
def test_one_lattice_full_2000_substep_episode(precision):
    """The uneven benchmark's horizon: 2000 substeps, checkpoint every 50,
    on its 700-vertex lattice (trajectory compared over the first 100)."""
    _check(_lattices()[2:], [0], 2000, 50, precision)
