"""FP64 MLS-MPM oracle: forward against the reference's own 2D kernels (golden
made by tests/golden/make_golden.py) and reverse pass against central finite
differences, in 2D (fixed-corotated, neo-Hookean) and 3D (neo-Hookean with
fibre actuation)."""
import numpy as np
import pytest

from helpers import GOLDEN, max_rel
from oracle.mpm_oracle import MPMOracle


def _golden():
    g = np.load(GOLDEN + "/mpm2d_ref.npz")
    return {k: g[k] for k in g.files}


def _oracle2d(g, material="fixed_corotated"):
    steps, B = int(g["steps"]), int(g["B"])
    o = MPMOracle(g["objects"], g["actuator_id"], B, steps, dim=2, n_grid=int(g["n_grid"]),
                  dt=float(g["dt"]), p_vol=float(g["p_vol"]), mu=float(g["mu"]), la=float(g["la"]),
                  act_strength=float(g["act_strength"]), gravity=float(g["gravity"]),
                  bound=int(g["bound"]), n_muscles=4, material=material)
    o.act[...] = g["actuation"][:steps]
    return o, steps


def test_mpm2d_forward_matches_reference_kernels():
    g = _golden()
    o, steps = _oracle2d(g)
    o.forward(steps)
    for name in ("x", "v", "C", "F"):
        assert max_rel(getattr(o, name), g[name]) < 1e-12, name


def body3d(rng, nx=4, ny=3, nz=3, ppc=2, origin=(0.4, 0.2, 0.4), n_grid=24):
    """A small voxelised box, ppc^3 particles per cell, legs = lower layer."""
    dx = 1.0 / n_grid
    pts, musc = [], []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                for a in range(ppc):
                    for b in range(ppc):
                        for c in range(ppc):
                            pts.append((origin[0] + (i + (a + 0.5) / ppc) * dx,
                                        origin[1] + (j + (b + 0.5) / ppc) * dx,
                                        origin[2] + (k + (c + 0.5) / ppc) * dx))
                            musc.append((i % 2) + 2 * (k % 2) if j == 0 else -1)
    fib = rng.normal(size=(len(pts), 3))
    fib /= np.linalg.norm(fib, axis=1, keepdims=True)
    return np.array(pts), np.array(musc), fib


def _fd(o, steps, arrays, rng, n=4, h=1e-6, rtol=2e-4):
    grads = {k: gref.copy() for k, (arr, gref, _) in arrays.items()}
    L0 = o.compute_loss(steps)
    atol = 50 * 1e-16 * max(abs(L0), 1.0) / h      # central-difference round-off
    for name, (arr, _, lead) in arrays.items():
        for _ in range(n):
            idx = tuple(int(rng.integers(s)) for s in arr.shape[lead:])
            full = (0,) * lead + idx
            old = arr[full]
            arr[full] = old + h
            o.forward(steps)
            lp = o.compute_loss(steps)
            arr[full] = old - h
            o.forward(steps)
            lm = o.compute_loss(steps)
            arr[full] = old
            fd = (lp - lm) / (2 * h)
            an = grads[name][idx]
            assert abs(fd - an) <= rtol * max(abs(fd), abs(an)) + atol, (name, idx, fd, an)


@pytest.mark.parametrize("material", ["fixed_corotated", "neo_hookean"])
def test_mpm2d_gradients_match_finite_differences(material):
    g = _golden()
    o, steps = _oracle2d(g, material)
    o.loss_pw[...] = (g["actuator_id"] >= 0) * 1.0 + 0.1
    o.loss_w[steps] = 1.0
    o.loss_w[steps // 2] = 0.5
    o.target[...] = 0.5
    o.run(steps)
    rng = np.random.default_rng(0)
    _fd(o, steps, {"act": (o.act, o.gact, 0), "x0": (o.x, o.gx0, 1), "v0": (o.v, o.gv0, 1),
                   "F0": (o.F, o.gF0, 1), "C0": (o.C, o.gC0, 1)}, rng)


def test_mpm3d_neo_hookean_fibre_gradients_match_finite_differences():
    rng = np.random.default_rng(1)
    pts, musc, fib = body3d(rng)
    steps, B = 10, 2
    o = MPMOracle(pts, musc, B, steps, dim=3, n_grid=24, dt=2e-4, p_vol=1.0, mu=3846.0,
                  la=5769.0, act_strength=500.0, gravity=-10.0, bound=3, material="neo_hookean",
                  fibre=fib, n_muscles=4)
    o.act[...] = rng.uniform(-1, 1, o.act.shape)
    o.v[0] = rng.normal(scale=0.05, size=o.v[0].shape)
    o.loss_pw[...] = (musc >= 0) * 1.0 + 0.2
    o.loss_w[steps] = 1.0
    o.target[...] = 0.45
    o.run(steps)
    _fd(o, steps, {"act": (o.act, o.gact, 0), "x0": (o.x, o.gx0, 1), "v0": (o.v, o.gv0, 1),
                   "F0": (o.F, o.gF0, 1)}, rng, n=4)


def legged64_oracle(steps=50, seed=0):
    """The 3D MPM benchmark's body and solver: the voxelised legged body on a
    64^3 grid (dx = 1/64, ~29.5k particles), neo-Hookean E = 1e4, nu = 0.3,
    fibre actuation of 16 muscle groups, dt = 1e-4, sticky walls; one env,
    seeded actuation in [-1, 1]; loss: the muscle-weighted centre at the last
    step towards a point 0.05 ahead."""
    from cls_b200 import workloads
    pos, mus, fib = workloads.legged_body()
    E, nu = 1e4, 0.3
    o = MPMOracle(pos, mus, 1, steps, dim=3, n_grid=64, dt=1e-4, p_vol=1.0, mu=E / (2 * (1 + nu)),
                  la=E * nu / ((1 + nu) * (1 - 2 * nu)), act_strength=1e3, gravity=-10.0, bound=3,
                  material="neo_hookean", fibre=fib, n_muscles=16)
    rng = np.random.default_rng(seed)
    o.act[...] = rng.uniform(-1, 1, o.act.shape)
    o.loss_pw[...] = (mus >= 0) * 1.0 + 0.1
    o.loss_w[steps] = 1.0
    o.target[...] = pos.mean(axis=0) + np.array([0.05, 0.0, 0.0])
    return o, pos, mus, fib


def test_mpm3d_legged_body_64_grid_50_substeps_matches_finite_differences():
    """The benchmark body over 50 substeps: the hand-written adjoint against
    FP64 central differences on the actuation and initial-position entries
    with the largest gradients (and one random entry of each), at the FD
    tests' rel 2e-4 (truncation of the quadratic B-spline weights)."""
    steps = 50
    o, pos, mus, fib = legged64_oracle(steps)
    L0 = o.run(steps)
    rng = np.random.default_rng(3)
    checks = []
    for arr, g, h in ((o.act, o.gact, 1e-4), (o.x, o.gx0, 1e-6)):
        ga = g.reshape(-1)
        picks = list(np.argsort(-np.abs(ga))[:2]) + [int(rng.integers(ga.size))]
        for flat in picks:
            idx = np.unravel_index(flat, g.shape)
            full = idx if arr is o.act else (0,) + idx
            checks.append((arr, full, float(g[idx]), h))
    for arr, full, an, h in checks:
        old = arr[full]
        arr[full] = old + h
        o.forward(steps)
        lp = o.compute_loss(steps)
        arr[full] = old - h
        o.forward(steps)
        lm = o.compute_loss(steps)
        arr[full] = old
        fd = (lp - lm) / (2 * h)
        atol = 50 * 1e-16 * abs(L0) / h
        assert abs(fd - an) <= 2e-4 * max(abs(fd), abs(an)) + atol, (full, fd, an)
