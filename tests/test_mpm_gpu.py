"""CUDA MLS-MPM (through the C ABI) against the reference's own 2D kernels
(golden) and the FP64 oracle's gradients.  Tolerances as for the mass-spring
path: FP64 build 1e-9 (forward) / 1e-8 (gradients), FP32 build 1e-5 / 1e-4."""
import numpy as np
import pytest

from helpers import max_rel, rel_err
from oracle.mpm_oracle import MPMOracle
from test_mpm_oracle import _golden, body3d

pytestmark = pytest.mark.gpu
TOL = {64: (1e-9, 1e-8), 32: (1e-5, 1e-4)}


def _batch2d(g, precision, material="fixed_corotated", K=7):
    from cls_b200.mpm import MPMBatch
    steps, B = int(g["steps"]), int(g["B"])
    b = MPMBatch(g["objects"], g["actuator_id"], B, dim=2, n_muscles=4, max_steps=steps,
                 n_grid=int(g["n_grid"]), bound=int(g["bound"]), material=material,
                 precision=precision, checkpoint_every=K, dt=float(g["dt"]),
                 gravity=float(g["gravity"]), p_vol=float(g["p_vol"]), mu=float(g["mu"]),
                 la=float(g["la"]), act_strength=float(g["act_strength"]), mass=1.0)
    b.set_actuation(g["actuation"][:steps])
    return b, steps


@pytest.mark.parametrize("precision", [64, 32])
def test_mpm2d_forward_matches_reference_golden(precision):
    g = _golden()
    b, steps = _batch2d(g, precision)
    b.forward(steps)
    x, v, C, F = b.final_state()
    tf = TOL[precision][0]
    assert max_rel(x, g["x"][steps]) < tf
    assert max_rel(v, g["v"][steps]) < max(tf, 1e-12) * 100
    assert max_rel(F, g["F"][steps]) < tf * 10
    b.close()


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("material", ["fixed_corotated", "neo_hookean"])
def test_mpm2d_gradients_match_oracle(material, precision):
    g = _golden()
    steps, B = int(g["steps"]), int(g["B"])
    o = MPMOracle(g["objects"], g["actuator_id"], B, steps, dim=2, n_grid=int(g["n_grid"]),
                  dt=float(g["dt"]), p_vol=float(g["p_vol"]), mu=float(g["mu"]), la=float(g["la"]),
                  act_strength=float(g["act_strength"]), gravity=float(g["gravity"]),
                  bound=int(g["bound"]), n_muscles=4, material=material)
    o.act[...] = g["actuation"][:steps]
    pw = (g["actuator_id"] >= 0) * 1.0 + 0.1
    o.loss_pw[...] = pw
    o.loss_w[steps] = 1.0
    o.loss_w[steps // 2] = 0.5
    o.target[...] = 0.5
    L = o.run(steps)
    b, _ = _batch2d(g, precision, material)
    b.set_loss(o.loss_w, o.target, pw)
    Lg = b.run(steps)
    tf, tg = TOL[precision]
    assert abs(Lg - L) <= tf * 10 * abs(L)
    gr = b.grads()
    assert rel_err(gr["act"], o.gact) < tg
    assert rel_err(gr["x0"], o.gx0) < tg
    assert rel_err(gr["v0"], o.gv0) < tg
    assert rel_err(gr["F0"], o.gF0) < tg
    assert rel_err(gr["C0"], o.gC0) < tg
    b.close()


@pytest.mark.parametrize("precision,tile,order", [(64, 0, "cells"), (32, 0, "cells"), (64, 256, "cells"),
                                                  (32, 256, "cells"), (64, 48, "cells"), (64, -1, "cells"),
                                                  (32, -1, "cells"), (64, 0, "base_runs"),
                                                  (32, 0, "base_runs")])
def test_mpm3d_neo_hookean_fibre_matches_oracle(precision, tile, order):
    """tile 0 / -1: L1 gathers and vector reductions straight to the grid
    (default); 256: warp-private tiles for gathers and scatters; 48: a capacity
    that some warps' boxes exceed (mixed tiled / global); order base_runs:
    particles sorted by base cell, runs of a warp summed by shuffles before
    the reductions."""
    from cls_b200.mpm import MPMBatch
    rng = np.random.default_rng(1)
    pts, musc, fib = body3d(rng)
    steps, B = 12, 2
    kw = dict(dim=3, n_grid=24, dt=2e-4, p_vol=1.0, mu=3846.0, la=5769.0, act_strength=500.0,
              gravity=-10.0, bound=3)
    o = MPMOracle(pts, musc, B, steps, material="neo_hookean", fibre=fib, n_muscles=4, **kw)
    o.act[...] = rng.uniform(-1, 1, o.act.shape)
    o.v[0] = rng.normal(scale=0.05, size=o.v[0].shape)
    pw = (musc >= 0) * 1.0 + 0.2
    o.loss_pw[...] = pw
    o.loss_w[steps] = 1.0
    o.loss_w[5] = 0.3
    o.target[...] = 0.45
    L = o.run(steps)
    b = MPMBatch(pts, musc, B, fibre=fib, n_muscles=4, max_steps=steps, material="neo_hookean",
                 precision=precision, checkpoint_every=5, mass=1.0, tile_nodes=tile, particle_order=order,
                 **kw)
    b.set_state(np.broadcast_to(pts, (B,) + pts.shape), o.v[0])
    b.set_actuation(o.act)
    b.set_loss(o.loss_w, o.target, pw)
    Lg = b.run(steps)
    tf, tg = TOL[precision]
    assert abs(Lg - L) <= tg * abs(L)  # the loss bar: 1e-4 (FP32), 1e-8 (FP64)
    x, _, _, _ = b.final_state()
    assert max_rel(x, o.x[steps]) < tf  # trajectory bar: 1e-5 (FP32), 1e-9 (FP64)
    gr = b.grads()
    for name, ref in (("act", o.gact), ("x0", o.gx0), ("v0", o.gv0), ("F0", o.gF0)):
        assert rel_err(gr[name], ref) < tg, name
    b.close()


def test_mpm_checkpoint_interval_and_graph_replay():
    import torch
    g = _golden()
    ref, steps = _batch2d(g, 64, K=24)
    w = np.zeros(steps + 1)
    w[steps] = 1.0
    tgt = np.full((steps + 1, int(g["B"]), 2), 0.5)
    pw = (g["actuator_id"] >= 0) * 1.0 + 0.1
    ref.set_loss(w, tgt, pw)
    L0 = ref.run(steps)
    ga0 = ref.grads()["act"]
    for K in (1, 5):
        b, _ = _batch2d(g, 64, K=K)
        b.set_loss(w, tgt, pw)
        assert b.run(steps) == pytest.approx(L0, rel=1e-12)
        assert rel_err(b.grads()["act"], ga0) < 1e-10
        b.close()
    b, _ = _batch2d(g, 64, K=8)
    b.set_loss(w, tgt, pw)
    s = torch.cuda.Stream()
    b.set_stream(s.cuda_stream)
    b.graph_capture(steps)
    b.graph_launch()
    b.graph_launch()
    torch.cuda.synchronize()
    assert b.loss() == pytest.approx(L0, rel=1e-12)
    assert rel_err(b.grads()["act"], ga0) < 1e-10


@pytest.mark.parametrize("order", ["cells", "base_runs"])
@pytest.mark.parametrize("precision", [64, 32])
def test_mpm3d_legged_body_64_grid_50_substeps_matches_oracle(precision, order):
    """The benchmark configuration (64^3 grid, ~29.5k particles, 16 fibre
    muscle groups, neo-Hookean, dt 1e-4) over 50 substeps, K = 10, against
    the FP64 oracle whose adjoint the finite-difference test pins on the same
    body (tests/test_mpm_oracle.py)."""
    from cls_b200.mpm import MPMBatch
    from test_mpm_oracle import legged64_oracle
    steps = 50
    o, pos, mus, fib = legged64_oracle(steps)
    L = o.run(steps)
    E, nu = 1e4, 0.3
    b = MPMBatch(pos, mus, 1, dim=3, fibre=fib, n_muscles=16, max_steps=steps, n_grid=64, bound=3,
                 material="neo_hookean", precision=precision, checkpoint_every=10, dt=1e-4, gravity=-10.0,
                 p_vol=1.0, mu=E / (2 * (1 + nu)), la=E * nu / ((1 + nu) * (1 - 2 * nu)), act_strength=1e3,
                 mass=1.0, particle_order=order)
    b.set_state(pos[None])
    b.set_actuation(o.act)
    b.set_loss(o.loss_w, o.target, (mus >= 0) * 1.0 + 0.1)
    Lg = b.run(steps)
    tf, tg = TOL[precision]
    assert abs(Lg - L) <= tg * abs(L)  # the loss bar: 1e-4 (FP32), 1e-8 (FP64)
    x, _, _, _ = b.final_state()
    assert max_rel(x, o.x[steps]) < tf  # trajectory bar: 1e-5 (FP32), 1e-9 (FP64)
    gr = b.grads()
    for name, ref in (("act", o.gact), ("x0", o.gx0), ("v0", o.gv0), ("F0", o.gF0)):
        assert rel_err(gr[name], ref) < tg, name
    b.close()


@pytest.mark.parametrize("precision", [64, 32])
def test_mpm3d_base_runs_long_runs_match_oracle(precision):
    """Dense clusters (60 particles per base cell: runs as long as a warp,
    runs broken by motion) through the base-cell order's run sums, against
    the oracle and against the cells order."""
    from cls_b200.mpm import MPMBatch
    rng = np.random.default_rng(7)
    n_grid, dx = 24, 1.0 / 24
    # each cluster inside one base cell (centred on a node; a particle's base
    # cell is floor(x / dx - 0.5)): runs of 60 lanes, cut into a full warp
    # and the rest; the edge particles leave the base cell within the steps
    centres = np.array([[10.0, 7.0, 11.0], [12.0, 7.0, 11.0], [11.0, 9.0, 12.0]]) * dx
    pts = np.concatenate([c + rng.uniform(-0.499, 0.499, size=(60, 3)) * dx for c in centres])
    musc = (np.arange(len(pts)) % 3) - 1
    fib = rng.normal(size=pts.shape)
    fib /= np.linalg.norm(fib, axis=1, keepdims=True)
    steps, B = 10, 2
    kw = dict(dim=3, n_grid=n_grid, dt=2e-4, p_vol=1.0, mu=3846.0, la=5769.0, act_strength=500.0,
              gravity=-10.0, bound=3)
    o = MPMOracle(pts, musc, B, steps, material="neo_hookean", fibre=fib, n_muscles=2, **kw)
    o.act[...] = rng.uniform(-1, 1, o.act.shape)
    o.v[0] = rng.normal(scale=0.2, size=o.v[0].shape)
    # weighted centre: the plain centre of mass does not move under internal
    # (actuation) stress, which would leave d loss / d act at round-off level
    pw = 1.0 + 0.3 * (np.arange(len(pts)) % 5)
    o.loss_pw[...] = pw
    o.loss_w[steps] = 1.0
    o.loss_w[4] = 0.3
    o.target[...] = 0.45
    L = o.run(steps)
    tf, tg = TOL[precision]
    out = {}
    for order in ("base_runs", "cells"):
        b = MPMBatch(pts, musc, B, fibre=fib, n_muscles=2, max_steps=steps, material="neo_hookean",
                     precision=precision, checkpoint_every=4, mass=1.0, particle_order=order, **kw)
        b.set_state(np.broadcast_to(pts, (B,) + pts.shape), o.v[0])
        b.set_actuation(o.act)
        b.set_loss(o.loss_w, o.target, pw)
        Lg = b.run(steps)
        assert abs(Lg - L) <= tg * abs(L)
        x = b.final_state()[0]
        assert max_rel(x, o.x[steps]) < tf
        gr = b.grads()
        for name, ref in (("act", o.gact), ("x0", o.gx0), ("v0", o.gv0), ("F0", o.gF0)):
            assert rel_err(gr[name], ref) < tg, (order, name)
        out[order] = (Lg, x)
        b.close()
    if precision == 64:
        assert out["base_runs"][0] == pytest.approx(out["cells"][0], rel=1e-12)
        assert max_rel(out["base_runs"][1], out["cells"][1]) < 1e-12
