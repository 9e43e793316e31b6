"""Batched controller path (per-substep step kernels + one GEMM per layer over
all envs of a robot type; FP32 on the tensor cores with a 3xTF32 split, FP64
as SIMT tiles) against the reference-generated golden vectors, the FP64
oracle and the fused per-env path.

Tolerances are the mass-spring suite's: FP64 1e-9 on trajectories and
losses, 1e-8 on gradients; FP32 rel 1e-5 on trajectories over these
<= 48-substep rollouts, rel 1e-4 on losses and gradients.
"""
import numpy as np
import pytest

from helpers import (TRAIN_CASES, batch_from_golden, load_golden, many_env_batch, max_rel,
                     oracle_from_golden, rel_err)

pytestmark = pytest.mark.gpu

TOL = {64: dict(traj=1e-9, loss=1e-9, grad=1e-8), 32: dict(traj=1e-5, loss=1e-4, grad=1e-4)}


def _batched(g, precision, K, **over):
    b = batch_from_golden(g, precision=precision, K=K, **over)
    b.set_controller_path("batched")
    assert b.controller_batched
    return b


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("case", TRAIN_CASES)
def test_batched_forward_matches_golden(case, precision):
    g = load_golden(case)
    steps = int(g["steps"])
    b = _batched(g, precision, K=7)
    b.forward(steps)
    terms, env = b.loss()
    obs = b.observables()
    tol = TOL[precision]
    assert max_rel(obs["center"], g["center"]) < tol["traj"]
    assert max_rel(obs["height"], g["height"]) < tol["traj"]
    B, N = int(g["B"]), g["objects"].shape[0]
    gx = g["x"].reshape(g["x"].shape[0], B * N, 3)
    assert max_rel(b.trajectory()[:steps], gx[:steps]) < tol["traj"]
    xf, _ = b.final_state()
    assert max_rel(xf, gx[steps - 1]) < tol["traj"]
    assert abs(terms["total"] - float(g["loss"])) <= tol["loss"] * abs(float(g["loss"]))
    b.close()


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("case", TRAIN_CASES)
def test_batched_gradients_match_oracle(case, precision):
    g = load_golden(case)
    steps = int(g["steps"])
    o = oracle_from_golden(g)
    o.run(steps)
    b = _batched(g, precision, K=9)
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


def _run(b, steps, n_layers):
    loss = b.simulate(steps)
    grads = [b.get_grads(0, l) for l in range(n_layers)]
    x, _ = b.final_state()
    gx0, _ = b.state_grads()
    return loss, grads, x, gx0


def test_batched_equals_per_env_with_partial_tiles_fp64():
    """300 envs (tiles of 64 envs: four full and one partial) and hidden
    widths 70 and 50 (partial output tiles); several checkpoint segments."""
    hidden, steps = [70, 50], 40
    ref = many_env_batch(64, 300, hidden, 9, 48, "per_env")
    assert not ref.controller_batched
    r_loss, r_grads, r_x, r_gx = _run(ref, steps, 3)
    ref.close()
    b = many_env_batch(64, 300, hidden, 9, 48, "auto")
    assert b.controller_batched          # >= 256 envs of one type: automatic
    loss, grads, x, gx = _run(b, steps, 3)
    b.close()
    tol = TOL[64]
    assert abs(loss - r_loss) <= tol["loss"] * abs(r_loss)
    assert max_rel(x, r_x) < tol["traj"]
    for (gW, gb), (rW, rb) in zip(grads, r_grads):
        assert rel_err(gW, rW) < tol["grad"] and rel_err(gb, rb) < tol["grad"]
    assert rel_err(gx, r_gx) < tol["grad"]


def test_batched_fp32_as_accurate_as_per_env_fp32():
    """The same 300-env batch with random Xavier weights and contact-heavy
    targets is ill-conditioned enough that FP32 itself (the fused per-env
    path, plain FP32 arithmetic) misses the FP64 gradients by ~2.5e-4.  The
    tensor-core path (3xTF32, FP32 accumulate) must agree with the FP32
    per-env path to 1e-4 and be no less accurate than it against FP64."""
    hidden, steps = [70, 50], 40
    runs = {}
    for prec, path in ((64, "per_env"), (32, "per_env"), (32, "batched")):
        b = many_env_batch(prec, 300, hidden, 9, 48, path)
        runs[(prec, path)] = _run(b, steps, 3)
        b.close()
    r64, p32, b32 = runs[(64, "per_env")], runs[(32, "per_env")], runs[(32, "batched")]
    assert abs(b32[0] - p32[0]) <= 1e-5 * abs(p32[0])
    assert max_rel(b32[2], p32[2]) < 1e-5
    for (gW, gb), (pW, pb), (rW, rb) in zip(b32[1], p32[1], r64[1]):
        assert rel_err(gW, pW) < 1e-4 and rel_err(gb, pb) < 1e-4
        assert rel_err(gW, rW) <= 1.25 * rel_err(pW, rW) + 1e-5
        assert rel_err(gb, rb) <= 1.25 * rel_err(pb, rb) + 1e-5
    assert rel_err(b32[3], p32[3]) < 1e-4
    assert rel_err(b32[3], r64[3]) <= 1.25 * rel_err(p32[3], r64[3]) + 1e-5


@pytest.mark.parametrize("precision", [64, 32])
def test_batched_single_segment_equals_segments(precision):
    """The batched path with the episode as one segment (records from the
    first pass, no recompute) against the same batch with K = 9."""
    hidden, steps = [70, 50], 40
    ref = many_env_batch(precision, 300, hidden, 9, 48, "batched")
    r_loss, r_grads, _, r_gx = _run(ref, steps, 3)
    ref.close()
    b = many_env_batch(precision, 300, hidden, 48, 48, "batched")
    b.profile(True)
    loss, grads, _, gx = _run(b, steps, 3)
    _, n = b.profile_read(reset=True)
    b.close()
    assert n["recompute"] == 0
    assert loss == r_loss                 # the same first pass
    tol = 1e-12 if precision == 64 else 1e-5
    for (gW, gb), (rW, rb) in zip(grads, r_grads):
        assert rel_err(gW, rW) < tol and rel_err(gb, rb) < tol
    assert rel_err(gx, r_gx) < tol


@pytest.mark.parametrize("precision", [64, 32])
def test_batched_direct_spring_gathers_equal_tables(precision):
    """The batched path's step kernels with the spring impulse table and with
    the direct gathers."""
    hidden, steps = [70, 50], 40
    runs = []
    for mode in (1, 0):
        b = many_env_batch(precision, 300, hidden, 9, 48, "batched")
        b.set_spring_tables(mode)
        runs.append(_run(b, steps, 3))
        b.close()
    same = 1e-12 if precision == 64 else 1e-5
    (l1, g1, x1, s1), (l0, g0, x0, s0) = runs
    assert abs(l1 - l0) <= same * abs(l0)
    assert max_rel(x1, x0) < same
    for (gW, gb), (rW, rb) in zip(g1, g0):
        assert rel_err(gW, rW) < same and rel_err(gb, rb) < same
    assert rel_err(s1, s0) < same


def test_batched_graph_replay_matches_eager():
    """The forward pass (spring gather, tensor-core GEMMs) is deterministic, so
    the replayed loss is identical; the atomic adds of the reverse pass
    (actuation gradients, split-K weight gradients) only change the gradients'
    rounding."""
    import torch
    b = many_env_batch(32, 260, [64], 10, 40, "batched")
    e_loss, e_grads, _, _ = _run(b, 30, 2)
    s = torch.cuda.Stream()
    b.set_stream(s.cuda_stream)
    b.graph_capture(30)
    for _ in range(2):
        b.graph_launch()
    b.synchronize()
    g_loss, _ = b.loss()
    assert g_loss["total"] == e_loss
    for l in range(2):
        gW, gb = b.get_grads(0, l)
        assert rel_err(gW, e_grads[l][0]) < 1e-5
        assert rel_err(gb, e_grads[l][1]) < 1e-5
    b.close()


def test_batched_profile_counts_gemm_launches():
    b = many_env_batch(32, 256, [64, 64], 10, 30, "batched")
    b.profile(True)
    b.simulate(20)
    ms, n = b.profile_read(reset=True)
    b.close()
    # forward: 19 substeps x 3 layers; recompute: 19 x 3; reverse: 19 x 3
    assert n["ctrl_gemm"] == 2 * 19 * 3
    assert n["ctrl_gemm_adj"] == 19 * 3
    assert ms["ctrl_gemm"] > 0 and ms["ctrl_gemm_adj"] > 0
