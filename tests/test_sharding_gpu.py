"""Shared-controller sharding on one GPU: two shards of a batch, each
dividing its losses by the whole batch's env count (cls_set_loss_envs), give
gradients and losses that sum to the unsharded batch's (FP64, rel 1e-12);
summing the shards' device gradient buffers (cls_grad_buffers, the in-place
all-reduce's operands) and stepping Adam reproduces the unsharded Adam step;
and a one-rank NCCL group reduces the device buffers in place."""
import numpy as np
import pytest

from helpers import load_golden, params_from_golden, rel_err

pytestmark = pytest.mark.gpu


def _batch(g, envs, loss_envs=None):
    import cls_b200
    robot = cls_b200.Robot(g["objects"], g["springs"], robot_id=int(g["robot_id"]), hidden=[int(g["n_hidden"])])
    b = cls_b200.MassSpringBatch([robot], [0] * len(envs), params_from_golden(g, precision=64, K=7))
    b.set_state(g["x0"][envs].reshape(-1, 3))
    b.set_weights(0, 0, g["W1"], g["b1"])
    b.set_weights(0, 1, g["W2"], g["b2"])
    b.set_targets(g["target_v"][:, envs], g["target_h"][:, envs], g["target_c"][:, envs])
    if loss_envs:
        b.set_loss_envs(0, loss_envs)
    return b


def test_shards_sum_to_the_whole_batch():
    import torch
    from cls_b200.sharding import grad_tensors
    g = load_golden("x_all_losses")
    steps, B = int(g["steps"]), int(g["B"])
    full = _batch(g, list(range(B)))
    loss = full.simulate(steps)
    shards = [_batch(g, [0, 1], B), _batch(g, [2], B)]
    losses = [s.simulate(steps) for s in shards]
    assert abs(sum(losses) - loss) <= 1e-12 * abs(loss)
    for l in range(2):
        gW, gb = full.get_grads(0, l)
        parts = [s.get_grads(0, l) for s in shards]
        assert rel_err(parts[0][0] + parts[1][0], gW) < 1e-12
        assert rel_err(parts[0][1] + parts[1][1], gb) < 1e-12
    # the all-reduce's work, done by hand on the device buffers
    ta, tb = grad_tensors(shards[0]), grad_tensors(shards[1])
    assert [t.dtype for t in ta] == [torch.float64, torch.float64]
    for x, y in zip(ta, tb):
        x.add_(y)
    torch.cuda.synchronize()
    full.adam_step(0)
    shards[0].adam_step(0)
    for l in range(2):
        W, bb = full.get_weights(0, l)
        W2, bb2 = shards[0].get_weights(0, l)
        np.testing.assert_allclose(W2, W, rtol=0, atol=1e-13)
        np.testing.assert_allclose(bb2, bb, rtol=0, atol=1e-13)
    for b in (full, *shards):
        b.close()


def test_one_rank_nccl_group_reduces_in_place():
    import socket
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    from cls_b200.sharding import allreduce_shared_grads, grad_tensors
    g = load_golden("quad_ref")
    b = _batch(g, [0, 1])
    b.simulate(int(g["steps"]))
    before = [t.clone() for t in grad_tensors(b)]
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    store = dist.TCPStore("127.0.0.1", port, 1, True, timeout=timedelta(seconds=30))
    dist.init_process_group("nccl", store=store, rank=0, world_size=1, timeout=timedelta(seconds=60))
    try:
        allreduce_shared_grads(b)
        torch.cuda.synchronize()
        after = grad_tensors(b)
        for x, y in zip(before, after):
            assert torch.equal(x, y)
    finally:
        dist.destroy_process_group()
    b.close()
