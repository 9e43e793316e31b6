"""Data-parallel training of a shared controller (cls_b200.sharding) over
world-size-2 gloo ranks on CPU.  Each rank computes the gradient of its
contiguous env shard, with its losses divided by the total env count (the
reference divides by the batch size, multitask/taichi_env.py:185-293) --
here with the FP64 oracle standing in for the GPU batch, which needs a
device -- and all-reduces it; the sum must equal the single-process
gradient and loss of the whole batch to rounding (rel 1e-12)."""
import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case():
    from helpers import load_golden
    g = load_golden("x_all_losses")        # 3 envs: shards of 2 and 1
    return g, int(g["steps"])


def _oracle(g, envs, loss_envs=0):
    from helpers import oracle_from_golden
    o = oracle_from_golden(g)
    if envs is None:
        return o
    from helpers import golden_kwargs
    from oracle.ms_oracle import MassSpringOracle
    sub = MassSpringOracle(g["objects"], g["springs"], len(envs), int(g["T"]), hidden=[int(g["n_hidden"])],
                           initial_objects=g["x0"][0], loss_envs=loss_envs, **golden_kwargs(g))
    sub.set_weights([g["W1"], g["W2"]], [g["b1"], g["b2"]])
    sub.x[0] = g["x0"][envs]
    sub.set_targets(g["target_v"][:, envs], g["target_h"][:, envs], g["target_c"][:, envs])
    return sub


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from cls_b200 import sharding
    g, steps = _case()
    B = int(g["B"])
    b0, b1 = sharding.env_shard(B, rank, world)
    o = _oracle(g, list(range(b0, b1)), loss_envs=B)
    loss = o.run(steps)
    tensors = [torch.from_numpy(np.concatenate([a.ravel() for a in (*o.gW, *o.gb)]).copy())]
    sharding.sum_gradients_(tensors)
    total = sharding.sum_losses({"total": loss})["total"]
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, b1 - b0, tensors[0].numpy(), total))


def test_env_shards_cover_the_batch():
    from cls_b200.sharding import env_shard
    for n, w in ((4096, 8), (32, 3), (3, 2), (5, 8)):
        ranges = [env_shard(n, r, w) for r in range(w)]
        assert ranges[0][0] == 0 and ranges[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
        sizes = [e - s for s, e in ranges]
        assert max(sizes) - min(sizes) <= 1


def test_two_gloo_ranks_reproduce_the_single_process_gradient():
    import multiprocessing as mp
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(60)
    assert all(p.exitcode == 0 for p in procs)
    assert [r[1] for r in res] == [2, 1]
    g, steps = _case()
    o = _oracle(g, None)
    loss = o.run(steps)
    full = np.concatenate([a.ravel() for a in (*o.gW, *o.gb)])
    for _, _, reduced, total in res:
        err = np.linalg.norm(reduced - full) / np.linalg.norm(full)
        assert err < 1e-12, err
        assert abs(total - loss) <= 1e-12 * abs(loss)
