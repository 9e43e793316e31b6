"""Data-parallel training of one shared controller across GPUs.

Environments are independent within an iteration, so a batch whose envs
share one controller per robot type (the quadruped and spider
configurations; the reference's single ``Model`` for its whole batch,
multitask/diffphy_trainer.py:178-185) is sharded by contiguous env ranges,
one shard per rank.  Each rank runs its shard's rollout and reverse pass; the
only exchange is one in-place all-reduce (sum) of the weight and bias
gradients per iteration, between ``cls_backward`` and ``cls_adam_step``.
Every rank then applies the same Adam step to the same weights, so the
controllers stay identical.

Every loss term is divided by the batch's env count
(multitask/taichi_env.py:185-293).  Each shard therefore divides by the
*total* env count of its type (``cls_set_loss_envs``): its loss and gradients
are then its share of the whole batch's, and their sum over ranks is the
single-process batch's loss and gradient.

On NCCL the reduction runs in place on the library's device buffers
(``cls_grad_buffers``); on other backends (gloo, for CPU tests) through host
copies.
"""
import ctypes

import numpy as np

from . import _capi


def env_shard(n_envs, rank, world):
    """Contiguous env range [begin, end) of `rank` out of `n_envs` envs
    (the first n_envs % world ranks take one env more)."""
    base, extra = divmod(int(n_envs), int(world))
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def shard_loss_envs(batch, total_envs_per_robot):
    """Makes `batch` (this rank's shard) divide robot type r's losses by
    total_envs_per_robot[r], the type's env count over all ranks."""
    for r, n in enumerate(total_envs_per_robot):
        batch.set_loss_envs(r, int(n))


class _DeviceArray:
    """__cuda_array_interface__ over a raw device pointer (zero-copy)."""

    def __init__(self, ptr, n, elem_bytes):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f%d" % elem_bytes,
                                         "data": (int(ptr), False), "version": 3, "strides": None}


def grad_tensors(batch):
    """torch views (no copy) of the batch's weight- and bias-gradient device
    buffers (cls_grad_buffers)."""
    import torch
    w, b = ctypes.c_void_p(), ctypes.c_void_p()
    nw, nb = ctypes.c_int64(), ctypes.c_int64()
    e = np.zeros(1, dtype=np.int32)
    batch._c(batch.lib.cls_grad_buffers(batch.h, ctypes.byref(w), ctypes.byref(nw), ctypes.byref(b),
                                        ctypes.byref(nb), _capi.ptr(e, _capi.P_I)))
    out = []
    for p, n in ((w, nw), (b, nb)):
        if n.value > 0:
            out.append(torch.as_tensor(_DeviceArray(p.value, n.value, int(e[0])), device="cuda"))
    return out


def sum_gradients_(tensors, group=None):
    """In place: each tensor <- its sum over the group's ranks.  Device
    tensors on an NCCL group are reduced where they lie; other combinations
    go through host copies."""
    import torch.distributed as dist
    backend = dist.get_backend(group)
    for t in tensors:
        if t.is_cuda and backend != "nccl":
            h = t.detach().to("cpu", copy=True)
            dist.all_reduce(h, op=dist.ReduceOp.SUM, group=group)
            t.copy_(h)
        else:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return tensors


def allreduce_shared_grads(batch, group=None, stream=None):
    """Sums every rank's shard gradients into every rank's batch (call between
    backward() and adam_step(); the shards' losses must divide by the total
    env counts, shard_loss_envs).  `stream`: the torch stream the batch runs
    on (its cuda_stream given to set_stream), so that the reduction follows
    the reverse pass and Adam follows the reduction; None: the batch runs on
    the legacy default stream."""
    import torch
    tensors = grad_tensors(batch)
    if stream is None:
        sum_gradients_(tensors, group)
    else:
        with torch.cuda.stream(stream):
            sum_gradients_(tensors, group)
    return tensors


def sum_losses(terms, group=None):
    """The whole batch's loss terms (dict of floats) from every rank's shard."""
    import torch
    import torch.distributed as dist
    keys = sorted(terms)
    t = torch.tensor([float(terms[k]) for k in keys], dtype=torch.float64)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return dict(zip(keys, t.cpu().tolist()))
