"""The N > 1 host paths of bench.py on CPU: world-size-2 gloo ranks for the
timing reductions (the job's time is the slowest rank's, its work the sum of
every rank's), and the reference arm under torchrun (rank 0 alone measures and
prints one JSON line; the other rank exits 0 without work)."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    from datetime import timedelta
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    import bench
    mx = bench.max_over_ranks(1.5 + rank, world, device="cpu")
    sm = bench.sum_over_ranks(10.0 * (rank + 1), world, device="cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, mx, sm))


def test_timing_reductions_over_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(60)
    assert all(p.exitcode == 0 for p in procs)
    assert res == [(0, 2.5, 30.0), (1, 2.5, 30.0)]
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.0, 1) == 3.0 and bench.sum_over_ranks(4.0, 1) == 4.0


def test_reference_arm_under_torchrun_prints_one_line():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py",
           "--impl", "reference", "--config", "quadruped", "--gpus", "2", "--steps", "1",
           "--warmup", "0"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "port"
