"""Benchmark: fused forward + adjoint training iterations of batched uneven
mass-spring robots (512 random lattices of 50-2000 vertices, 2000 substeps,
checkpoint every 50, MLP 2x128 tanh, FP32) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one training iteration over the whole batch: first-pass rollout,
loss, checkpointed reverse pass (recompute + adjoint + weight-gradient
products) and the Adam update.  The metric is env-substeps per second of that
forward + adjoint iteration (whole job, all GPUs).  Under torchrun every rank
runs its own 512 robots (weak scaling, no data-path collective).

``--impl reference`` times the reference algorithm's CPU implementation (the
project's FP64 restatement, all host cores) on a bounded sample of the same
workload; the reference itself needs Taichi, which is not installed.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+adjoint env-substeps/s (batched uneven mass-spring)"
# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) of one launch
# divided by the algorithmic bytes of that launch, from one `ncu --set full`
# capture of this workload at 128 robots x 100 substeps (the 512-robot workload
# is too large to capture); the traffic reported below scales the full launch's
# algorithmic bytes by it.
TRAFFIC_RATIO = {"reverse": 8.620194e9 / 10.330433e9, "recompute": 8.787660e9 / 10.441533e9}
UNIT = "env-substeps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--robots", type=int, default=512)
    ap.add_argument("--substeps", type=int, default=2000)
    ap.add_argument("--checkpoint", type=int, default=50)
    ap.add_argument("--plain-sample", type=int, default=24)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--threads", type=int, default=0, help="threads per CTA (0: automatic)")
    return ap.parse_args()


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def config_dict(a, n_gpus):
    return {"workload": "batched uneven mass-spring: %d random lattices (50-2000 vertices, "
                        "log-uniform; 30%% springs actuated) x %d substeps, checkpoint every %d, "
                        "MLP 2x128 tanh, velocity+rotation loss, Adam" % (a.robots, a.substeps, a.checkpoint),
            "robots_per_gpu": a.robots, "substeps": a.substeps, "checkpoint_every": a.checkpoint,
            "parallelism": "env-sharded replicas x%d (no data-path collective)" % n_gpus,
            "l2": "inputs larger than L2 (controller weights ~0.8 GB per GPU)"}


# ----------------------------------------------------------- CPU baseline
def cpu_sample(robots, seed, n_robots, substeps, threads):
    """Time the FP64 oracle (reference algorithm restated) on a bounded sample:
    n_robots robots of the workload, `substeps` substeps each, forward + loss +
    backward, one robot per worker thread."""
    from oracle.ms_oracle import MassSpringOracle
    from cls_b200 import workloads
    rng = np.random.default_rng(seed)
    pick = rng.choice(len(robots), size=min(n_robots, len(robots)), replace=False)
    T = substeps

    def one(r):
        rb = robots[r]
        o = MassSpringOracle(rb.objects, rb.springs, 1, T, n_sin=8, dup_v=1, dup_h=1, dup_c=0,
                             hidden=list(rb.hidden), dt=2e-3, gravity=-9.8, ground=0.0,
                             drag=-math.log(0.99) / 2e-3, dashpot=0.1, friction=0.5,
                             spring_omega=2 * math.pi / 2e-3 / 100, run_period=100,
                             turn_period=500, jump_period=500, act_hidden="tanh", act_out="tanh",
                             out_index=rb.spring_output, n_out=rb.n_outputs,
                             loss=("velocity", "rotation"), n_threads=1)
        wr = np.random.default_rng(r)
        for l in range(o.L):
            o.W[l][...] = (wr.random(o.W[l].shape) * 2 - 1) * math.sqrt(6 / o.W[l].shape[1])
        o.set_initial_state(rb.objects)
        tv, th = workloads.targets(wr, T, 1)
        o.set_targets(tv, th)
        t0 = time.perf_counter()
        o.run(T)
        return time.perf_counter() - t0, T - 1

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        res = list(ex.map(one, pick))
    wall = time.perf_counter() - t0
    env_substeps = sum(n for _, n in res)
    return env_substeps / wall, "%d robots of the workload x %d substeps (forward+loss+backward, FP64)" % (
        len(pick), T - 1), wall


def run_reference(a):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from cls_b200 import workloads
    robots = workloads.uneven_robots(a.robots, seed=0)
    cores = os.cpu_count() or 1
    vals = []
    sample = ""
    for i in range(a.warmup + a.steps):
        v, sample, wall = cpu_sample(robots, 100 + i, n_robots=cores * 2, substeps=200, threads=cores)
        if i >= a.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": config_dict(a, a.gpus),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample + "; reference Taichi not installed (no network)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------- clocks
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.QUERY,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None
        loaded = [s for s in sm if smax and s > 0.5 * smax] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": smax,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ ours
def run_ours(a):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    import cls_b200
    from cls_b200 import workloads
    b, robots, (tv, th) = workloads.uneven_batch(n_robots=a.robots, steps=a.substeps,
                                                K=a.checkpoint, seed=1000 * rank,
                                                threads_per_block=a.threads)
    stream = torch.cuda.Stream()
    b.set_stream(stream.cuda_stream)
    env_substeps = b.n_envs * (a.substeps - 1)

    def iteration(it):
        b.simulate(a.substeps)
        b.adam_step(it)

    for it in range(a.warmup):
        iteration(it)
    b.synchronize()
    b.profile(True)
    b.profile_read(reset=True)
    clk = ClockSampler(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clk.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for it in range(a.steps):
        iteration(a.warmup + it)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = ev0.elapsed_time(ev1)
    prof_ms, prof_n = b.profile_read(reset=True)
    b.profile(False)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    ms_per_step = ms / a.steps
    value = world * env_substeps / (ms_per_step / 1e3)
    print("timed: %.1f ms/step, %.3e %s, kernels %s" % (ms_per_step, value, UNIT, prof_ms),
          file=sys.stderr)

    # roofline of the dominant kernel (CUDA events around each launch above)
    alg = workloads.algorithmic_bytes(robots, list(range(len(robots))))
    subs_total = a.substeps - 1
    kinds = {"forward": subs_total, "recompute": subs_total, "reverse": subs_total}
    top = max(kinds, key=lambda k: prof_ms[k])
    bytes_region = alg[top] * subs_total * a.steps
    achieved = bytes_region / (prof_ms[top] / 1e3) / 1e9
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        peak, peak_src = 6650.0, "fallback"
    kernel_name = {"forward": "ms_forward_kernel (first pass)", "recompute": "ms_forward_kernel (recompute)",
                   "reverse": "ms_reverse_kernel"}[top]
    traffic = None
    if top in TRAFFIC_RATIO:
        per_launch = alg[top] * (subs_total if top == "forward" else a.checkpoint)
        traffic = TRAFFIC_RATIO[top] * per_launch
    roofline = {"kernel": kernel_name, "bound": "hbm", "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_src,
                "traffic": traffic,
                "share_of_step": prof_ms[top] / max(1e-9, sum(prof_ms.values())),
                "kernel_ms": prof_ms, "launches": prof_n}

    # plain form: the same kernels, one robot per launch, on a bounded sample
    plain = None
    if rank == 0 and a.plain_sample > 0:
        sub = robots[:a.plain_sample]
        pb, _, _ = workloads.uneven_batch(robots=sub, steps=a.substeps, K=a.checkpoint, seed=7)
        ps = torch.cuda.Stream()
        pb.set_stream(ps.cuda_stream)
        pb.simulate(a.substeps, per_env=True)
        pb.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ps)
        pb.simulate(a.substeps, per_env=True)
        e1.record(ps)
        torch.cuda.synchronize()
        pms = e0.elapsed_time(e1)
        e0.record(ps)
        pb.simulate(a.substeps)
        e1.record(ps)
        torch.cuda.synchronize()
        bms = e0.elapsed_time(e1)
        n_sub = len(sub) * (a.substeps - 1)
        plain = {"value": n_sub / (pms / 1e3), "unit": UNIT,
                 "sample": "first %d robots of the workload, one robot per launch (same kernels)" % len(sub),
                 "batched_same_sample": n_sub / (bms / 1e3),
                 "batched_full_over_plain": value / world / (n_sub / (pms / 1e3))}
        pb.close()

    # end to end through the C ABI with host buffers (pinned), copies inside
    e2e = None
    if a.e2e_steps > 0:
        x0 = torch.empty((b.n_vertices_total, 3), dtype=torch.float64).pin_memory()
        v0 = torch.zeros((b.n_vertices_total, 3), dtype=torch.float64).pin_memory()
        x0.copy_(torch.from_numpy(np.concatenate([r.objects for r in robots])))
        tvh = torch.from_numpy(np.ascontiguousarray(tv)).pin_memory()
        thh = torch.from_numpy(np.ascontiguousarray(th)).pin_memory()
        loss_terms = torch.zeros(8, dtype=torch.float64).pin_memory()
        lib, h = b.lib, b.h
        import ctypes
        P = ctypes.POINTER(ctypes.c_double)
        pd = lambda t: ctypes.cast(t.data_ptr(), P)  # noqa: E731
        env_loss = torch.zeros((8, b.n_envs), dtype=torch.float64).pin_memory()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for it in range(a.e2e_steps):
            cls_b200._capi.check(lib.cls_set_state(h, pd(x0), pd(v0)), h)
            cls_b200._capi.check(lib.cls_set_targets(h, pd(tvh), pd(thh), None), h)
            cls_b200._capi.check(lib.cls_forward(h, a.substeps), h)
            cls_b200._capi.check(lib.cls_loss(h, pd(loss_terms), pd(env_loss)), h)
            cls_b200._capi.check(lib.cls_backward(h), h)
            cls_b200._capi.check(lib.cls_adam_step(h, it, None), h)
            cls_b200._capi.check(lib.cls_synchronize(h), h)
        e2e_s = (time.perf_counter() - t0) / a.e2e_steps
        if world > 1:
            t = torch.tensor([e2e_s], device="cuda")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e2e_s = float(t.item())
        h2d = (x0.numel() + v0.numel() + tvh.numel() + thh.numel()) * 8
        d2h = (loss_terms.numel() + b.n_envs * 8) * 8
        e2e = {"value": world * env_substeps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h),
               "path": "cls_set_state/cls_set_targets (pinned host) -> cls_forward -> cls_loss "
                       "(D2H) -> cls_backward -> cls_adam_step -> cls_synchronize"}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cores = os.cpu_count() or 1
        v, sample, wall = cpu_sample(robots, 11, n_robots=cores * 2, substeps=200, threads=cores)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": sample + "; wall %.1f s; reference Taichi not installed (no network)" % wall}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded random lattices, targets and weights)",
                "config": config_dict(a, world), "clocks": clocks,
                "gpu_launches": int(sum(prof_n.values())), "roofline": roofline,
                "plain": plain, "e2e": e2e, "cpu_baseline": cpu}
        print(json.dumps(line))
    b.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
