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

``--config`` selects another workload for the same measurement (the default,
``uneven``, is the headline line): ``quadruped`` (32 envs of the quadruped
lattice, 1000 substeps, MLP 1x64), ``spider`` (4096 envs of the spider lattice,
1000 substeps, MLP 2x256) or ``mpm`` (3D MLS-MPM legged body of 29,504
particles on a 64^3 grid, 8 envs, 1000 substeps of dt 1e-4, neo-Hookean with
16 fibre-actuated muscle groups, forward + checkpointed adjoint).  The
quadruped and spider episodes run as one checkpoint segment by default (their
records fit in HBM; ``--checkpoint`` sets K).

Before warm-up the mass-spring configurations run the launch-shape autotuner
(``cls_autotune``: threads per CTA, CTAs per SM, controller in shared memory,
and the batched controller path for types with many envs) on their own
workload; the chosen shape and the timed candidates are reported as
``launch_shape`` (``--no-autotune`` or ``--threads N`` skip it).
"""
import argparse
import dataclasses
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

METRICS = {"uneven": "fwd+adjoint env-substeps/s (batched uneven mass-spring)",
           "quadruped": "fwd+adjoint env-substeps/s (quadruped lattice, 32 envs)",
           "spider": "fwd+adjoint env-substeps/s (spider lattice, 4096 envs)",
           "mpm": "fwd+adjoint env-substeps/s (3D MLS-MPM legged body, 8 envs)",
           "serve": "served env-substeps/s of Poisson rollout requests (p50/p99 latency beside)"}
DEFAULT_SUBSTEPS = {"uneven": 2000, "quadruped": 1000, "spider": 1000, "mpm": 1000, "serve": 2000}
DEFAULT_ENVS = {"uneven": 512, "quadruped": 32, "spider": 4096, "mpm": 8, "serve": 32}
SERVE_RATE = 200.0          # requests per second
SERVE_SECONDS_PER_STEP = 2.0  # seconds of arrivals per bench step
# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) of one launch
# divided by the algorithmic bytes of that launch, from one `ncu --set full`
# capture of this workload at 128 robots x 100 substeps (the 512-robot workload
# is too large to capture); the traffic reported below scales the full launch's
# algorithmic bytes by it.
TRAFFIC_RATIO = {"reverse": 8.622361e9 / 10.330433e9, "recompute": 8.787660e9 / 10.441533e9}
UNIT = "env-substeps/s"
SERVE_MPM_SLOTS = 4     # whole-rollout MPM slots of the serving workload (one-env handles)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="uneven", choices=sorted(METRICS))
    ap.add_argument("--robots", "--envs", dest="robots", type=int, default=None,
                    help="robots (uneven) or envs per GPU (default: the configuration's)")
    ap.add_argument("--substeps", type=int, default=None)
    ap.add_argument("--checkpoint", type=int, default=None,
                    help="substeps per checkpoint segment (default: 50; the spider and quadruped "
                         "episodes as one segment, whose records the first pass keeps)")
    ap.add_argument("--plain-sample", type=int, default=24)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-grad-error", action="store_true",
                    help="skip the FP32-vs-FP64 gradient error block")
    ap.add_argument("--grad-study", action="store_true",
                    help="uneven: print the FP32-vs-FP64 gradient error of the workload's median robot "
                         "against the episode length over seeded input draws (no timing)")
    ap.add_argument("--threads", type=int, default=0,
                    help="threads per CTA of the fused kernels (0: autotuned, see --no-autotune)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="mass-spring: skip the launch-shape autotuner (cls_autotune) before warm-up")
    ap.add_argument("--controller", default="auto", choices=["auto", "per_env", "batched"],
                    help="controller path: batched = one tensor-core GEMM per layer over all envs "
                         "of a robot type (automatic for types with >= 256 envs)")
    ap.add_argument("--particle-order", default="base_runs", choices=["cells", "base_runs"],
                    help="mpm: internal particle order (base_runs: sorted by base cell, each warp's "
                         "runs of equal base cells summed by shuffles before the grid reductions)")
    ap.add_argument("--tick-segments", type=int, default=2,
                    help="serve: checkpoint segments a tick advances every request by (measured on "
                         "B200, 6 s of arrivals: 1 / 2 / 4 segments gave p50 135 / 133 / 183 ms, "
                         "p99 1.22 / 1.18 / 1.19 s at the same throughput)")
    a = ap.parse_args()
    if a.robots is None:
        a.robots = DEFAULT_ENVS[a.config]
    if a.substeps is None:
        a.substeps = DEFAULT_SUBSTEPS[a.config]
    if a.checkpoint is None:
        # the uneven configuration fixes 50; the spider and quadruped episodes
        # fit in HBM with every substep's records (tens of GB for the spider),
        # so they run as one segment and skip the recompute pass
        a.checkpoint = a.substeps if a.config in ("spider", "quadruped") else 50
    return a


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(x, world, device="cuda"):
    """The largest of every rank's x (a time: the job takes as long as its
    slowest rank); x itself when there is one rank.  Every rank calls it at the
    same point."""
    if world <= 1:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world, device="cuda"):
    """The sum of every rank's x (work done); x itself when there is one rank."""
    if world <= 1:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
    return float(t.item())


def config_dict(a, n_gpus):
    par = "env-sharded replicas x%d (no data-path collective)" % n_gpus
    if a.config in ("quadruped", "spider") and n_gpus > 1:
        par = ("dp%d: env shards of one shared controller, one NCCL all-reduce of the weight "
               "gradients per iteration" % n_gpus)
    if a.config == "uneven":
        return {"workload": "batched uneven mass-spring: %d random lattices (50-2000 vertices, "
                            "log-uniform; 30%% springs actuated) x %d substeps, checkpoint every %d, "
                            "MLP 2x128 tanh, velocity+rotation loss, Adam"
                            % (a.robots, a.substeps, a.checkpoint),
                "robots_per_gpu": a.robots, "substeps": a.substeps, "checkpoint_every": a.checkpoint,
                "parallelism": par,
                "l2": "inputs larger than L2 (controller weights ~0.8 GB per GPU)"}
    if a.config in ("quadruped", "spider"):
        from cls_b200 import robot_design
        obj, spr = (robot_design.quadruped_lattice() if a.config == "quadruped" else
                    robot_design.spider_lattice())
        shape = "%s lattice (%d vertices, %d springs, %d actuated), MLP %s tanh" % (
            a.config, obj.shape[0], spr.shape[0], int((spr[:, 4] > 0).sum()),
            "1x64" if a.config == "quadruped" else "2x256")
        return {"workload": "%d envs of the %s x %d substeps, checkpoint every %d, "
                            "velocity+rotation loss, Adam" % (a.robots, shape, a.substeps, a.checkpoint),
                "envs_per_gpu": a.robots, "substeps": a.substeps, "checkpoint_every": a.checkpoint,
                "parallelism": par,
                "l2": "trajectory and checkpoints written every iteration exceed L2"}
    if a.config == "serve":
        return {"workload": "serving: Poisson rollout requests at %.0f/s over %.0f s; robot mix quadruped "
                            "25%% (MLP 1x64), spider 20%% (MLP 2x256), random lattices of 100/300/800/1500 "
                            "vertices 50%% (MLP 2x128), 3D MPM legged body 5%% (64^3 grid, dt 1e-4, %d "
                            "whole-rollout slots); episodes U{100..2000} substeps; 80%% forward-only "
                            "evaluation, 20%% forward+adjoint gradient queries; %d slots per mass-spring "
                            "type, ticks of %d substeps" % (SERVE_RATE, a.steps * SERVE_SECONDS_PER_STEP,
                                                             SERVE_MPM_SLOTS, a.robots,
                                                             a.checkpoint * a.tick_segments),
                "slots_per_type": a.robots, "rate_per_s": SERVE_RATE,
                "arrival_seconds": a.steps * SERVE_SECONDS_PER_STEP, "checkpoint_every": a.checkpoint,
                "parallelism": "independent servers x%d (no data-path collective)" % n_gpus,
                "l2": "per-slot trajectories and checkpoints of all resident requests exceed L2"}
    return {"workload": "3D MLS-MPM: legged body of 29504 particles (8 per cell, 16 fibre-actuated "
                        "muscle groups), 64^3 grid, neo-Hookean E=1e4 nu=0.3, dt 1e-4, %d envs x %d "
                        "substeps, checkpoint every %d, centre loss" % (a.robots, a.substeps, a.checkpoint),
            "envs_per_gpu": a.robots, "substeps": a.substeps, "checkpoint_every": a.checkpoint,
            "particle_order": a.particle_order, "parallelism": par,
            "l2": "state trajectory checkpoints and per-step records exceed L2"}


# ----------------------------------------------------------- CPU baseline
def cpu_sample(robots, seed, n_robots, substeps, threads, min_wall=0.0):
    """Time the FP64 oracle (reference algorithm restated) on a bounded sample:
    batches of n_robots robots of the workload (seeded picks), `substeps`
    substeps each, forward + loss + backward, one robot per worker thread;
    batches repeat until `min_wall` seconds have passed."""
    from oracle.ms_oracle import MassSpringOracle
    from cls_b200 import workloads
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

    wall, env_substeps, n_run, batch = 0.0, 0, 0, 0
    with ThreadPoolExecutor(max_workers=threads) as ex:
        while batch == 0 or wall < min_wall:
            rng = np.random.default_rng(seed + 7919 * batch)
            pick = rng.choice(len(robots), size=min(n_robots, len(robots)), replace=False)
            t0 = time.perf_counter()
            res = list(ex.map(one, pick))
            wall += time.perf_counter() - t0
            env_substeps += sum(n for _, n in res)
            n_run += len(pick)
            batch += 1
    return env_substeps / wall, ("%d robots of the workload (%d batches) x %d substeps "
                                 "(forward+loss+backward, FP64)" % (n_run, batch, T - 1)), wall


def run_reference(a):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from cls_b200 import workloads
    if a.config == "mpm":
        return run_reference_mpm(a)
    if a.config == "serve":
        return run_reference_serve(a)
    if a.config == "uneven":
        robots = workloads.uneven_robots(a.robots, seed=0)
    else:
        from cls_b200 import robot_design
        from cls_b200.batch import Robot
        if a.config == "quadruped":
            obj, spr = robot_design.quadruped_lattice()
            robots = [Robot.actuated_outputs(obj, spr, hidden=[64])] * a.robots
        else:
            obj, spr = robot_design.spider_lattice()
            robots = [Robot.actuated_outputs(obj, spr, hidden=[256, 256])] * a.robots
    cores = os.cpu_count() or 1
    vals = []
    sample = ""
    # warm-up steps run one batch; each timed step is a bounded sample of at
    # least min(10 s, 150 s / steps) so that the whole run ends within minutes
    per_step = min(10.0, 150.0 / max(1, a.steps))
    for i in range(a.warmup + a.steps):
        v, sample, wall = cpu_sample(robots, 100 + i, n_robots=cores * 2, substeps=200, threads=cores,
                                     min_wall=per_step if i >= a.warmup else 0.0)
        if i >= a.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRICS[a.config], "value": value, "unit": UNIT, "n_gpus": a.gpus,
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
def make_ms_batch(a, n, seed, robots=None):
    """The mass-spring batch of the selected configuration: (batch, robot list,
    robot index of every env, (target velocities, target heights))."""
    from cls_b200 import workloads
    if a.config == "uneven":
        b, robots, tt = workloads.uneven_batch(n_robots=n, steps=a.substeps, K=a.checkpoint,
                                               seed=seed, robots=robots,
                                               threads_per_block=a.threads)
        return b, robots, list(range(len(robots))), tt
    build = workloads.quadruped_batch if a.config == "quadruped" else workloads.spider_batch
    # every rank's shard holds the same controller (weights seeded alike);
    # targets come from the rank's own seed
    b, robots, tt = build(n_envs=n, steps=a.substeps, K=a.checkpoint, seed=seed, weights_seed=2,
                          threads_per_block=a.threads)
    return b, robots, [0] * n, tt


def grad_error_block(a, robots, env_robot):
    """The FP32 result against an FP64 build of the same kernels on the same
    inputs (state, targets, FP32-representable weights): relative 2-norm
    errors of the loss, of every robot's weight and bias gradients (worst
    layer and robot) and of d loss / d x0 (worst env), on bounded subsets of
    the workload; the configuration's gradient bar is rel 1e-4."""
    from cls_b200 import workloads
    from cls_b200.batch import MassSpringBatch, default_params
    if a.config == "uneven":
        # the FP64 build's state of one robot must fit one CTA's shared
        # memory: robots of up to 900 vertices
        fit = [r for r in robots if r.n_vertices <= 900]
        sub = fit[:16]
        med = float(np.median([r.n_vertices for r in robots]))
        one = min(fit, key=lambda r: abs(r.n_vertices - med))
        cases = [("first %d robots of <= 900 vertices x 200 substeps" % len(sub), sub, list(range(len(sub))), 200),
                 ("the %d-vertex robot (workload median %d) x %d substeps" % (one.n_vertices, med, a.substeps),
                  [one], [0], a.substeps)]
    else:
        n = min(16, len(env_robot))
        cases = [("%d envs x %d substeps" % (n, a.substeps), robots, [0] * n, a.substeps)]

    def rel(x, y):
        x, y = np.asarray(x, np.float64).ravel(), np.asarray(y, np.float64).ravel()
        d = np.linalg.norm(y)
        return float(np.linalg.norm(x - y) / (d if d > 0 else 1.0))

    def f32(x):
        return np.asarray(x, np.float64).astype(np.float32).astype(np.float64)

    def errors(p, q, sl):
        (lp, gp, xp), (lq, gq, xq) = p[:3], q[:3]
        return (abs(lp - lq) / abs(lq), max(rel(u[0], w[0]) for u, w in zip(gp, gq)),
                max(rel(u[1], w[1]) for u, w in zip(gp, gq)), max(rel(xp[s_], xq[s_]) for s_ in sl))

    out = []
    for desc, rb, er, steps in cases:
        # the FP32 build rounds its inputs (vertex positions, spring rest
        # lengths / stiffnesses / actuation coefficients, targets) to FP32 on
        # upload; the third run feeds the FP64 build those rounded inputs, so
        # its distance from the plain FP64 run is the part of the FP32 error
        # that exact arithmetic on FP32 inputs would keep (the problem's
        # conditioning), the rest being FP32 arithmetic
        rb_rounded = [dataclasses.replace(r, objects=f32(r.objects), springs=f32(r.springs)) for r in rb]
        runs = {}
        for key, prec, robots_k, rounded in (("fp32", 32, rb, False), ("fp64", 64, rb, False),
                                             ("fp64_rounded", 64, rb_rounded, True)):
            K = min(a.checkpoint, steps)
            b = MassSpringBatch(robots_k, er, default_params(**workloads._params(steps, K, precision=prec)))
            rng = np.random.default_rng(5)
            tv, th = workloads.targets(rng, steps, len(er))
            if rounded:
                tv, th = f32(tv), f32(th)
            b.set_targets(tv, th)
            for r, robot in enumerate(robots_k):
                for l in range(len(robot.hidden) + 1):
                    rows, cols = b.layer_shape(r, l)
                    W = (rng.uniform(-1, 1, (rows, cols)) * np.sqrt(6 / cols)).astype(np.float32)
                    b.set_weights(r, l, W.astype(np.float64), np.zeros(rows))
            loss = b.simulate(steps)
            grads = [b.get_grads(r, l) for r, robot in enumerate(robots_k) for l in range(len(robot.hidden) + 1)]
            gx0 = b.state_grads()[0]
            runs[key] = (loss, grads, gx0, [b.env_slice(e) for e in range(len(er))])
            b.close()
        sl = runs["fp32"][3]
        lr, gw, gb, gx = errors(runs["fp32"], runs["fp64"], sl)
        cl, cw, cb, cx = errors(runs["fp64_rounded"], runs["fp64"], sl)
        out.append({"sample": desc, "loss_rel": lr, "grad_W_rel": gw, "grad_b_rel": gb, "grad_x0_rel": gx,
                    "fp64_on_fp32_inputs": {"loss_rel": cl, "grad_W_rel": cw, "grad_b_rel": cb,
                                            "grad_x0_rel": cx}})
    worst = max(max(c["loss_rel"], c["grad_W_rel"], c["grad_b_rel"]) for c in out)
    floor = max(max(c["fp64_on_fp32_inputs"][k] for k in ("loss_rel", "grad_W_rel", "grad_b_rel")) for c in out)
    return {"against": "FP64 build of the same kernels", "bar": 1e-4, "cases": out,
            "worst_rel": worst, "meets_bar": bool(worst <= 1e-4),
            "input_rounding_rel": floor,
            "input_rounding": "the FP64 build on the FP32-rounded inputs against the FP64 build "
                              "(what exact arithmetic would still miss given FP32 inputs)"}


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
    b, robots, env_robot, (tv, th) = make_ms_batch(a, a.robots, 1000 * rank)
    stream = torch.cuda.Stream()
    b.set_stream(stream.cuda_stream)
    # one controller shared by the envs of every rank (quadruped, spider):
    # each rank's losses are its shard's share of the whole batch's, and the
    # weight gradients are summed over ranks before every Adam step
    shared = world > 1 and a.config in ("quadruped", "spider")
    if shared:
        from cls_b200 import sharding
        sharding.shard_loss_envs(b, [world * a.robots])
    # launch shape (and, with --controller auto, the controller path) picked
    # by timing this workload's own rollouts, before warm-up and outside the
    # timed region
    tuned = None
    if not a.no_autotune and not a.threads:
        t0 = time.perf_counter()
        tuned = b.autotune(repeats=1)
        tuned["seconds"] = time.perf_counter() - t0
    if a.controller != "auto" or tuned is None:
        b.set_controller_path(a.controller)
    batched = b.controller_batched
    tpb, cps, wsh = b.launch_shape
    launch_shape = {"threads_per_block": tpb, "ctas_per_sm": cps, "weights_shared": wsh,
                    "autotuned": tuned is not None}
    if tuned is not None:
        launch_shape.update(candidates=len(tuned["table"]), tuning_s=round(tuned["seconds"], 2),
                            table=[[e["controller_path"], e["threads_per_block"], e["ctas_per_sm"],
                                    e["weights_shared"], round(e["ms"], 3)] for e in tuned["table"]])
    env_substeps = b.n_envs * (a.substeps - 1)

    def reduce_grads():
        if shared:
            sharding.allreduce_shared_grads(b, stream=stream)

    def iteration(it):
        b.simulate(a.substeps)
        reduce_grads()
        b.adam_step(it)

    # the timed training iteration (forward, loss, backward, [gradient
    # all-reduce,] Adam) is one CUDA graph replay (the replay, the all-reduce
    # and an eager Adam step when the controller is shared); the eager path is
    # measured as e2e below
    iteration(0)
    b.synchronize()
    b.graph_capture(a.substeps, with_adam=not shared)

    def replay(it):
        b.graph_launch(it)
        if shared:
            reduce_grads()
            cls_b200._capi.check(b.lib.cls_adam_step(b.h, it, None), b.h)

    for it in range(a.warmup):
        replay(it)
    b.synchronize()
    clk = ClockSampler(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clk.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for it in range(a.steps):
        replay(a.warmup + it)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    ms_per_step = ms / a.steps
    # per-kernel breakdown: one more iteration, outside the timed region, with
    # CUDA events around every launch (their gaps would inflate the timed loop)
    b.profile(True)
    b.profile_read(reset=True)
    iteration(a.warmup + a.steps)
    b.synchronize()
    prof_ms, prof_n = b.profile_read(reset=True)
    b.profile(False)
    value = world * env_substeps / (ms_per_step / 1e3)
    print("timed: %.1f ms/step, %.3e %s, kernels %s" % (ms_per_step, value, UNIT, prof_ms),
          file=sys.stderr)

    # roofline of the dominant kernel (CUDA events around each launch above)
    # per-env path over several checkpoint segments: the library keeps the
    # whole episode's controller records when they fit a quarter of the free
    # memory (they do for these workloads) and its recomputes replay the
    # controller from them
    replay = not batched and a.substeps - 1 > a.checkpoint
    alg = workloads.algorithmic_bytes(robots, env_robot, batched=batched, replay=replay)
    subs_total = a.substeps - 1
    cands = ["forward", "recompute", "reverse"] + (["ctrl_gemm", "ctrl_gemm_adj"] if batched else [])
    top = max(cands, key=lambda k: prof_ms[k])
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
        hbm, bf16, peak_src = float(peaks["hbm_gbs"]), float(peaks["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        hbm, bf16, peak_src = 6650.0, 1590.0, "fallback"
    share = prof_ms[top] / max(1e-9, sum(prof_ms.values()))
    if top in ("ctrl_gemm", "ctrl_gemm_adj"):
        # tensor-core GEMMs: the three TF32 products of the 3xTF32 split, 2 M N K
        # each; TF32 runs at half the BF16 dense rate
        fl = workloads.controller_flops(robots, env_robot)
        passes = 2 if top == "ctrl_gemm" else 1       # first pass + recompute / reverse
        flops = 3 * fl["forward" if top == "ctrl_gemm" else "adjoint"] * subs_total * passes
        achieved = flops / (prof_ms[top] / 1e3) / 1e12
        peak = 0.5 * bf16
        roofline = {"kernel": "ms_ctrl_gemm_tc_kernel (%s)" % ("forward" if top == "ctrl_gemm" else "adjoint"),
                    "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": None,
                    "peak_source": peak_src + " bf16 dense x 0.5 (TF32 rate)",
                    "note": "achieved counts the 3 TF32 MMA products per FP32 product (3xTF32 split)",
                    "share_of_step": share, "kernel_ms": prof_ms, "launches": prof_n}
    else:
        bytes_region = alg[top] * subs_total
        achieved = bytes_region / (prof_ms[top] / 1e3) / 1e9
        if batched:
            kernel_name = {"forward": "ms_step_fwd_kernel (first pass)",
                           "recompute": "ms_step_fwd_kernel (recompute)", "reverse": "ms_step_rev_kernel"}[top]
        else:
            kernel_name = {"forward": "ms_forward_kernel (first pass)",
                           "recompute": "ms_forward_kernel (recompute)", "reverse": "ms_reverse_kernel"}[top]
        traffic = None
        if top in TRAFFIC_RATIO and not batched:
            per_launch = alg[top] * (subs_total if top == "forward" else a.checkpoint)
            traffic = TRAFFIC_RATIO[top] * per_launch
        roofline = {"kernel": kernel_name, "bound": "hbm", "achieved": achieved, "peak": hbm,
                    "unit": "GB/s", "frac": achieved / hbm, "peak_source": peak_src,
                    "traffic": traffic, "share_of_step": share, "kernel_ms": prof_ms, "launches": prof_n}

    # plain form: the same kernels, one robot per launch, on a bounded sample
    plain = None
    if rank == 0 and a.plain_sample > 0:
        pb, _, sub, _ = make_ms_batch(a, min(a.plain_sample, a.robots), 7, robots=robots[:a.plain_sample])
        pb.set_launch_shape(tpb, cps, wsh)
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
                 "sample": "first %d envs of the workload, one env per launch (same kernels)" % len(sub),
                 "batched_same_sample": n_sub / (bms / 1e3),
                 "batched_full_over_plain": value / world / (n_sub / (pms / 1e3))}
        pb.close()

    # end to end through the C ABI with host buffers (pinned), copies inside
    e2e = None
    if a.e2e_steps > 0:
        x0 = torch.empty((b.n_vertices_total, 3), dtype=torch.float64).pin_memory()
        v0 = torch.zeros((b.n_vertices_total, 3), dtype=torch.float64).pin_memory()
        x0.copy_(torch.from_numpy(np.concatenate([robots[r].objects for r in env_robot])))
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
            reduce_grads()
            cls_b200._capi.check(lib.cls_adam_step(h, it, None), h)
            cls_b200._capi.check(lib.cls_synchronize(h), h)
        e2e_s = (time.perf_counter() - t0) / a.e2e_steps
        e2e_s = max_over_ranks(e2e_s, world)
        h2d = (x0.numel() + v0.numel() + tvh.numel() + thh.numel()) * 8
        d2h = (loss_terms.numel() + b.n_envs * 8) * 8
        e2e = {"value": world * env_substeps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h),
               "path": "cls_set_state/cls_set_targets (pinned host) -> cls_forward -> cls_loss "
                       "(D2H) -> cls_backward -> cls_adam_step -> cls_synchronize"}

    grad_err = None
    if rank == 0 and not a.no_grad_error:
        t0 = time.perf_counter()
        grad_err = grad_error_block(a, robots, env_robot)
        grad_err["seconds"] = round(time.perf_counter() - t0, 2)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cores = os.cpu_count() or 1
        v, sample, wall = cpu_sample([robots[r] for r in env_robot], 11, n_robots=cores * 2,
                                     substeps=200, threads=cores, min_wall=10.0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": sample + "; wall %.1f s; reference Taichi not installed (no network)" % wall}

    if rank == 0:
        line = {"metric": METRICS[a.config], "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded random lattices, targets and weights)",
                "config": config_dict(a, world), "controller_path": "batched" if batched else "per_env",
                "launch_shape": launch_shape,
                "clocks": clocks,
                "gpu_launches": int(sum(prof_n.values())) * a.steps, "roofline": roofline,
                "plain": plain, "e2e": e2e, "cpu_baseline": cpu, "grad_rel_err": grad_err}
        print(json.dumps(line))
    b.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


# ------------------------------------------------------------------- MPM
def mpm_cpu_sample(a, seed, envs, substeps, min_wall=0.0):
    """Time the FP64 MPM oracle (OpenMP over envs, all host cores) on `envs`
    envs of the workload body for `substeps` substeps, forward + loss +
    backward, repeated with fresh seeded actuation until `min_wall` seconds
    have passed."""
    from oracle.mpm_oracle import MPMOracle
    from cls_b200 import workloads
    pos, mus, fib = workloads.legged_body()
    E, nu = 1e4, 0.3
    o = MPMOracle(pos, mus, envs, substeps, dim=3, n_grid=64, dt=1e-4, p_vol=1.0,
                  mu=E / (2 * (1 + nu)), la=E * nu / ((1 + nu) * (1 - 2 * nu)), act_strength=1e3,
                  gravity=-10.0, bound=3, material="neo_hookean", fibre=fib, n_muscles=16)
    rng = np.random.default_rng(seed)
    o.loss_w[substeps] = 1.0
    o.target[...] = pos.mean(axis=0) + np.array([0.05, 0.0, 0.0])
    wall, runs = 0.0, 0
    while runs == 0 or wall < min_wall:
        o.act[...] = rng.uniform(-1, 1, o.act.shape)
        t0 = time.perf_counter()
        o.run(substeps)
        wall += time.perf_counter() - t0
        runs += 1
    return runs * envs * substeps / wall, "%d envs x %d substeps of the workload body, %d runs " \
        "(forward+loss+backward, FP64, OpenMP over envs)" % (envs, substeps, runs), wall


def run_reference_mpm(a):
    cores = os.cpu_count() or 1
    vals, sample = [], ""
    per_step = min(10.0, 150.0 / max(1, a.steps))
    for i in range(a.warmup + a.steps):
        v, sample, _ = mpm_cpu_sample(a, 100 + i, envs=cores, substeps=24,
                                      min_wall=per_step if i >= a.warmup else 0.0)
        if i >= a.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRICS[a.config], "value": value, "unit": UNIT,
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": config_dict(a, a.gpus),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample + "; the reference's MPM is 2D and needs Taichi "
                                                "(not installed)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_mpm(a):
    import ctypes
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    import cls_b200
    from cls_b200 import workloads
    T = a.substeps
    b, pos = workloads.mpm_batch(n_envs=a.robots, steps=T, K=a.checkpoint, seed=1000 * rank,
                                 particle_order=a.particle_order)
    stream = torch.cuda.Stream()
    b.set_stream(stream.cuda_stream)
    env_substeps = b.E * T

    # per-kernel profile of one iteration (events around every launch)
    b.forward(T)
    b.backward()
    torch.cuda.synchronize()
    b.profile(True)
    b.profile_read(reset=True)
    b.forward(T)
    b.backward()
    prof_ms, prof_n = b.profile_read(reset=True)
    b.profile(False)

    # timed: the captured forward + backward graph, one launch per iteration
    b.graph_capture(T)
    for _ in range(a.warmup):
        b.graph_launch()
    clk = ClockSampler(local)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clk.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(a.steps):
        b.graph_launch()
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1), world)
    ms_per_step = ms / a.steps
    value = world * env_substeps / (ms_per_step / 1e3)
    print("timed: %.1f ms/step, %.3e %s, kernels %s" % (ms_per_step, value, UNIT, prof_ms),
          file=sys.stderr)

    alg = workloads.mpm_algorithmic_bytes(pos, b.E, n_grid=64)
    kinds = [k for k in alg if prof_n.get(k, 0) > 0]
    top = max(kinds, key=lambda k: prof_ms[k])
    achieved = alg[top] * prof_n[top] / (prof_ms[top] / 1e3) / 1e9
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, peak_src = float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        peak, peak_src = 6650.0, "fallback"
    roofline = {"kernel": top, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_src, "traffic": None,
                "share_of_step": prof_ms[top] / max(1e-9, sum(prof_ms.values())),
                "kernel_ms": prof_ms, "launches": prof_n,
                "per_kernel_frac": {k: alg[k] * prof_n[k] / (prof_ms[k] / 1e3) / 1e9 / peak
                                    for k in kinds}}
    # the particle kernels' working set (~33 MB of grid, ~24 MB of particles
    # for 8 envs) is L2-resident: their scatter roofline is the measured rate
    # of 16-byte vector reductions, against which each kernel's 27 node
    # updates per particle and step are counted (P2G in the forward kernels,
    # G2P^T's velocity adjoint in the reverse; with the base-cell order the
    # forward kernels issue one reduction per run of lanes on one base cell,
    # fewer than 27 per particle)
    from cls_b200 import mpm as mpm_mod
    n_nodes = b.E * (64 // 4) ** 3 * 64
    red_peak = mpm_mod.reduction_peak(n_nodes)
    reds = b.E * pos.shape[0] * 27
    scatter = {}
    for k in ("particle", "particle_recompute", "particle_adj"):
        if prof_n.get(k, 0) > 0:
            rate = reds * prof_n[k] / (prof_ms[k] / 1e3)
            scatter[k] = {"achieved": rate, "frac": rate / red_peak}
    roofline["scatter"] = {"bound": "l2 vector reductions", "unit": "node updates/s", "peak": red_peak,
                           "particle_order": a.particle_order,
                           "peak_source": "measured in this run (cls_mpm_reduction_peak, %d nodes)" % n_nodes,
                           "per_kernel": scatter}

    # end to end through the C ABI with host buffers: initial state and
    # actuation in, loss and actuation gradient out, every iteration
    e2e = None
    if a.e2e_steps > 0:
        lib, h = b.lib, b.h
        P = ctypes.POINTER(ctypes.c_double)
        pd = lambda t: ctypes.cast(t.data_ptr(), P)  # noqa: E731
        x0 = torch.from_numpy(np.ascontiguousarray(np.broadcast_to(pos, (b.E,) + pos.shape))).pin_memory()
        v0 = torch.zeros_like(x0).pin_memory()
        act = torch.from_numpy(np.random.default_rng(3).uniform(-1, 1, (T, b.E, b.M))).pin_memory()
        gact = torch.zeros_like(act).pin_memory()
        loss = ctypes.c_double()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(a.e2e_steps):
            b._c(lib.cls_mpm_set_state(h, pd(x0), pd(v0)))
            b._c(lib.cls_mpm_set_actuation(h, pd(act)))
            b._c(lib.cls_mpm_forward(h, T))
            b._c(lib.cls_mpm_loss(h, ctypes.byref(loss)))
            b._c(lib.cls_mpm_backward(h))
            b._c(lib.cls_mpm_get_grads(h, pd(gact), None, None, None, None))
        e2e_s = (time.perf_counter() - t0) / a.e2e_steps
        e2e_s = max_over_ranks(e2e_s, world)
        e2e = {"value": world * env_substeps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int((x0.numel() + v0.numel() + act.numel()) * 8),
               "d2h_bytes_per_step": int(gact.numel() * 8 + 8),
               "path": "cls_mpm_set_state/cls_mpm_set_actuation (pinned host) -> cls_mpm_forward "
                       "-> cls_mpm_loss (D2H) -> cls_mpm_backward -> cls_mpm_get_grads (D2H)"}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cores = os.cpu_count() or 1
        v, sample, wall = mpm_cpu_sample(a, 11, envs=cores, substeps=24, min_wall=10.0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": sample + "; wall %.1f s; the reference's MPM is 2D and needs Taichi" % wall}

    if rank == 0:
        line = {"metric": METRICS[a.config], "value": value, "unit": UNIT, "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_per_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded voxelised body and actuation)",
                "config": config_dict(a, world), "clocks": clocks,
                "gpu_launches": int(sum(prof_n.values())) * a.steps, "roofline": roofline,
                "e2e": e2e, "cpu_baseline": cpu}
        print(json.dumps(line))
    b.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


# ----------------------------------------------------------------- serving
def serve_oracle_sample(types, reqs, threads, cap=200):
    """Time the FP64 oracle on requests of the serving mix (episodes capped
    at `cap` substeps): forward + loss, and the reverse pass for gradient
    queries; one request per worker thread."""
    from oracle.ms_oracle import MassSpringOracle
    from cls_b200.serving import request_targets

    reqs = [r for r in reqs if hasattr(types[r.kind], "robot")]   # mass-spring requests

    def one(req):
        rb = types[req.kind].robot
        T = min(req.steps, cap)
        o = MassSpringOracle(rb.objects, rb.springs, 1, T, n_sin=8, dup_v=1, dup_h=1, dup_c=0,
                             hidden=list(rb.hidden), dt=2e-3, gravity=-9.8, ground=0.0,
                             drag=-math.log(0.99) / 2e-3, dashpot=0.1, friction=0.5,
                             spring_omega=2 * math.pi / 2e-3 / 100, run_period=100,
                             turn_period=500, jump_period=500, act_hidden="tanh", act_out="tanh",
                             out_index=rb.spring_output, n_out=rb.n_outputs,
                             loss=("velocity", "rotation"), n_threads=1)
        wr = np.random.default_rng(req.seed)
        for l in range(o.L):
            o.W[l][...] = (wr.random(o.W[l].shape) * 2 - 1) * math.sqrt(6 / o.W[l].shape[1])
        o.set_initial_state(rb.objects)
        tv, th = request_targets(req.seed, T, T, 500)
        o.set_targets(tv[:, None, :], th[:, None])
        t0 = time.perf_counter()
        if req.grad:
            o.run(T)
        else:
            o.forward(T)
            o.compute_loss(T)
        return time.perf_counter() - t0, T - 1

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        res = list(ex.map(one, reqs))
    wall = time.perf_counter() - t0
    n = sum(k for _, k in res)
    return n / wall, "%d mass-spring requests of the serving mix, episodes capped at %d substeps (FP64; " \
        "forward + loss, + reverse pass for gradient queries)" % (len(reqs), cap), wall


def run_reference_serve(a):
    from cls_b200 import workloads
    from cls_b200.serving import poisson_requests
    types, kinds, probs = workloads.serving_types()
    cores = os.cpu_count() or 1
    vals, sample = [], ""
    for i in range(a.warmup + a.steps):
        reqs = poisson_requests(np.random.default_rng(100 + i), SERVE_RATE, 2.0 * cores / SERVE_RATE,
                                kinds, probs)[:2 * cores]
        v, sample, _ = serve_oracle_sample(types, reqs, cores)
        if i >= a.warmup:
            vals.append(v)
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRICS[a.config], "value": value, "unit": UNIT,
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": config_dict(a, a.gpus),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": sample + "; requests run back to back on the host cores (no "
                                                "request loop); reference Taichi not installed"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_serve(a):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    from cls_b200 import workloads
    from cls_b200.batch import default_params
    from cls_b200.serving import Server, poisson_requests
    types, kinds, probs = workloads.serving_types()
    params = default_params(**workloads._params(a.substeps, a.checkpoint))
    srv = Server(types, {k: (SERVE_MPM_SLOTS if k.startswith("mpm") else a.robots) for k in kinds}, params,
                 tick_segments=a.tick_segments)
    # warm-up: a short burst of requests (kernels loaded, slots exercised)
    warm = poisson_requests(np.random.default_rng(77 + rank), SERVE_RATE, 0.5 * a.warmup, kinds, probs,
                            steps_hi=400)
    srv.run(warm)
    srv.results, srv.substeps_done, srv.ticks = [], 0, 0
    ms_pools = [p for p in srv.pools if hasattr(p.backend, "batch")]
    for p in ms_pools:
        p.backend.batch.profile(True)
        p.backend.batch.profile_read(reset=True)
    reqs = poisson_requests(np.random.default_rng(1000 * rank + 1), SERVE_RATE,
                            a.steps * SERVE_SECONDS_PER_STEP, kinds, probs)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    res, st = srv.run(reqs)
    torch.cuda.synchronize()
    clocks = clk.stop()
    kern_ms, launches = {}, {}
    for p in ms_pools:
        ms, n = p.backend.batch.profile_read(reset=True)
        for k in ms:
            kern_ms[k] = kern_ms.get(k, 0.0) + ms[k]
            launches[k] = launches.get(k, 0) + n[k]
    wall = st["wall_s"]
    substeps = st["env_substeps_per_s"] * wall
    wall = max_over_ranks(wall, world)
    substeps = sum_over_ranks(substeps, world)
    value = substeps / wall
    # roofline of the first-pass kernel: algorithmic bytes of the served
    # forward substeps over its device time
    fwd_bytes = 0.0
    for r in res:
        if not hasattr(types[r.kind], "robot"):
            continue
        per = workloads.algorithmic_bytes([types[r.kind].robot], [0])["forward"]
        fwd_bytes += per * (r.steps - 1)
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak, peak_src = float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        peak, peak_src = 6650.0, "fallback"
    # the pools' streams run concurrently, so per-launch event times overlap:
    # the forward kernel's achieved rate is taken over the run's wall time
    # (a lower bound)
    achieved = fwd_bytes / wall / 1e9
    roofline = {"kernel": "ms_forward_kernel (served windows)", "bound": "hbm", "achieved": achieved,
                "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_src,
                "traffic": None, "basis": "algorithmic first-pass bytes of the served requests / wall time",
                "kernel_ms_overlapping_streams": kern_ms, "launches": launches}
    n_req = max(1, len(res))

    def io_bytes(r):
        t = types[r.kind]
        if hasattr(t, "robot"):
            n = t.robot.n_vertices
            return (n * 24 + params.max_steps * 40,
                    n * 24 + 64 * a.robots * len(types) +
                    (sum(W.size + b.size for W, b in r.grads) * 8 if r.grads else 0))
        P, M = t.positions.shape[0], t.n_muscles      # MPM: state, actuation, loss in; state, grads out
        return (P * 24 + params.max_steps * (M + 4) * 8,
                P * 24 + (r.steps * M * 8 + P * 24 if r.grads else 0))

    h2d = sum(io_bytes(r)[0] for r in res) / n_req
    d2h = sum(io_bytes(r)[1] for r in res) / n_req
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cores = os.cpu_count() or 1
        sample = [r for r in reqs[:4 * cores]]
        v, desc, w = serve_oracle_sample(types, sample, cores)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": desc + "; wall %.1f s; reference Taichi not installed" % w}
    if rank == 0:
        line = {"metric": METRICS[a.config], "value": value, "unit": UNIT, "n_gpus": world,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": wall * 1e3 / a.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded Poisson arrivals, robots, targets and controllers)",
                "config": config_dict(a, world), "clocks": clocks,
                "latency_ms": {"p50": st["p50_ms"], "p99": st["p99_ms"], "mean": st["mean_ms"],
                               "queue": st["queue_ms"], "service": st["service_ms"],
                               "per_kind": st["per_kind_ms"]},
                "requests": st["requests"], "ticks": st["ticks"],
                "gpu_launches": int(sum(launches.values())), "roofline": roofline,
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": int(h2d * len(res) / a.steps),
                        "d2h_bytes_per_step": int(d2h * len(res) / a.steps),
                        "path": "Server.run: requests -> cls_serve_reset_env (host targets/state) -> "
                                "cls_serve_forward / cls_serve_backward ticks -> cls_serve_loss, "
                                "cls_serve_env_state, cls_get_grads (host results)"},
                "cpu_baseline": cpu}
        print(json.dumps(line))
    srv.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def grad_study(a):
    """How the FP32 gradient's distance from an FP64 build of the same kernels
    grows with the episode, on the uneven workload's median robot (<= 900
    vertices), over seeded draws of its inputs:

    * ``fp32_vs_fp64``: per horizon, 8 draws of the initial positions
      (the rest pose x (1 + 1e-6 u), u ~ U(-1, 1)), every input
      FP32-representable so that both builds see the same numbers: relative
      2-norm errors of the weight gradients (worst layer), of d loss / d x0
      and of the final positions;
    * ``fp64_sensitivity``: the FP64 gradient's own change under 1e-7
      relative perturbations of x0 (8 draws), i.e. how well the gradient of
      the contact model is defined at the level of FP32 rounding."""
    from cls_b200 import workloads
    from cls_b200.batch import MassSpringBatch, default_params
    robots = workloads.uneven_robots()
    fit = [r for r in robots if r.n_vertices <= 900]
    med = float(np.median([r.n_vertices for r in robots]))
    one = min(fit, key=lambda r: abs(r.n_vertices - med))

    def f32(x):
        return np.asarray(x, np.float64).astype(np.float32).astype(np.float64)

    def rel(x, y):
        x, y = np.asarray(x, np.float64).ravel(), np.asarray(y, np.float64).ravel()
        return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))

    robot = dataclasses.replace(one, objects=f32(one.objects), springs=f32(one.springs))

    def run(prec, steps, x0):
        b = MassSpringBatch([robot], [0], default_params(**workloads._params(steps, a.checkpoint,
                                                                             precision=prec)))
        rng = np.random.default_rng(5)
        tv, th = workloads.targets(rng, steps, 1)
        b.set_targets(f32(tv), f32(th))
        for l in range(len(robot.hidden) + 1):
            rows, cols = b.layer_shape(0, l)
            W = (rng.uniform(-1, 1, (rows, cols)) * np.sqrt(6 / cols)).astype(np.float32)
            b.set_weights(0, l, W.astype(np.float64), np.zeros(rows))
        b.set_state(x0)
        b.simulate(steps)
        g = [b.get_grads(0, l)[0] for l in range(len(robot.hidden) + 1)]
        gx0 = b.state_grads()[0]
        xf = b.final_state()[0]
        b.close()
        return g, gx0, xf

    pr = np.random.default_rng(77)
    draws = [f32(robot.objects * (1 + 1e-6 * pr.uniform(-1, 1, robot.objects.shape))) for _ in range(8)]
    out = {"study": "FP32 vs FP64 gradients against the episode length",
           "robot": {"vertices": robot.n_vertices, "springs": robot.n_springs,
                     "hidden": list(robot.hidden), "workload_median_vertices": med},
           "checkpoint_every": a.checkpoint, "fp32_vs_fp64": [], "fp64_sensitivity": []}
    for steps in (500, 1000, 1500, 2000):
        row = {"substeps": steps, "grad_W_rel": [], "grad_x0_rel": [], "final_x_rel": []}
        for xp in draws:
            (g32, x32, f32x), (g64, x64, f64x) = run(32, steps, xp), run(64, steps, xp)
            row["grad_W_rel"].append(max(rel(u, w) for u, w in zip(g32, g64)))
            row["grad_x0_rel"].append(rel(x32, x64))
            row["final_x_rel"].append(rel(f32x, f64x))
        row["within_1e-4"] = sum(e <= 1e-4 for e in row["grad_W_rel"])
        out["fp32_vs_fp64"].append(row)
    for steps in (1000, 2000):
        base = run(64, steps, draws[0])[0]
        d = []
        for k in range(8):
            xp = draws[0] * (1 + 1e-7 * pr.uniform(-1, 1, draws[0].shape))
            d.append(max(rel(u, w) for u, w in zip(run(64, steps, xp)[0], base)))
        out["fp64_sensitivity"].append({"substeps": steps, "x0_perturbation": 1e-7, "grad_W_rel": d})
    print(json.dumps(out))


def main():
    a = parse()
    if a.grad_study:
        grad_study(a)
    elif a.impl == "reference":
        run_reference(a)
    elif a.config == "mpm":
        run_mpm(a)
    elif a.config == "serve":
        run_serve(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
