"""Seeded synthetic workloads with the shapes of the benchmark configurations.

All inputs are generated from a seed (no dataset is involved):

* ``quadruped_batch``   -- one quadruped lattice (torso 4x2x1 cubes on four
  1x1x2 legs), 32 envs, 1000 substeps, 1 hidden layer of 64 tanh;
* ``uneven_batch``      -- 512 random lattices of 50-2000 vertices (log-uniform),
  30 % of springs actuated, 2000 substeps, checkpoint every 50, MLP 2x128 tanh;
* ``spider_batch``      -- 4096 envs of a spider-like lattice (3x3x1 torso, eight
  1x1x3 legs, 96 actuators), 1000 substeps, MLP 2x256 tanh.

Physics of these synthetic configurations: stiffness 3e4 (the reference's
/10 scaling applies), dt 2e-3, gravity -9.8, ground at y = 0 with friction 0.5,
velocity damping 0.99 per substep (drag = -ln(0.99) / dt).  The controller
input is the reference's layout with 8 sinusoids and one copy of each goal
value.
"""
import math

import numpy as np

from . import robot_design
from .batch import MassSpringBatch, Robot, default_params

PHYSICS = dict(dt=2e-3, gravity=-9.8, ground_height=0.0, friction=0.5,
               drag_damping=-math.log(0.99) / 2e-3, dashpot_damping=0.1, stiffness_scale=0.1)


def _params(steps, K, hidden_act="tanh", precision=32, loss=("velocity", "rotation"), **over):
    p = dict(PHYSICS)
    p.update(max_steps=steps, checkpoint_every=K, run_period=100, turn_period=500,
             jump_period=500, spring_omega=2 * math.pi / p["dt"] / 100, n_sin_waves=8,
             duplicate_v=1, duplicate_h=1, duplicate_c=0, activation_hidden=hidden_act,
             activation_output=hidden_act, loss=list(loss), precision=precision,
             max_speed=0.1, max_height=0.1)
    p.update(over)
    return p


def targets(rng, T, n_envs, turn_period=500, lo=-0.1, hi=0.1):
    """Goal values (target vx, vz, height) ~ U(lo, hi), one draw per env per
    turn period, held for the period."""
    n_blocks = T // turn_period + 1
    draws = rng.uniform(lo, hi, size=(n_blocks, n_envs, 3))
    idx = np.arange(T) // turn_period
    tv = np.zeros((T, n_envs, 3))
    tv[:, :, 0] = draws[idx, :, 0]
    tv[:, :, 2] = draws[idx, :, 1]
    th = draws[idx, :, 2]
    return tv, th


def uneven_robots(n_robots=512, seed=0, vmin=50, vmax=2000, hidden=(128, 128)):
    rng = np.random.default_rng(seed)
    robots = []
    for _ in range(n_robots):
        n = int(round(math.exp(rng.uniform(math.log(vmin), math.log(vmax)))))
        obj, spr = robot_design.random_lattice(rng, n)
        robots.append(Robot.actuated_outputs(obj, spr, hidden=list(hidden)))
    return robots


def uneven_batch(n_robots=512, steps=2000, K=50, seed=0, precision=32, hidden=(128, 128),
                 vmin=50, vmax=2000, robots=None, **over):
    """Batched uneven mass-spring: every robot its own type and controller."""
    robots = robots if robots is not None else uneven_robots(n_robots, seed, vmin, vmax, hidden)
    p = default_params(**_params(steps, K, precision=precision, **over))
    b = MassSpringBatch(robots, list(range(len(robots))), p)
    rng = np.random.default_rng(seed + 1)
    tv, th = targets(rng, steps, len(robots))
    b.set_targets(tv, th)
    b.weights_init(seed + 2)
    return b, robots, (tv, th)


def quadruped_batch(n_envs=32, steps=1000, K=50, seed=0, precision=32, weights_seed=None, **over):
    obj, spr = robot_design.quadruped_lattice()
    robot = Robot.actuated_outputs(obj, spr, hidden=[64])
    p = default_params(**_params(steps, K, precision=precision, **over))
    b = MassSpringBatch([robot], [0] * n_envs, p)
    rng = np.random.default_rng(seed + 1)
    tv, th = targets(rng, steps, n_envs)
    b.set_targets(tv, th)
    b.weights_init(seed + 2 if weights_seed is None else weights_seed)
    return b, [robot], (tv, th)


def spider_batch(n_envs=4096, steps=1000, K=50, seed=0, precision=32, weights_seed=None, **over):
    obj, spr = robot_design.spider_lattice()
    robot = Robot.actuated_outputs(obj, spr, hidden=[256, 256])
    p = default_params(**_params(steps, K, precision=precision, **over))
    b = MassSpringBatch([robot], [0] * n_envs, p)
    rng = np.random.default_rng(seed + 1)
    tv, th = targets(rng, steps, n_envs)
    b.set_targets(tv, th)
    b.weights_init(seed + 2 if weights_seed is None else weights_seed)
    return b, [robot], (tv, th)


def _widths(rb):
    N, S = rb.n_vertices, rb.n_springs
    return [(-(-3 * N // 4) * 4) + 8 + 2 + 1] + list(rb.hidden) + [rb.n_outputs if rb.n_outputs > 0 else S]


def algorithmic_bytes(robots, env_robot, keep_trajectory=True, dtype_bytes=4, batched=False, replay=False):
    """Compulsory DRAM bytes per substep of the whole batch, per kernel.

    Fused per-env path, per env-substep of robot r (N vertices, S springs, MLP
    rows x pitch):
      weights:   sum_l rows_l * pitch_l * 4   (read once per pass; the batch's
                 weights exceed L2, so every pass streams them)
      forward:   weights + trajectory write 16 N (x[t], when kept)
      recompute: weights + record writes 32 N (x, v) + 4 n_c (input) + 4 sum rows
      reverse:   weights + record reads 32 N + 4 sum rows (z) + writes 4 sum rows
                 (dz) + trajectory reads 32 N (rotation loss at t - rp, t + rp)
    The spring table (32 B per incidence, 2 S per robot) is read from L2 each
    substep and counted once per pass.  With ``replay`` (whole-episode
    controller records, episodes of several segments), the first pass also
    writes every substep's controller records (4 n_c + 4 sum rows) and the
    recompute reads only the output layer's pre-activations (4 n_out) instead
    of the weights:
      forward:   weights + trajectory 16 N + 4 n_c + 4 sum rows
      recompute: record writes 32 N (x, v) + 4 n_out

    Batched-controller path, step kernels only (the controller's GEMMs are
    counted in FLOPs by controller_flops), per env-substep:
      forward:   state read + write 64 N, input row write 4 n_c, output-layer
                 pre-activations read 4 n_out, trajectory write 16 N
      recompute: forward without the trajectory + record writes 32 N (x, v)
                 + 16 N (v_inc)
      reverse:   record reads 48 N (x, v, v_inc) + 16 N (x of t + 1), adjoint
                 state read + write 64 N, d input positions 12 N, output-layer
                 z read + dz write 8 n_out, trajectory reads 32 N
    """
    out = dict(forward=0.0, recompute=0.0, reverse=0.0)
    for r in env_robot:
        rb = robots[r]
        N, S = rb.n_vertices, rb.n_springs
        widths = _widths(rb)
        traj = 16 * N if keep_trajectory else 0
        if batched:
            n_c, n_out = widths[0], widths[-1]
            out["forward"] += 64 * N + 4 * n_c + 4 * n_out + traj
            out["recompute"] += 64 * N + 4 * n_c + 4 * n_out + 48 * N
            out["reverse"] += 64 * N + 64 * N + 12 * N + 8 * n_out + 2 * traj
            continue
        pitch = [-(-w // 4) * 4 for w in widths]
        wbytes = sum(widths[l + 1] * pitch[l] for l in range(len(widths) - 1)) * dtype_bytes
        rows = sum(widths[1:]) * dtype_bytes
        springs = 2 * S * 32
        if replay:
            out["forward"] += wbytes + springs + traj + widths[0] * dtype_bytes + rows
            out["recompute"] += springs + 32 * N + widths[-1] * dtype_bytes
        else:
            out["forward"] += wbytes + springs + traj
            out["recompute"] += wbytes + springs + 32 * N + widths[0] * dtype_bytes + rows
        out["reverse"] += wbytes + springs + 32 * N + 2 * rows + 2 * traj
    return out


def controller_flops(robots, env_robot):
    """Useful FP32 FLOPs (2 M N K) of the batched controller's GEMMs per
    substep of the whole batch: forward (every layer, K = the layer's inputs)
    and adjoint (every layer back to its inputs; the first layer only to the
    3 N position columns)."""
    fw = ad = 0.0
    for r in env_robot:
        rb = robots[r]
        w = _widths(rb)
        for l in range(len(w) - 1):
            fw += 2.0 * w[l + 1] * w[l]
            ad += 2.0 * w[l + 1] * (w[l] if l > 0 else 3 * rb.n_vertices)
    return {"forward": fw, "adjoint": ad}


def legged_body(n_grid=64, ppc=2, torso=(24, 8, 14), leg=(5, 10, 5), origin_cells=(18, 4, 25)):
    """Voxelised legged body for the 3D MPM configuration: a torso box on four
    legs, ppc^3 particles per cell at cell-centred sub-positions.  Each leg is
    split into 4 muscle groups (front/back half x upper/lower half) = 16 groups
    with vertical fibres; the torso is passive.  Returns positions [P][3],
    muscle [P], fibre [P][3]."""
    dx = 1.0 / n_grid
    ox, oy, oz = origin_cells
    pts, mus = [], []

    def add_box(c0, size, muscle_of):
        for i in range(size[0]):
            for j in range(size[1]):
                for k in range(size[2]):
                    m = muscle_of(i, j, k)
                    for a in range(ppc):
                        for b in range(ppc):
                            for c in range(ppc):
                                pts.append(((c0[0] + i + (a + 0.5) / ppc) * dx,
                                            (c0[1] + j + (b + 0.5) / ppc) * dx,
                                            (c0[2] + k + (c + 0.5) / ppc) * dx))
                                mus.append(m)

    lx, ly, lz = leg
    tx, ty, tz = torso
    corners = [(0, 0), (tx - lx, 0), (0, tz - lz), (tx - lx, tz - lz)]
    for li, (cx, cz) in enumerate(corners):
        add_box((ox + cx, oy, oz + cz), leg,
                lambda i, j, k, li=li: 4 * li + (0 if i < lx // 2 else 1) + (0 if j < ly // 2 else 2))
    add_box((ox, oy + ly, oz), torso, lambda i, j, k: -1)
    pos = np.array(pts)
    fib = np.zeros_like(pos)
    fib[:, 1] = 1.0
    return pos, np.array(mus, dtype=np.int32), fib


def mpm_batch(n_envs=8, steps=1000, K=50, seed=0, precision=32, n_grid=64, **over):
    """3D MLS-MPM configuration: legged body on a 64^3 grid, neo-Hookean
    (E = 1e4, nu = 0.3), 16 fibre-actuated muscle groups driven by seeded
    sinusoids, dt = 1e-4, sticky walls and floor; the loss tracks the body's
    centre towards a point 0.05 ahead at the last step."""
    from . import mpm as mpm_mod
    pos, mus, fib = legged_body(n_grid=n_grid)
    E, nu = 1e4, 0.3
    mu, la = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
    b = mpm_mod.MPMBatch(pos, mus, n_envs, dim=3, fibre=fib, n_muscles=16, max_steps=steps,
                         n_grid=n_grid, bound=3, material="neo_hookean", precision=precision,
                         checkpoint_every=K, dt=1e-4, gravity=-10.0, p_vol=1.0, mu=mu, la=la,
                         act_strength=1e3, mass=1.0, **over)
    rng = np.random.default_rng(seed)
    t = np.arange(steps)[:, None, None] * 1e-4
    freq = rng.uniform(2.0, 6.0, size=(1, n_envs, 16))
    phase = rng.uniform(0, 2 * np.pi, size=(1, n_envs, 16))
    b.set_actuation(np.sin(2 * np.pi * freq * t + phase))
    w = np.zeros(steps + 1)
    w[steps] = 1.0
    c0 = pos.mean(axis=0)
    target = np.broadcast_to(c0 + np.array([0.05, 0.0, 0.0]), (steps + 1, n_envs, 3)).copy()
    b.set_loss(w, target)
    return b, pos


def mpm_touched_nodes(pos, n_grid=64):
    """Grid nodes inside the 3^D quadratic B-spline stencil of at least one
    particle at positions `pos` [P][D]."""
    base = np.floor(pos * n_grid - 0.5).astype(np.int64)
    D = pos.shape[1]
    offs = np.stack(np.meshgrid(*([np.arange(3)] * D), indexing="ij"), -1).reshape(-1, D)
    nodes = (base[:, None, :] + offs[None, :, :]).reshape(-1, D)
    key = np.zeros(len(nodes), dtype=np.int64)
    for d in range(D):
        key = key * n_grid + nodes[:, d]
    return int(np.unique(key).size)


def mpm_algorithmic_bytes(pos, n_envs, n_grid=64, dtype_bytes=4):
    """Compulsory DRAM bytes of ONE launch of each MPM kernel over the batch
    (FP32, 3D; P particles and G touched grid nodes per env; grid nodes are
    16-byte (velocity, mass) / (momentum, mass) records):

      particle:            G2P of step f + P2G of step f+1: read x, F, muscle
                           id, fibre, centre weight (68 P), write x, F (48 P);
                           gather the staged grid (16 G), flush the tile (16 G)
      particle_recompute:  the same + v, C of the recorded step (48 P)
      grid:                read the accumulator (16 G), write (velocity, mass)
                           (16 G), clear the accumulator (16 G)
      particle_adj:        P2G^T of step f + G2P^T of step f-1: read x, v, C, F
                           of step f, muscle id, fibre, weight (116 P), a_x and
                           a_F in (48 P), x of step f-1 (12 P); write a_x, a_F
                           (48 P); grid adjoint and grid gathers (32 G), flush
                           of the velocity adjoint (16 G)
      grid_adj:            read the adjoint accumulator and the grid (32 G),
                           write the grid adjoint (16 G), clear (16 G)
    """
    P, D = pos.shape
    G = mpm_touched_nodes(pos, n_grid)
    s = dtype_bytes / 4.0
    per_env = {
        "particle": 116 * P + 32 * G,
        "particle_recompute": 164 * P + 32 * G,
        "grid": 48 * G,
        "particle_adj": 224 * P + 48 * G,
        "grid_adj": 64 * G,
    }
    return {k: v * s * n_envs for k, v in per_env.items()}


def mpm_serving_type(n_grid=64):
    """The 3D MPM configuration's body and solver as a served type: the
    legged body, neo-Hookean E = 1e4, nu = 0.3, 16 fibre muscle groups,
    dt = 1e-4, FP32."""
    from .serving import MpmType
    pos, mus, fib = legged_body(n_grid=n_grid)
    E, nu = 1e4, 0.3
    solver = dict(n_grid=n_grid, bound=3, material="neo_hookean", precision=32, dt=1e-4, gravity=-10.0,
                  p_vol=1.0, mu=E / (2 * (1 + nu)), la=E * nu / ((1 + nu) * (1 - 2 * nu)), act_strength=1e3,
                  mass=1.0)
    return MpmType(pos, mus, fib, n_muscles=16, solver=solver)


def serving_types(seed=0, lattice_sizes=(100, 300, 800, 1500), mpm=True):
    """Robot types of the serving workload (the training configurations'
    robots): the quadruped lattice (MLP 1x64), the spider lattice (MLP
    2x256), random lattices of the uneven batch (MLP 2x128) and, with
    ``mpm``, the MPM legged body, with the request mix: quadruped 25 %,
    spider 20 %, MPM body 5 %, lattices 50 % (equal shares); without MPM the
    spider takes its 5 %.  Controllers are drawn per type by the server."""
    from .serving import RobotType
    types = {}
    obj, spr = robot_design.quadruped_lattice()
    types["quadruped"] = RobotType(Robot.actuated_outputs(obj, spr, hidden=[64]))
    obj, spr = robot_design.spider_lattice()
    types["spider"] = RobotType(Robot.actuated_outputs(obj, spr, hidden=[256, 256]))
    rng = np.random.default_rng(seed)
    for n in lattice_sizes:
        o, s = robot_design.random_lattice(rng, n)
        types["lattice%d" % n] = RobotType(Robot.actuated_outputs(o, s, hidden=[128, 128]))
    if mpm:
        types["mpm_legged"] = mpm_serving_type()
    kinds = list(types)
    p = [0.25, 0.20 if mpm else 0.25] + [0.5 / len(lattice_sizes)] * len(lattice_sizes) + ([0.05] if mpm else [])
    return types, kinds, p
