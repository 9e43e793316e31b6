"""Where the FP32 gradient's distance from FP64 comes from on long episodes.

    python tests/study_fp32_state.py [--steps 1500,2000] [--draws 4]

CPU only (the FP64 oracle built with its precision-study hooks,
``oracle.ms_oracle.study_library``).  The robot and inputs are those of
``bench.py --grad-study``: the uneven workload's median lattice (288 vertices,
1684 springs, controller 2x128 tanh), velocity + rotation losses, every input
FP32-representable, initial positions drawn as the rest pose x (1 + 1e-6 u).

Each case runs the oracle in FP64 and then with one kind of stored field
rounded to FP32 after every write (the arithmetic stays FP64), and reports the
weight gradient's relative 2-norm distance from the plain FP64 run (worst
layer) with the number of contact decisions of advance_toi
(multitask/solver_mass_spring.py:129) that differ from the FP64 run:

* ``x``, ``v``, ``v_inc``, ``mlp`` (pre-activations and activations),
  ``input`` (controller input and centre), ``adjoint`` (d x, d v, d v_inc),
  ``wsum`` (the weight-gradient sums), ``forward`` (x, v, v_inc, mlp, input);
* ``x_exact``: positions kept exactly (a compensated position update) while
  every reader sees them rounded; ``forward_x_exact`` the same with the other
  forward fields rounded;
* ``forward_exact_flags``: ``forward`` with the FP64 run's contact decisions
  forced, to separate branch flips from the rest.

Prints one JSON object per (substeps, draw) case.
"""
import argparse
import ctypes
import dataclasses
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

from cls_b200 import workloads  # noqa: E402
from cls_b200.batch import default_params  # noqa: E402
from helpers import workload_oracle_kwargs  # noqa: E402
from oracle.ms_oracle import MassSpringOracle, study_library  # noqa: E402

# ST_* bits of oracle/ms_oracle.c
ST_X, ST_V, ST_VINC, ST_MLP, ST_INPUT, ST_ADJ, ST_WSUM, ST_X_EXACT = 1, 2, 4, 8, 16, 32, 64, 128
FORWARD = ST_X | ST_V | ST_VINC | ST_MLP | ST_INPUT
VARIANTS = [("x", ST_X), ("v", ST_V), ("v_inc", ST_VINC), ("mlp", ST_MLP), ("input", ST_INPUT),
            ("adjoint", ST_ADJ), ("wsum", ST_WSUM), ("forward", FORWARD), ("x_exact", ST_X_EXACT),
            ("forward_x_exact", (FORWARD & ~ST_X) | ST_X_EXACT)]


def f32(x):
    return np.asarray(x, np.float64).astype(np.float32).astype(np.float64)


def rel(x, y):
    x, y = np.asarray(x).ravel(), np.asarray(y).ravel()
    return float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))


def median_robot():
    robots = workloads.uneven_robots()
    fit = [r for r in robots if r.n_vertices <= 900]
    med = float(np.median([r.n_vertices for r in robots]))
    one = min(fit, key=lambda r: abs(r.n_vertices - med))
    return dataclasses.replace(one, objects=f32(one.objects), springs=f32(one.springs))


def make_oracle(robot, steps, x0, lib):
    p = default_params(**workloads._params(steps, 50, precision=64))
    o = MassSpringOracle(robot.objects, robot.springs, 1, steps, initial_objects=robot.objects,
                         **workload_oracle_kwargs(p, robot))
    o.lib = lib
    rng = np.random.default_rng(5)
    tv, th = workloads.targets(rng, steps, 1)
    o.set_targets(f32(tv), f32(th))
    Ws, bs = [], []
    for l in range(o.L):
        rows, cols = o.W[l].shape
        Ws.append(f32(rng.uniform(-1, 1, (rows, cols)) * np.sqrt(6 / cols)))
        bs.append(np.zeros(rows))
    o.set_weights(Ws, bs)
    o.x[0, 0] = x0
    return o


def run(o, lib, steps, bits, flags, mode, x_exact):
    if x_exact is not None:
        x_exact[...] = 0.0
        x_exact[0] = o.x[0]
    lib.orc_study_set(bits, flags.ctypes.data, mode, None if x_exact is None else x_exact.ctypes.data)
    try:
        o.run(steps)
    finally:
        lib.orc_study_set(0, None, 0, None)
    return [g.copy() for g in o.gW]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", default="1500,2000")
    ap.add_argument("--draws", type=int, default=4)
    a = ap.parse_args()
    lib = study_library()
    robot = median_robot()
    pr = np.random.default_rng(77)
    draws = [f32(robot.objects * (1 + 1e-6 * pr.uniform(-1, 1, robot.objects.shape))) for _ in range(8)]
    for steps in (int(s) for s in a.steps.split(",")):
        for d in range(a.draws):
            o = make_oracle(robot, steps, draws[d], lib)
            exact_flags = np.zeros((steps, 1, robot.n_vertices), np.uint8)
            xe = np.zeros_like(o.x)
            g64 = run(o, lib, steps, 0, exact_flags, 1, None)
            res = {"substeps": steps, "draw": d, "contact_decisions": int(exact_flags.sum())}
            for name, bits in VARIANTS:
                flags = np.zeros_like(exact_flags)
                g = run(o, lib, steps, bits, flags, 1, xe if bits & ST_X_EXACT else None)
                res[name] = {"grad_W_rel": max(rel(u, w) for u, w in zip(g, g64)),
                             "contact_flips": int((flags != exact_flags).sum())}
            g = run(o, lib, steps, FORWARD, exact_flags.copy(), 2, None)
            res["forward_exact_flags"] = {"grad_W_rel": max(rel(u, w) for u, w in zip(g, g64)),
                                          "contact_flips": 0}
            print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
