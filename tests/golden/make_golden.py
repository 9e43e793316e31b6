"""Generate golden vectors for the mass-spring path by running the reference's
own Python/Taichi kernel source under a NumPy interpretation of the Taichi
primitives it uses (``taichi_numpy_shim.py``; Taichi itself is absent here).

Run in a container where the reference checkout is readable:

    python tests/golden/make_golden.py --reference /root/reference

It constructs the reference ``ConfigSim`` / ``DiffPhyTrainer`` /
``TaichiEnv`` / ``SolverMassSpring`` / ``Model`` objects unchanged, initialises
weights and training targets through the reference's ``weights_init`` and
``initialize_train`` (fed by a seeded ``ti.random``), and calls the reference's
``DiffPhyTrainer.simulate`` (multitask/diffphy_trainer.py:219-268), which runs
``clear_states``, ``nn.clear``, the substep loop (``pre_advance``,
``nn_input``, ``nn.forward``, ``advance``) and ``get_loss``.  The resulting
fields are written to ``tests/golden/<case>.npz``.  Gradients are not produced
(the shim's ``ti.ad.Tape`` is a no-op); tests pin the oracle's gradients with
finite differences of this forward instead.

Nothing in the product reads these files; tests do.
"""
import argparse
import copy
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# Small cases: reference robots and reference cfg3d files, with the horizon,
# batch and task periods shortened so the pure-Python run stays in seconds while
# every loss window is exercised.
CASES = {
    # the reference quadruped exactly as cfg3d/sim_quad.json (n_in = 838, sin MLP)
    "quad_ref": dict(cfg="sim_quad", seed=11, train=True,
                     over={"nn": {"batch_size": 2},
                           "process": {"max_steps": 48, "run_period": 10,
                                       "turn_period": 24, "jump_period": 24}},
                     steps=48, loss={"velocity", "rotation"}),
    # spider (skeleton.json), exercises the head/tail rotation branch
    "spider_ref": dict(cfg="sim_spider", seed=12, train=True,
                       over={"nn": {"batch_size": 2, "n_sin_waves": 20,
                                    "duplicate_v": 10, "duplicate_h": 10},
                             "process": {"max_steps": 40, "run_period": 8,
                                         "turn_period": 20, "jump_period": 20}},
                       steps=40, loss={"velocity", "rotation"}),
    # robot 101 with every 3D loss switched on and a crawl target planted
    "x_all_losses": dict(cfg="sim_x", seed=13, train=True,
                         over={"nn": {"batch_size": 3, "n_sin_waves": 8,
                                      "duplicate_v": 4, "duplicate_h": 3,
                                      "duplicate_c": 2, "n_hidden": 24},
                               "process": {"max_steps": 40, "run_period": 6,
                                           "turn_period": 16, "jump_period": 13}},
                         steps=38,
                         loss={"velocity", "rotation", "height", "pose",
                               "actuation", "crawl"},
                         crawl_env=1),
    # snake (robot 104), forward-only evaluation rollout with scripted targets
    "snake_eval": dict(cfg="sim_snake", seed=14, train=False,
                       over={"nn": {"batch_size": 1, "n_sin_waves": 16,
                                    "duplicate_v": 4, "duplicate_h": 4},
                             "process": {"max_steps": 36, "run_period": 6,
                                         "turn_period": 15, "jump_period": 15}},
                       steps=34, loss={"velocity", "rotation"}),
}


def install_shims():
    sys.path.insert(0, HERE)
    import taichi_numpy_shim as ti_shim
    sys.modules["taichi"] = ti_shim
    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    for name in ("figure", "plot", "close", "savefig"):
        setattr(plt, name, lambda *a, **k: None)
    mpl.pyplot = plt
    sys.modules["matplotlib"] = mpl
    sys.modules["matplotlib.pyplot"] = plt
    return ti_shim


def deep_update(d, over):
    for k, v in over.items():
        if isinstance(v, dict):
            deep_update(d[k], v)
        else:
            d[k] = v


def run_case(name, spec, ref_root, ti_shim):
    from multitask.config_sim import ConfigSim
    from multitask.diffphy_trainer import DiffPhyTrainer
    from util import read_json

    path = "cfg3d/{}.json".format(spec["cfg"])
    raw = read_json(path)
    deep_update(raw, copy.deepcopy(spec["over"]))
    config = ConfigSim(raw, file_name=path, if_mkdir=False)
    args = types.SimpleNamespace(evaluate=False, num_processes=1, no_tensorboard=True)
    trainer = DiffPhyTrainer(args, config)
    env = trainer.taichi_env
    env.setup_robot()
    ti_shim.seed(spec["seed"])
    trainer.nn.weights_init()
    weights = [w.to_numpy() for w in trainer.nn.weights]
    steps = spec["steps"]
    cfg = config.get_config()
    if spec.get("crawl_env") is not None:
        env.target_c.arr[:, spec["crawl_env"]] = 1.0
    x0 = env.x.to_numpy()[0].copy()
    trainer.simulate(steps, iter=0, train=spec["train"],
                     max_height=cfg["process"]["max_height"],
                     max_speed=cfg["process"]["max_speed"],
                     loss_enable=spec["loss"])
    sol = env.solver
    springs = np.array(cfg["robot"]["springs"], dtype=np.float64)
    out = dict(
        steps=np.int64(steps), train=np.int64(spec["train"]),
        T=np.int64(cfg["process"]["max_steps"]), B=np.int64(cfg["nn"]["batch_size"]),
        robot_id=np.int64(cfg["robot"]["robot_id"]),
        dt=np.float64(cfg["process"]["dt"]), gravity=np.float64(cfg["simulator"]["gravity"]),
        ground=np.float64(cfg["simulator"]["ground_height"]),
        drag=np.float64(cfg["simulator"]["drag_damping"]),
        dashpot=np.float64(cfg["simulator"]["dashpot_damping"]),
        spring_omega=np.float64(cfg["process"]["spring_omega"]),
        run_period=np.int64(cfg["process"]["run_period"]),
        turn_period=np.int64(cfg["process"]["turn_period"]),
        jump_period=np.int64(cfg["process"]["jump_period"]),
        max_speed=np.float64(cfg["process"]["max_speed"]),
        max_height=np.float64(cfg["process"]["max_height"]),
        n_sin=np.int64(cfg["nn"]["n_sin_waves"]), dup_v=np.int64(cfg["nn"]["duplicate_v"]),
        dup_h=np.int64(cfg["nn"]["duplicate_h"]), dup_c=np.int64(cfg["nn"]["duplicate_c"]),
        n_hidden=np.int64(cfg["nn"]["n_hidden"]),
        loss_names=np.array(sorted(spec["loss"])),
        objects=np.array(cfg["robot"]["objects"], dtype=np.float64),
        springs=springs,
        W1=weights[0], W2=weights[1], b1=weights[2], b2=weights[3],
        x0=x0,
        x=env.x.to_numpy(), v=env.v.to_numpy(),
        center=env.center.to_numpy(), height=env.height.to_numpy(),
        upper_height=env.upper_height.to_numpy(), rotation=env.rotation.to_numpy(),
        actuation=env.actuation.to_numpy(),
        hidden=trainer.nn.hidden.to_numpy(), output=trainer.nn.output.to_numpy(),
        input_state=env.input_state.to_numpy(),
        target_v=env.target_v.to_numpy(), target_h=env.target_h.to_numpy(),
        target_c=env.target_c.to_numpy(),
        loss=np.float64(env.loss[None]),
        loss_terms=np.array([env.loss_dict[k][None] for k in
                             ("loss_velocity", "loss_height", "loss_pose", "loss_rotation",
                              "loss_weight", "loss_actuation", "loss_crawl")]),
        loss_batch=env.loss_batch.to_numpy(),
        loss_terms_batch=np.stack([env.loss_dict_batch[k].to_numpy() for k in
                                   ("loss_velocity", "loss_height", "loss_pose", "loss_rotation",
                                    "loss_weight", "loss_actuation", "loss_crawl")]),
        current_max_height=np.float64(env.current_max_height[None]),
    )
    return out


def robot_geometry(ref_root):
    """objects / springs / faces of the five 3D robots from the reference's own
    builder (multitask/robot_design.py:319-591)."""
    from multitask.robot_design import RobotDesignMassSpring3D
    out = {}
    for name in ("sim_quad", "sim_x", "sim_y", "sim_spider", "sim_snake"):
        builder = RobotDesignMassSpring3D.from_file("cfg3d/%s.json" % name)
        objects, springs, faces = builder.build()
        rid = builder.robot_id
        out["objects_%d" % rid] = np.array(objects, dtype=np.float64)
        out["springs_%d" % rid] = np.array(springs, dtype=np.float64)
        out["faces_%d" % rid] = np.array(faces, dtype=np.int64)
        out["stiffness_%d" % rid] = np.float64(builder.spring_stiffness)
        out["actuation_%d" % rid] = np.float64(builder.spring_actuation)
    # the spider's node / link table (cfg3d/skeleton.json), so that the tests
    # can rebuild robot 103 without the reference tree
    with open("cfg3d/skeleton.json") as f:
        sk = json.load(f)
    keys = list(sk["nodes"])
    out["skeleton_node_keys"] = np.array(keys)
    out["skeleton_nodes"] = np.array([sk["nodes"][k] for k in keys], dtype=np.float64)
    out["skeleton_links"] = np.array(sk["links"], dtype=np.int64)
    return out


def _jsonable(v):
    if isinstance(v, (set, frozenset)):
        return sorted(v)
    if isinstance(v, (list, tuple)):
        return [_jsonable(x) for x in v]
    if isinstance(v, dict):
        return {k: _jsonable(x) for k, x in v.items()}
    if isinstance(v, np.generic):
        return v.item()
    return v


def simulate_trace(ti_shim):
    """The calls that the reference's own DiffPhyTrainer.simulate
    (multitask/diffphy_trainer.py:219-268) makes on its env, solver and model,
    recorded by running that method unchanged on recording stand-ins, for the
    golden cases quad_ref (training rollout) and snake_eval (evaluation
    rollout).  Entries are [object, method, args, kwargs]; ``tape`` marks the
    ti.ad.Tape context.  The drop-in objects replay this trace on the GPU."""
    from multitask.diffphy_trainer import DiffPhyTrainer
    calls = []

    class Scalar:
        def __init__(self, name):
            self.name = name

        def __setitem__(self, key, value):
            calls.append([self.name, "__setitem__", [key, _jsonable(value)], {}])

    class Obj:
        def __init__(self, name, **attrs):
            self._name = name
            self.__dict__.update(attrs)

        def __getattr__(self, attr):
            if attr.startswith("__"):
                raise AttributeError(attr)
            return lambda *a, **k: calls.append([self._name, attr, _jsonable(list(a)), _jsonable(k)])

    class Tape:
        def __init__(self, loss):
            calls.append(["tape", "__enter__", [loss.name], {}])

        def __enter__(self):
            return self

        def __exit__(self, *exc):
            calls.append(["tape", "__exit__", [], {}])
            return False

    losses = [Scalar("env.losses[%d]" % i) for i in range(7)]
    env = Obj("env", solver=Obj("solver"), loss=Scalar("env.loss"), losses=losses, dim=3)
    out = {}
    saved = ti_shim.ad.Tape
    ti_shim.ad.Tape = Tape
    try:
        for name in ("quad_ref", "snake_eval"):
            spec = CASES[name]
            path = "cfg3d/{}.json".format(spec["cfg"])
            with open(path) as f:
                raw = json.load(f)
            deep_update(raw, copy.deepcopy(spec["over"]))
            pr = raw["process"]
            fake = types.SimpleNamespace(taichi_env=env, nn=Obj("nn"),
                                         control_length=raw["robot"]["control_length"])
            del calls[:]
            DiffPhyTrainer.simulate(fake, spec["steps"], iter=0, train=spec["train"],
                                    max_height=pr["max_height"], max_speed=pr["max_speed"],
                                    loss_enable=spec["loss"])
            out[name] = dict(steps=spec["steps"], train=spec["train"], calls=list(calls))
    finally:
        ti_shim.ad.Tape = saved
    return out


def run_mpm_case(steps=24, B=2, seed=21):
    """The reference's 2D MLS-MPM kernels (multitask/solver_mpm.py:60-165) on
    its MPM robot design robot_design/robot_mpm_1.json.  The reference's env
    cannot construct this solver (taichi_env.py:136 omits the config), so the
    solver is constructed and stepped directly: clear_states, then per step
    clear_grid, p2g, grid_op, g2p (advance_core's forward, :175-180)."""
    from multitask.config_sim import ConfigSim
    from multitask.solver_mpm import SolverMPM
    from util import read_json
    path = "cfg3d/sim_quad.json"
    raw = read_json(path)
    raw["robot"].update({"dim": 2, "simulator": "mpm", "solver": "mpm",
                         "design_file": "robot_design/robot_mpm_1.json"})
    raw["nn"]["batch_size"] = B
    raw["process"]["max_steps"] = steps + 1
    config = ConfigSim(raw, file_name=path, if_mkdir=False)
    cfg = config.get_config()
    solver = SolverMPM(config)
    solver.initialize_robot()
    objects = np.array(cfg["robot"]["objects"], dtype=np.float64) + np.array([0.35, 0.12])
    for k in range(B):
        solver.x.arr[0, k] = objects
    rng = np.random.default_rng(seed)
    act = rng.uniform(-1.0, 1.0, size=(steps + 1, B, 4))
    solver.actuation.arr[:, :, :4] = act
    solver.clear_states(steps + 1)
    for f in range(steps):
        solver.clear_grid()
        solver.p2g(f)
        solver.grid_op()
        solver.g2p(f)
    sim = cfg["simulator"]
    return dict(
        steps=np.int64(steps), B=np.int64(B), n_grid=np.int64(sim["mpm"]["n_grid"]),
        dx=np.float64(sim["mpm"]["dx"]), inv_dx=np.float64(sim["mpm"]["inv_dx"]),
        dt=np.float64(cfg["process"]["dt"]), gravity=np.float64(sim["gravity"]),
        p_vol=np.float64(sim["p_vol"]), E=np.float64(sim["E"]), mu=np.float64(sim["mu"]),
        la=np.float64(sim["la"]), act_strength=np.float64(sim["act_strength"]),
        bound=np.int64(sim["bound"]), actuator_id=np.array(cfg["robot"]["springs"], dtype=np.int64),
        objects=objects, actuation=act,
        x=solver.x.to_numpy()[:steps + 1], v=solver.v.to_numpy()[:steps + 1],
        C=solver.C.to_numpy()[:steps + 1], F=solver.F.to_numpy()[:steps + 1])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("CLS_REFERENCE_ROOT"),
                    help="root of the reference checkout (default: $CLS_REFERENCE_ROOT)")
    ap.add_argument("--cases", nargs="*", default=sorted(CASES))
    ap.add_argument("--only-robots", action="store_true",
                    help="regenerate robots.npz only")
    ap.add_argument("--only-trace", action="store_true",
                    help="regenerate simulate_trace.json only")
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    if not a.reference:
        ap.error("--reference (or CLS_REFERENCE_ROOT) is required")
    ti_shim = install_shims()
    ref_root = os.path.abspath(a.reference)
    sys.path.insert(0, ref_root)
    cwd = os.getcwd()
    out_dir = os.path.abspath(a.out)
    os.chdir(ref_root)  # the reference opens cfg3d/*.json relative to its root
    try:
        if a.only_robots:
            geo = robot_geometry(ref_root)
            np.savez_compressed(os.path.join(out_dir, "robots.npz"), **geo)
            return
        if a.only_trace:
            with open(os.path.join(out_dir, "simulate_trace.json"), "w") as f:
                json.dump(simulate_trace(ti_shim), f, indent=0)
            return
        mpm = run_mpm_case()
        np.savez_compressed(os.path.join(out_dir, "mpm2d_ref.npz"), **mpm)
        print("mpm2d_ref x", mpm["x"].shape)
        geo = robot_geometry(ref_root)
        np.savez_compressed(os.path.join(out_dir, "robots.npz"), **geo)
        print("robots", sorted(k for k in geo if k.startswith("objects")))
        with open(os.path.join(out_dir, "simulate_trace.json"), "w") as f:
            json.dump(simulate_trace(ti_shim), f, indent=0)
        for name in a.cases:
            data = run_case(name, CASES[name], ref_root, ti_shim)
            np.savez_compressed(os.path.join(out_dir, name + ".npz"), **data)
            print(name, "loss", float(data["loss"]), "x", data["x"].shape,
                  "springs", data["springs"].shape)
    finally:
        os.chdir(cwd)


if __name__ == "__main__":
    main()
