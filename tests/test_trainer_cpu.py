"""cfg3d loader (derived keys, robot build), scripted evaluation targets and
the reference weight-pickle layout, on the CPU."""
import math

import numpy as np
import pytest

from helpers import load_golden


def golden_config(g, **extra):
    """A cfg3d-schema config with the golden run's settings."""
    spr = g["springs"]
    cfg = {
        "train": {"name": "golden", "save_dir": "unused", "task": [str(s) for s in g["loss_names"]]},
        "validation": {"velocity": [0.0], "height": [0.0]},
        "robot": {"dim": 3, "robot_id": int(g["robot_id"]), "simulator": "mass_spring",
                  "design_file": "unused", "control_length": 1, "name": "golden", "id": int(g["robot_id"]),
                  "spring_stiffness": float(spr[:, 3].max()), "spring_actuation": float(spr[:, 4].max()),
                  "solver": "mass_spring"},
        "process": {"max_steps": int(g["T"]), "evaluate_max_steps": 60, "vis_interval": 256,
                    "output_vis_interval": 8, "run_period": int(g["run_period"]),
                    "jump_period": int(g["jump_period"]), "turn_period": int(g["turn_period"]),
                    "max_speed": float(g["max_speed"]), "max_height": float(g["max_height"]), "dt": 0.01},
        "simulator": {"mpm": {"n_grid": 32}, "ground_height": float(g["ground"]), "gravity": -9.8,
                      "drag_damping": float(g["drag"]), "dash_damping": 0.2, "p_vol": 1, "E": 40, "mu": 40,
                      "la": 40, "act_strength": 4, "bound": 3, "coeff": 5},
        "nn": {"n_sin_waves": int(g["n_sin"]), "n_hidden": int(g["n_hidden"]), "duplicate_v": int(g["dup_v"]),
               "duplicate_h": int(g["dup_h"]), "duplicate_c": int(g["dup_c"]), "batch_size": int(g["B"]),
               "max_reset_step": 4, "optimizer": "adam", "learning_rate": 3e-4, "adam_b1": 0.9,
               "adam_b2": 0.9},
    }
    cfg.update(extra)
    return cfg


@pytest.mark.parametrize("case", ["quad_ref", "x_all_losses"])
def test_load_config_derives_the_reference_keys(case):
    from cls_b200.trainer import load_config
    g = load_golden(case)
    cfg = load_config(golden_config(g), seed=5)
    assert np.array_equal(np.asarray(cfg["robot"]["objects"]), g["objects"])
    assert np.array_equal(np.asarray(cfg["robot"]["springs"]), g["springs"])
    pr, sim, nn = cfg["process"], cfg["simulator"], cfg["nn"]
    assert pr["dt"] == 0.004 and sim["gravity"] == -1.8 and sim["dashpot_damping"] == 0.1
    assert pr["dt"] == float(g["dt"]) and sim["gravity"] == float(g["gravity"])
    assert pr["spring_omega"] == pytest.approx(2 * math.pi / 0.004 / pr["run_period"])
    assert pr["spring_omega"] == pytest.approx(float(g["spring_omega"]))
    N = len(g["objects"])
    assert nn["n_input_states"] == nn["n_sin_waves"] + 6 * N + 2 * nn["duplicate_v"] + nn["duplicate_h"] \
        + nn["duplicate_c"]
    assert nn["n_input_states"] == g["input_state"].shape[-1]
    assert nn["adam_a"] == nn["learning_rate"] and cfg["train"]["random_seed"] == 5
    ov = load_config(golden_config(g), overrides={"simulator": {"friction": 0.5}, "process": {"dt": 0.002}})
    assert ov["simulator"]["friction"] == 0.5 and ov["process"]["dt"] == 0.002
    with pytest.raises(NotImplementedError):
        c = golden_config(g)
        c["robot"]["simulator"] = "mpm"
        load_config(c)


def test_script_targets_phases():
    from cls_b200.trainer import script_targets
    tv, th = script_targets(6100, 6000, 0.08)
    assert tuple(tv[0, [0, 2]]) == (-0.08, 0.0) and tuple(tv[1500, [0, 2]]) == (0.0, 0.08)
    assert tuple(tv[2500, [0, 2]]) == (0.08, 0.0) and tuple(tv[3999, [0, 2]]) == (0.0, -0.08)
    assert th[4500] == -1.0 and th[5999] == 1.0 and th[6000] == 0.0
    assert np.all(tv[4000:, :] == 0) and np.all(th[:4000] == 0)


def test_reference_pickle_layout_roundtrip():
    from cls_b200.trainer import from_reference_list, to_reference_list
    rng = np.random.default_rng(0)
    layers = [(rng.normal(size=(64, 838)), rng.normal(size=64)), (rng.normal(size=(272, 64)), rng.normal(size=272))]
    lst = to_reference_list(layers)
    assert [a.shape for a in lst] == [(64, 838), (272, 64), (64,), (272,)]
    back = from_reference_list(lst)
    for (W, b), (W2, b2) in zip(layers, back):
        assert np.array_equal(W, W2) and np.array_equal(b, b2)
    with pytest.raises(ValueError):
        to_reference_list(layers + layers)


def test_obj_frames_format(tmp_path):
    """write_obj_frames: every stride-th state, 6-decimal vertex lines, then
    1-based triangles (the evaluation visualiser's mesh files)."""
    from cls_b200.trainer import write_obj_frames
    rng = np.random.default_rng(0)
    x = rng.uniform(-1, 1, (25, 4, 3))
    faces = np.array([[0, 1, 2], [3, 0, 2]])
    paths = write_obj_frames(x, faces, str(tmp_path / "mesh"), stride=10)
    assert [p.rsplit("/", 1)[1] for p in paths] == ["000000.obj", "000001.obj", "000002.obj"]
    lines = open(paths[1]).read().splitlines()
    assert lines[:4] == ["v %.6f %.6f %.6f" % tuple(p) for p in x[10]]
    assert lines[4:] == ["f 1 2 3", "f 4 1 3"]


def test_load_config_keeps_the_builder_faces():
    from cls_b200.trainer import load_config
    g = load_golden("quad_ref")
    cfg = load_config(golden_config(g), seed=0)
    faces = np.asarray(cfg["robot"]["faces"])
    geo = np.load(__import__("os").path.join(__import__("helpers").GOLDEN, "robots.npz"))
    np.testing.assert_array_equal(faces, geo["faces_%d" % int(g["robot_id"])])


def test_malformed_configs_are_rejected_on_the_host(tmp_path):
    """A cfg3d file that is not JSON, lacks a required key, names an unknown
    robot or an unknown loss, or asks for the MPM simulator of the trainer,
    fails in load_config / the trainer's constructor with an exception, before
    any device work."""
    import json
    from cls_b200.trainer import load_config
    g = load_golden("quad_ref")
    bad = tmp_path / "bad.json"
    bad.write_text('{"robot": {"robot_id": 100,')
    with pytest.raises(json.JSONDecodeError):
        load_config(str(bad))
    cfg = golden_config(g)
    del cfg["nn"]["n_sin_waves"]
    with pytest.raises(KeyError):
        load_config(cfg)
    cfg = golden_config(g)
    cfg["robot"]["robot_id"] = 117
    with pytest.raises(ValueError, match="invalid robot id"):
        load_config(cfg)
    cfg = golden_config(g)
    cfg["robot"]["simulator"] = "mpm"
    with pytest.raises(NotImplementedError):
        load_config(cfg)
    from cls_b200.dropin import TaichiEnvCUDA
    cfg = load_config(golden_config(g), seed=0)
    cfg["train"]["task"] = ["velocity", "flying"]
    with pytest.raises(ValueError, match="unknown loss"):
        TaichiEnvCUDA(cfg, batch=object())
