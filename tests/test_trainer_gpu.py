"""The trainer drop-in on the GPU: a cfg3d config through load_config and
DiffPhyTrainer.simulate reproduces the reference's golden loss and the FP64
oracle's gradients; the torch autograd function returns the same gradients;
train() writes reference-layout pickles that load back; evaluate() runs the
scripted episode."""
import os

import numpy as np
import pytest

from helpers import load_golden, oracle_from_golden, rel_err
from test_trainer_cpu import golden_config

pytestmark = pytest.mark.gpu


def _trainer(g, precision=64, K=8):
    from cls_b200.trainer import DiffPhyTrainer, load_config
    tr = DiffPhyTrainer(load_config(golden_config(g), seed=3), precision=precision, checkpoint_every=K)
    tr.set_weights([(g["W1"], g["b1"]), (g["W2"], g["b2"])])
    return tr


@pytest.mark.parametrize("case", ["quad_ref", "x_all_losses"])
def test_simulate_matches_golden_loss_and_oracle_gradients(case):
    g = load_golden(case)
    steps = int(g["steps"])
    tr = _trainer(g)
    try:
        assert np.allclose(tr.initial_objects, g["x0"][0])
        tr.batch.set_state(g["x0"].reshape(-1, 3))
        loss = tr.simulate(steps, targets=(g["target_v"], g["target_h"], g["target_c"]))
        assert loss == pytest.approx(float(g["loss"]), rel=1e-9)
        o = oracle_from_golden(g)
        o.run(steps)
        (gW1, gb1), (gW2, gb2) = tr.grads()
        assert rel_err(gW1, o.gW[0]) < 1e-8 and rel_err(gW2, o.gW[1]) < 1e-8
        assert rel_err(gb1, o.gb[0]) < 1e-8 and rel_err(gb2, o.gb[1]) < 1e-8
    finally:
        tr.close()


def test_rollout_loss_autograd_matches_adjoint():
    import torch
    from cls_b200.trainer import rollout_loss
    g = load_golden("quad_ref")
    steps = int(g["steps"])
    tr = _trainer(g)
    try:
        params = [torch.tensor(a, dtype=torch.float64, requires_grad=True)
                  for a in (g["W1"], g["b1"], g["W2"], g["b2"])]
        targets = (g["target_v"], g["target_h"], g["target_c"])
        loss = rollout_loss(tr, steps, params, targets=targets)
        (2.0 * loss).backward()
        assert float(loss.detach()) == pytest.approx(float(g["loss"]), rel=1e-9)
        o = oracle_from_golden(g)
        o.run(steps)
        ref = [o.gW[0], o.gb[0], o.gW[1], o.gb[1]]
        for p, r in zip(params, ref):
            assert rel_err(p.grad.numpy() / 2.0, r) < 1e-8
    finally:
        tr.close()


def test_train_writes_reference_pickles_and_evaluates(tmp_path):
    import pickle
    from cls_b200.trainer import DiffPhyTrainer, load_config
    g = load_golden("quad_ref")
    cfg = load_config(golden_config(g), seed=1)
    tr = DiffPhyTrainer(cfg, precision=32, checkpoint_every=8, batch_size=4,
                        log_path=str(tmp_path / "metrics.jsonl"))
    try:
        losses = tr.train(3, save_dir=str(tmp_path))
        assert len(losses) == 3 and all(np.isfinite(losses))
        for f in ("best.pkl", "last.pkl", "iter0.pkl", "metrics.jsonl"):
            assert os.path.exists(tmp_path / f)
        with open(tmp_path / "last.pkl", "rb") as fh:
            lst = pickle.load(fh)
        H, N = int(g["n_hidden"]), len(g["objects"])
        assert [a.shape for a in lst] == [(H, cfg["nn"]["n_input_states"]), (len(g["springs"]), H), (H,),
                                          (len(g["springs"]),)]
        w = tr.weights()
        tr.set_weights([(np.zeros_like(W), np.zeros_like(b)) for W, b in w])
        tr.load_weights(str(tmp_path / "last.pkl"))
        for (W, b), (W2, b2) in zip(w, tr.weights()):
            assert rel_err(W2, W) < 1e-6 and rel_err(b2, b) < 1e-6
    finally:
        tr.close()
    ev = DiffPhyTrainer(cfg, precision=32, checkpoint_every=8, batch_size=2, evaluate=True)
    try:
        terms = ev.evaluate(str(tmp_path / "best.pkl"), steps=50)
        assert np.isfinite(terms["total"])
    finally:
        ev.close()


def test_evaluate_exports_obj_frames_of_the_rollout(tmp_path):
    """evaluate(mesh_dir=...) writes every 10th state of each env's scripted
    rollout as OBJ frames; the vertices are the rollout's own trajectory."""
    from cls_b200.trainer import DiffPhyTrainer, load_config
    g = load_golden("quad_ref")
    cfg = load_config(golden_config(g), seed=1)
    ev = DiffPhyTrainer(cfg, precision=64, checkpoint_every=8, batch_size=2, evaluate=True,
                        keep_trajectory=True)
    try:
        ev.set_weights([(g["W1"], g["b1"]), (g["W2"], g["b2"])])
        ev.evaluate(steps=45, mesh_dir=str(tmp_path / "video"))
        traj = ev.batch.trajectory()
        for k in range(2):
            files = sorted(os.listdir(tmp_path / "video" / str(k)))
            assert len(files) == len(traj[::10])
            xk = traj[:, ev.batch.env_slice(k)]
            lines = open(tmp_path / "video" / str(k) / files[3]).read().splitlines()
            v = np.array([[float(c) for c in ln.split()[1:]] for ln in lines if ln.startswith("v ")])
            np.testing.assert_allclose(v, xk[30], atol=5e-7)
            f = [ln for ln in lines if ln.startswith("f ")]
            assert len(f) == len(ev.faces)
    finally:
        ev.close()
