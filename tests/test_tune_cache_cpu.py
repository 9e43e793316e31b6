"""Host logic of MassSpringBatch.autotune: the workload signature and the JSON
cache of chosen launch shapes.  A fake library stands in for the C calls that
need a GPU (cls_autotune, cls_get/set_launch_shape, the controller path)."""
import json

import numpy as np

from helpers import load_golden


class FakeLib:
    TABLE = [(1, 128, 1, 0, 3.0), (1, 512, 1, 0, 1.5), (1, 256, 1, 1, 2.0), (2, 512, 1, 0, 1.2)]

    def __init__(self):
        self.shape = [256, 2, 0]
        self.path = 0
        self.tuned = 0
        self.set_shapes = []

    def cls_autotune(self, h, steps, repeats, table, cap, n):
        self.tuned += 1
        for i, e in enumerate(self.TABLE):
            t = table[i]
            t.controller_path, t.threads_per_block, t.ctas_per_sm, t.weights_shared, t.ms = e
        n[0] = len(self.TABLE)
        self.shape, self.path = [512, 1, 0], 2   # the fastest entry: the batched path
        return 0

    def cls_get_launch_shape(self, h, t, c, w):
        t[0], c[0], w[0] = self.shape
        return 0

    def cls_set_launch_shape(self, h, t, c, w):
        self.set_shapes.append((t, c, w))
        self.shape = [t, c, max(w, 0)]
        return 0

    def cls_set_controller_path(self, h, p):
        self.path = p
        return 0

    def cls_controller_batched(self, h, on):
        on[0] = 1 if self.path == 2 else 0
        return 0


def _fake_batch(n_envs, K=10):
    import cls_b200
    from cls_b200.batch import MassSpringBatch
    g = load_golden("quad_ref")
    b = object.__new__(MassSpringBatch)
    b.lib = FakeLib()
    b.h = None
    b.robots = [cls_b200.Robot(g["objects"], g["springs"], robot_id=int(g["robot_id"]), hidden=[64])]
    b.env_robot = np.zeros(n_envs, dtype=np.int32)
    b.params = cls_b200.default_params(checkpoint_every=K, precision=32)
    b.T = 200
    return b


def test_autotune_table_and_cache(tmp_path):
    cache = str(tmp_path / "shapes.json")
    b = _fake_batch(64)
    res = b.autotune(cache=cache)
    assert b.lib.tuned == 1 and not res["cached"]
    assert [r["threads_per_block"] for r in res["table"]] == [128, 512, 256, 512]
    assert [r["controller_path"] for r in res["table"]] == ["per_env"] * 3 + ["batched"]
    assert res["table"][2]["weights_shared"] == 1 and abs(res["table"][3]["ms"] - 1.2) < 1e-6  # float32 field
    assert (res["threads_per_block"], res["ctas_per_sm"], res["controller_path"]) == (512, 1, "batched")
    with open(cache) as f:
        data = json.load(f)
    assert len(data) == 1 and list(data.values())[0]["controller_path"] == "batched"

    # the same workload in another handle: applied from the cache, not timed
    b2 = _fake_batch(64)
    hit = b2.autotune(cache=cache)
    assert hit["cached"] and b2.lib.tuned == 0
    assert b2.lib.set_shapes == [(512, 1, 0)] and b2.lib.path == 2

    # another env count or checkpoint interval is another workload
    for other in (_fake_batch(32), _fake_batch(64, K=20)):
        assert not other.autotune(cache=cache)["cached"] and other.lib.tuned == 1
    with open(cache) as f:
        assert len(json.load(f)) == 3


def test_autotune_without_cache_always_times():
    b = _fake_batch(16)
    b.autotune()
    b.autotune()
    assert b.lib.tuned == 2
