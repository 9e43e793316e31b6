"""Host logic without a GPU: robot builders against the reference builder's
output, synthetic workload shapes, config schema handling."""
import json
import os

import numpy as np
import pytest

from helpers import GOLDEN


def _geo():
    g = np.load(os.path.join(GOLDEN, "robots.npz"))
    return {k: g[k] for k in g.files}


def skeleton_file(g, tmp_path):
    """The spider's node / link table (the reference's cfg3d/skeleton.json,
    kept in robots.npz by make_golden.py) written back as a JSON file."""
    path = os.path.join(str(tmp_path), "skeleton.json")
    nodes = {str(k): [float(c) for c in xyz] for k, xyz in zip(g["skeleton_node_keys"], g["skeleton_nodes"])}
    with open(path, "w") as f:
        json.dump({"nodes": nodes, "links": g["skeleton_links"].tolist()}, f)
    return path


@pytest.mark.parametrize("rid", [100, 101, 102, 104])
def test_cube_robots_match_reference_builder(rid):
    from cls_b200 import robot_design
    g = _geo()
    obj, spr, faces = robot_design.reference_robot(rid, float(g["stiffness_%d" % rid]),
                                                   float(g["actuation_%d" % rid]), faces=True)
    np.testing.assert_array_equal(obj, g["objects_%d" % rid])
    np.testing.assert_array_equal(spr, g["springs_%d" % rid])
    np.testing.assert_array_equal(faces, g["faces_%d" % rid])


def test_spider_matches_reference_builder(tmp_path):
    from cls_b200 import robot_design
    g = _geo()
    obj, spr, faces = robot_design.reference_robot(103, float(g["stiffness_103"]), float(g["actuation_103"]),
                                                   skeleton=skeleton_file(g, tmp_path), faces=True)
    np.testing.assert_array_equal(obj, g["objects_103"])
    np.testing.assert_array_equal(spr, g["springs_103"])
    np.testing.assert_array_equal(faces, g["faces_103"])


def test_reference_robot_counts():
    g = _geo()
    counts = {rid: (g["objects_%d" % rid].shape[0], g["springs_%d" % rid].shape[0],
                    int((g["springs_%d" % rid][:, 4] > 0).sum())) for rid in (100, 101, 102, 103, 104)}
    assert counts[100] == (48, 272, 48)
    assert counts[103][:2] == (39, 175)


def test_synthetic_lattices():
    from cls_b200 import robot_design
    # the configurations' robot sizes: quadruped ~90 vertices with 40
    # actuated springs, spider ~250 vertices / ~1400 springs / 96 actuators
    obj, spr = robot_design.quadruped_lattice()
    assert (obj.shape[0], spr.shape[0], int((spr[:, 4] > 0).sum())) == (93, 608, 40)
    obj, spr = robot_design.spider_lattice()
    assert (obj.shape[0], spr.shape[0], int((spr[:, 4] > 0).sum())) == (236, 1378, 96)
    obj, spr = robot_design.spider_lattice(refine=1)
    assert (obj.shape[0], spr.shape[0], int((spr[:, 4] > 0).sum())) == (136, 732, 96)
    for build in (robot_design.quadruped_lattice, robot_design.spider_lattice):
        obj, spr = build()
        a, b = spr[:, 0].astype(int), spr[:, 1].astype(int)
        np.testing.assert_allclose(spr[:, 2], np.linalg.norm(obj[a] - obj[b], axis=1), rtol=1e-12)
        assert abs(obj[:, 1].min() - 0.1) < 1e-12
    rng = np.random.default_rng(0)
    for n in (50, 300, 2000):
        obj, spr = robot_design.random_lattice(rng, n)
        assert n <= obj.shape[0] <= n + 4
        a, b = spr[:, 0].astype(int), spr[:, 1].astype(int)
        assert a.min() >= 0 and b.max() < obj.shape[0] and np.all(a != b)
        # rest length is the initial distance
        np.testing.assert_allclose(spr[:, 2], np.linalg.norm(obj[a] - obj[b], axis=1), rtol=1e-12)
        frac = (spr[:, 4] > 0).mean()
        assert abs(frac - 0.3) < 0.01
        # connected: every vertex reachable from vertex 0
        adj = [[] for _ in range(obj.shape[0])]
        for i, j in zip(a, b):
            adj[i].append(j)
            adj[j].append(i)
        seen, stack = {0}, [0]
        while stack:
            for j in adj[stack.pop()]:
                if j not in seen:
                    seen.add(j)
                    stack.append(j)
        assert len(seen) == obj.shape[0]


def test_uneven_workload_shape():
    from cls_b200 import workloads
    robots = workloads.uneven_robots(64, seed=0)
    n = np.array([r.n_vertices for r in robots])
    s = np.array([r.n_springs for r in robots])
    assert n.min() >= 50 and n.max() <= 2004
    assert s.min() >= 200
    assert all(r.n_outputs == int((r.springs[:, 4] > 0).sum()) for r in robots)
