"""Robot geometry: the reference's 3D cube-lattice robots and the seeded
synthetic lattices used for the batched configurations.

Cube lattice (restated from the reference's RobotDesignMassSpring3D,
multitask/robot_design.py:319-591): lattice point (i, j, k) sits at
``(0.05 i + 0.1, 0.05 j + 0.1, 0.05 k + 0.1)``; every cube contributes its 12
edges, 12 face diagonals and 4 body diagonals as springs (rest length = initial
distance, duplicates of an existing vertex pair skipped).  Points and springs
are numbered in creation order, which the tests compare with the reference
builder's output.  Rows are ``[a, b, rest_length, stiffness, actuation]``.
"""
import json
import math

import numpy as np

SPACING = 0.05
ORIGIN = 0.1

# The 28 springs of one cube in the reference's insertion order, as pairs of
# corner names; corners a..h are (i,j,k), (i,j+1,k), (i+1,j,k), (i+1,j+1,k),
# (i,j,k+1), (i,j+1,k+1), (i+1,j,k+1), (i+1,j+1,k+1).  The flag says whether the
# spring takes the cube's actuation coefficient ("square" cubes,
# robot_design.py:372-417) -- "lying" cubes (:507-552) flip the pattern.
_SQUARE = [("a", "b", 1), ("c", "d", 1), ("e", "f", 1), ("g", "h", 1),
           ("b", "d", 0), ("a", "c", 0), ("f", "h", 0), ("e", "g", 0),
           ("b", "f", 0), ("d", "h", 0), ("a", "e", 0), ("c", "g", 0),
           ("b", "g", 0), ("d", "e", 0), ("f", "c", 0), ("h", "a", 0),
           ("e", "c", 0), ("a", "g", 0), ("h", "b", 0), ("d", "f", 0),
           ("e", "b", 1), ("a", "f", 1), ("h", "c", 1), ("d", "g", 1),
           ("f", "g", 1), ("e", "h", 1), ("a", "d", 1), ("c", "b", 1)]
_LYING = [("a", "b", 0), ("c", "d", 0), ("e", "f", 0), ("g", "h", 0),
          ("b", "d", 0), ("a", "c", 0), ("f", "h", 0), ("e", "g", 0),
          ("b", "f", 1), ("d", "h", 1), ("a", "e", 1), ("c", "g", 1),
          ("b", "g", 1), ("d", "e", 1), ("f", "c", 1), ("h", "a", 1),
          ("e", "c", 1), ("a", "g", 1), ("h", "b", 1), ("d", "f", 1),
          ("e", "b", 1), ("a", "f", 1), ("h", "c", 1), ("d", "g", 1),
          ("f", "g", 0), ("e", "h", 0), ("a", "d", 0), ("c", "b", 0)]
_CORNER = {"a": (0, 0, 0), "b": (0, 1, 0), "c": (1, 0, 0), "d": (1, 1, 0),
           "e": (0, 0, 1), "f": (0, 1, 1), "g": (1, 0, 1), "h": (1, 1, 1)}
_CORNER_ORDER = "abcdefgh"


class CubeLattice:
    """Incremental cube-lattice builder with the reference's numbering rules."""

    def __init__(self, stiffness, actuation, spacing=SPACING, origin=ORIGIN, spacing_y=None):
        self.stiffness = float(stiffness)
        self.actuation = float(actuation)
        self.spacing = spacing
        self.spacing_y = spacing if spacing_y is None else spacing_y   # boxes of the refined lattices
        self.origin = origin
        self.objects = []
        self.springs = []
        self.faces = []
        self._point_id = {}
        self._pairs = set()

    def point(self, i, j, k):
        key = (i, j, k)
        if key not in self._point_id:
            self._point_id[key] = len(self.objects)
            self.objects.append((i * self.spacing + self.origin, j * self.spacing_y + self.origin,
                                 k * self.spacing + self.origin))
        return self._point_id[key]

    def spring(self, a, b, actuation, stiffness=None):
        if (a, b) in self._pairs or (b, a) in self._pairs:
            return
        self._pairs.add((a, b))
        pa, pb = self.objects[a], self.objects[b]
        # rest length = initial distance, evaluated as the reference does
        # (power 0.5 of the squared sum, robot_design.py:346-348)
        length = ((pa[0] - pb[0]) ** 2 + (pa[1] - pb[1]) ** 2 + (pa[2] - pb[2]) ** 2) ** 0.5
        self.springs.append([a, b, length, self.stiffness if stiffness is None else stiffness,
                             actuation])

    def cube(self, i, j, k, actuation=0.0, lying=False):
        ids = {c: self.point(i + _CORNER[c][0], j + _CORNER[c][1], k + _CORNER[c][2])
               for c in _CORNER_ORDER}
        for p, q, act in (_LYING if lying else _SQUARE):
            self.spring(ids[p], ids[q], actuation if act else 0.0)
        a, b, c, d, e, f, g, h = (ids[x] for x in _CORNER_ORDER)
        for quad in ((a, b, d, c), (b, f, h, d), (f, e, g, h), (e, a, c, g), (h, g, c, d),
                     (b, a, e, f)):
            self.faces.append((quad[0], quad[1], quad[2]))
            self.faces.append((quad[3], quad[0], quad[2]))

    def faces_array(self):
        return np.asarray(self.faces, dtype=np.int64).reshape(-1, 3)

    def arrays(self):
        return (np.asarray(self.objects, dtype=np.float64).reshape(-1, 3),
                np.asarray(self.springs, dtype=np.float64).reshape(-1, 5))


# ------------------------------------------------------- reference robots
def _robot_a(L, act):   # quadruped, id 100 (robot_design.py:429-443)
    for ijk in ((0, 0, 0), (2, 0, 2), (0, 0, 2), (2, 0, 0)):
        L.cube(*ijk, actuation=act)
    for i in range(3):
        for k in range(3):
            L.cube(i, 1, k, actuation=0)


def _robot_b(L, act):   # id 101 (:445-456)
    for ijk in ((0, 0, 1), (1, 0, 0), (1, 0, 2), (2, 0, 1)):
        L.cube(*ijk, actuation=act)
    for ijk in ((0, 1, 1), (1, 1, 0), (1, 1, 2), (2, 1, 1), (1, 1, 1), (1, 2, 1)):
        L.cube(*ijk, actuation=0)


def _robot_c(L, act):   # id 102 (:458-468)
    for ijk in ((0, 0, 0), (2, 0, 0), (1, 0, 2)):
        L.cube(*ijk, actuation=act)
    for ijk in ((0, 1, 0), (2, 1, 0), (1, 1, 2), (0, 1, 1), (1, 1, 1), (2, 1, 1)):
        L.cube(*ijk, actuation=0)


def _robot_e(L, act):   # snake, id 104 (:564-570)
    for k in range(6):
        L.cube(0, 0, k, actuation=act, lying=True)


# skeleton motors and extra links of the spider (robot_design.py:480-498)
_SPIDER_MOTORS = [(9, 21), (36, 24), (29, 26), (14, 11), (14, 26), (10, 9), (29, 11), (25, 24),
                  (25, 26), (36, 9), (21, 24), (10, 11)]
_SPIDER_EXTRA = [(14, 29), (29, 36), (36, 21), (21, 14), (11, 5), (26, 5), (24, 35), (9, 20),
                 (26, 35), (11, 20), (9, 8), (24, 8), (11, 31), (26, 16), (24, 23), (9, 38)]


def _robot_d(L, act, skeleton):   # spider, id 103 (:470-505)
    with open(skeleton) as f:
        data = json.load(f)
    for v in data["nodes"]:
        p = data["nodes"][v]
        L.objects.append((p[0] * 0.05, p[1] * 0.05 + 0.212, p[2] * 0.05 * 0.75))
    motors = set(_SPIDER_MOTORS)
    motor = lambda a, b: (a, b) in motors or (b, a) in motors  # noqa: E731
    for a, b in data["links"]:
        L.spring(a, b, act if motor(a, b) else 0.0)
    # the reference walks its motor set (a set display of constant tuples)
    # first; a set display of the same tuples iterates in the same
    # hash-determined order
    motor_set = {(9, 21), (36, 24), (29, 26), (14, 11), (14, 26), (10, 9), (29, 11), (25, 24),
                 (25, 26), (36, 9), (21, 24), (10, 11)}
    for a, b in list(motor_set) + _SPIDER_EXTRA:
        L.spring(a, b, act if motor(a, b) else 0.0)
    # mesh faces: every triangle of skeleton links, vertices ascending
    linked = set()
    for a, b in data["links"]:
        linked.add((a, b))
        linked.add((b, a))
    n = len(L.objects)
    nbr = [sorted(b for b in range(n) if (a, b) in linked) for a in range(n)]
    for a in range(n):
        for b in nbr[a]:
            if b <= a:
                continue
            for c in nbr[b]:
                if c > b and (a, c) in linked:
                    L.faces.append((a, b, c))


def reference_robot(robot_id, spring_stiffness, spring_actuation, skeleton=None, faces=False):
    """objects, springs of one of the reference's five 3D robots (ids 100-104)
    and, with ``faces=True``, also its triangle list [(a, b, c)] for mesh
    export (two triangles per cube face, robot_design.py:419-427; the spider's
    skeleton triangles, :500-504).  The spider (103) reads its node/link table
    from ``skeleton`` (the reference's cfg3d/skeleton.json)."""
    L = CubeLattice(spring_stiffness, spring_actuation)
    if robot_id == 100:
        _robot_a(L, spring_actuation)
    elif robot_id == 101:
        _robot_b(L, spring_actuation)
    elif robot_id == 102:
        _robot_c(L, spring_actuation)
    elif robot_id == 103:
        if skeleton is None:
            raise ValueError("robot 103 needs the skeleton.json path")
        _robot_d(L, spring_actuation, skeleton)
    elif robot_id == 104:
        _robot_e(L, spring_actuation)
    else:
        raise ValueError("invalid robot id %r" % (robot_id,))
    if faces:
        return L.arrays() + (np.asarray(L.faces, dtype=np.int64).reshape(-1, 3),)
    return L.arrays()


# ------------------------------------------------------ synthetic robots
def quadruped_lattice(stiffness=3e4, actuation=0.25, n_actuated=40, refine=2):
    """Torso of 4 x 2 x 1 cubes on four 1 x 1 x 2 legs at its corners.
    ``refine`` splits every cube into that many boxes along the height
    (``refine=2``: 93 vertices, 608 springs, the robot size of the plain
    quadruped configuration; ``refine=1``: 54 vertices, 323 springs).  The
    reference's per-cube actuation pattern marks the leg springs; the first
    ``n_actuated`` of them (in creation order) keep their coefficient."""
    r = int(refine)
    L = CubeLattice(stiffness, actuation, spacing_y=SPACING / r)
    for (i, k) in ((0, 0), (3, 0), (0, 1), (3, 1)):
        for j in range(2 * r):
            L.cube(i, j, k, actuation=actuation)
    for i in range(4):
        for k in range(2):
            for j in range(2 * r, 3 * r):
                L.cube(i, j, k, actuation=0.0)
    objects, springs = L.arrays()
    act = np.nonzero(springs[:, 4] > 0)[0]
    springs[act[n_actuated:], 4] = 0.0
    return objects, springs


def spider_lattice(stiffness=3e4, actuation=0.2, refine=2):
    """A 3 x 3 x 1 torso (cube layer 3) with eight 1 x 1 x 3 legs: vertical
    columns of three cubes beside it, one cell apart from each other, whose
    top cubes sit in the torso layer.  ``refine`` splits every cube into that
    many boxes along the height (``refine=2``: 236 vertices, 1378 springs,
    the robot size of the large-batch spider configuration; ``refine=1``:
    136 vertices, 732 springs).  Four vertical edges of one box per leg cube
    (the lowest box of each) are actuated: 8 legs x 3 cubes x 4 = 96
    actuators."""
    r = int(refine)
    L = CubeLattice(stiffness, 0.0, spacing_y=SPACING / r)
    legs = [(-1, -1), (-1, 1), (-1, 3), (1, -1), (1, 3), (3, -1), (3, 1), (3, 3)]
    vertical = {("a", "b"), ("c", "d"), ("e", "f"), ("g", "h")}
    for (i, k) in legs:
        for j in range(r, 4 * r):
            ids = {c: L.point(i + _CORNER[c][0], j + _CORNER[c][1], k + _CORNER[c][2])
                   for c in _CORNER_ORDER}
            act = actuation if (j - r) % r == 0 else 0.0
            for p, q, _ in _SQUARE:
                L.spring(ids[p], ids[q], act if (p, q) in vertical else 0.0)
    for i in range(3):
        for k in range(3):
            for j in range(3 * r, 4 * r):
                L.cube(i, j, k, actuation=0.0)
    objects, springs = L.arrays()
    objects[:, 1] -= SPACING  # legs stand on the lattice origin height
    return objects, springs


def random_lattice(rng, n_vertices, stiffness=3e4, actuation=0.2, actuated_fraction=0.3):
    """A random connected lattice: a branching chain of cubes grown from one
    seed cube, each new cube attached to the structure by a single face (60 %
    of the time extending the newest cube, else a random one), until at least
    ``n_vertices`` points exist.  Each cube then adds 4 points and 22 springs,
    so springs ~ 5.5 x vertices.  A random ``actuated_fraction`` of the
    springs is actuated."""
    L = CubeLattice(stiffness, 0.0)
    cubes = [(0, 0, 0)]
    occupied = {(0, 0, 0)}
    L.cube(0, 0, 0)
    nbr = ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1))
    misses = 0
    while len(L.objects) < n_vertices:
        base = cubes[-1] if rng.random() < 0.6 else cubes[int(rng.integers(len(cubes)))]
        d = nbr[int(rng.integers(6))]
        c = (base[0] + d[0], base[1] + d[1], base[2] + d[2])
        if c in occupied or c[1] < 0 or c[1] > 3:
            continue
        touching = sum((c[0] + e[0], c[1] + e[1], c[2] + e[2]) in occupied for e in nbr)
        if touching > 1 and misses < 1000:
            misses += 1
            continue
        misses = 0
        occupied.add(c)
        cubes.append(c)
        L.cube(*c)
    objects, springs = L.arrays()
    m = springs.shape[0]
    act = rng.choice(m, size=max(1, int(round(actuated_fraction * m))), replace=False)
    springs[act, 4] = actuation
    # shift so that the lowest point rests at the lattice origin height
    objects[:, 0] -= objects[:, 0].min() - ORIGIN
    objects[:, 2] -= objects[:, 2].min() - ORIGIN
    return objects, springs
