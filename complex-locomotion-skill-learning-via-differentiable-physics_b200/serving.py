"""Request loop: continuous batching of rollout requests on resident env slots.

The reference has no serving path; it trains one batch at a time
(multitask/diffphy_trainer.py:219-256).  Here a ``Server`` keeps a pool of
env slots on the GPU and folds rollout requests into the running batch:

* a request names a registered robot type, an episode length (``steps``), a
  target seed and whether it wants weight gradients (forward + adjoint) or
  the forward rollout only (controller evaluation);
* it is admitted when a slot of its type is free and its HBM footprint fits
  the remaining budget; admission restarts that slot alone
  (``cls_serve_reset_env``), so the other slots keep running;
* every tick advances each active slot through its own window of at most
  ``checkpoint_every`` substeps in ONE launch per pool (``cls_serve_forward``),
  and each slot in its reverse pass through one checkpointed segment
  (``cls_serve_backward``); requests that arrive meanwhile join at the next
  tick;
* a finished request returns its losses (``cls_serve_loss``), final state and,
  for gradient queries, the weight gradients of its slot's controller.

Each slot owns a controller (a robot entry of the batch), so a slot's weight
gradients are its request's alone, and a request's result does not depend on
what else is in the batch.  Each robot type is a pool (one batch on its own
CUDA stream) that ticks at its own pace, so a small robot's requests are not
held to a large robot's substep time, and the pools' work overlaps on the
device.

MPM rollouts (``MpmType`` kinds: a particle body driven by seeded muscle
actuations towards a centre target) are served by pools of their own: each
slot is a one-env MLS-MPM handle (``cls_mpm_*``) on its own CUDA stream, and a
request's whole rollout (forward, and the checkpointed reverse pass for
gradient queries) is enqueued when it is admitted, so the MPM slots' work
overlaps with each other and with the mass-spring pools' ticks; the MPM
solver has no per-env windows, so its requests are not folded into shared
launches.

The scheduling is separate from the GPU backend (``SlotBackend``): the tests
drive the scheduler with a fake backend on the CPU.
"""
import math
import time
import zlib
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence

import numpy as np


@dataclass
class RobotType:
    """A registered robot type: geometry + controller shape (``batch.Robot``)
    and its controller weights [(W, b) per layer] (None: seeded init)."""
    robot: object
    weights: Optional[list] = None


@dataclass
class Request:
    kind: str                 # robot type name
    steps: int                # episode steps (cls_forward's `steps`, >= 2)
    grad: bool = False        # forward + adjoint (weight gradients) or forward only
    seed: int = 0             # seeds the targets (target velocity / height)
    arrival: float = 0.0      # seconds, on the server's clock
    x0: Optional[np.ndarray] = None   # initial state [n_v][3] (None: the robot's objects)
    rid: int = -1


@dataclass
class Result:
    rid: int
    kind: str
    steps: int
    grad: bool
    loss: float
    loss_terms: Dict[str, float]
    final_x: np.ndarray
    grads: Optional[list]
    arrival: float
    admitted: float
    done: float

    @property
    def latency(self):
        return self.done - self.arrival


LOSS_SLOTS = ("total", "velocity", "height", "pose", "rotation", "weight", "actuation", "crawl")


def request_targets(seed, T, steps, turn_period, lo=-0.1, hi=0.1):
    """Targets of one request, drawn from its seed: target velocity (vx, 0, vz)
    and height ~ U(lo, hi), one draw per turn period (held for the period)."""
    rng = np.random.default_rng(seed)
    n_blocks = T // turn_period + 1
    d = rng.uniform(lo, hi, size=(n_blocks, 3))
    idx = np.arange(T) // turn_period
    tv = np.zeros((T, 3))
    tv[:, 0] = d[idx, 0]
    tv[:, 2] = d[idx, 1]
    return tv, d[idx, 2].copy()


def footprint_bytes(robot, steps, grad, K, dtype_bytes=4):
    """HBM bytes a request keeps resident while it is served: state and
    checkpoints, its trajectory and observables, targets, controller
    weights (x3 with gradient and optimiser-sized buffers) and, for
    gradient queries, the per-segment records of its reverse pass."""
    n = robot.n_vertices
    widths = [3 * n + 11] + list(robot.hidden) + [robot.n_outputs or robot.n_springs]
    params = sum(widths[i] * widths[i + 1] + widths[i + 1] for i in range(len(widths) - 1))
    ckpt = 2 * 16 * n * (steps // K + 2)
    traj = 16 * n * steps + 32 * steps + 24 * steps
    w = params * dtype_bytes * (3 if grad else 1)
    rec = K * (48 * n + 8 * sum(widths[1:]) + 4 * widths[0]) if grad else 0
    return int(ckpt + traj + w + rec)


@dataclass
class MpmType:
    """A registered MPM body type: particle positions [P][dim], muscle id
    per particle (-1 passive), fibre directions, and MPMBatch keyword
    arguments of the solver (material, n_grid, dt, mu, la, ...)."""
    positions: np.ndarray
    muscle: np.ndarray
    fibre: Optional[np.ndarray] = None
    n_muscles: int = 16
    solver: dict = field(default_factory=dict)
    target_offset: Sequence[float] = (0.05, 0.0, 0.0)


def mpm_request_inputs(seed, T, steps, n_muscles, dt, dim=3):
    """Actuation [T][n_muscles] of an MPM request: sinusoids of 2-6 Hz with
    random phases drawn from its seed (the MPM benchmark's muscle drive);
    zero after the request's horizon."""
    rng = np.random.default_rng(seed)
    freq = rng.uniform(2.0, 6.0, size=n_muscles)
    phase = rng.uniform(0, 2 * np.pi, size=n_muscles)
    t = np.arange(T)[:, None] * dt
    act = np.sin(2 * np.pi * freq[None, :] * t + phase[None, :])
    act[steps:] = 0.0
    return act


def mpm_footprint_bytes(mt, T, K, dtype_bytes=4):
    """HBM bytes of one MPM slot: particle checkpoints (x, v, C, F) every K
    steps over T, one segment's records, the actuation and centre tracks, and
    the grid (n_grid^dim nodes of 16 bytes, twice for the adjoint)."""
    P, D = mt.positions.shape
    n_grid = int(mt.solver.get("n_grid", 64))
    per_p = (2 * D + 2 * D * D) * dtype_bytes
    return int(P * per_p * (T // K + 2) + P * per_p * K + 2 * 16 * n_grid ** D
               + T * (mt.n_muscles + 2 * D) * dtype_bytes)


class MpmSlotBackend:
    """One-env MPM handles (one per slot) of one MPM type, each on its own
    CUDA stream (torch.cuda.Stream, or the default stream when streams is
    False)."""

    def __init__(self, mt: MpmType, n_slots, T, K, streams=True):
        from .mpm import MPMBatch
        self.mt = mt
        self.T, self.K = int(T), int(K)
        dim = mt.positions.shape[1]
        self.dim = dim
        self.batches, self.streams, self.events = [], [], []
        for _ in range(n_slots):
            b = MPMBatch(mt.positions, mt.muscle, 1, dim=dim, fibre=mt.fibre, n_muscles=mt.n_muscles,
                         max_steps=self.T, checkpoint_every=self.K, **mt.solver)
            st = None
            if streams:
                import torch
                st = torch.cuda.Stream()
                b.set_stream(st.cuda_stream)
            self.batches.append(b)
            self.streams.append(st)
            self.events.append(None)
        self.c0 = mt.positions.mean(axis=0)
        self.dt = float(self.batches[0].params.dt)

    def start(self, slot, req):
        """Enqueues the request's rollout (forward; reverse for gradient
        queries) on the slot's stream."""
        b = self.batches[slot]
        D = self.dim
        x0 = self.mt.positions if req.x0 is None else req.x0
        b.set_state(np.asarray(x0, np.float64)[None])
        b.set_actuation(mpm_request_inputs(req.seed, self.T, req.steps, self.mt.n_muscles, self.dt)[:, None, :])
        w = np.zeros(self.T + 1)
        w[req.steps] = 1.0
        target = np.broadcast_to(self.c0 + np.asarray(self.mt.target_offset[:D]), (self.T + 1, 1, D)).copy()
        b.set_loss(w, target)
        b.forward(req.steps)
        if req.grad:
            b.backward()
        if self.streams[slot] is not None:
            import torch
            ev = torch.cuda.Event()
            ev.record(self.streams[slot])
            self.events[slot] = ev

    def done(self, slot):
        ev = self.events[slot]
        return ev is None or ev.query()

    def result(self, slot, req):
        """(loss, final positions [P][dim], gradients or None) of the slot's
        finished request; gradients: d loss / d actuation [steps][muscles]
        and d loss / d x0."""
        b = self.batches[slot]
        loss = b.loss()
        x = b.final_state()[0][0]
        grads = None
        if req.grad:
            g = b.grads()
            grads = {"act": g["act"][:req.steps, 0], "x0": g["x0"][0]}
        self.events[slot] = None
        return loss, x, grads

    def close(self):
        for b in self.batches:
            b.close()


class MpmPool:
    """The slots of one MPM type.  A slot runs one request's whole rollout;
    admitted requests start at once, finished ones are collected as their
    streams complete."""

    def __init__(self, kind, n_slots, backend):
        self.kind = kind
        self.slots = [_Slot(kind) for _ in range(n_slots)]
        self.backend = backend
        self.plan = None              # not None while a slot is running

    def free_slot(self, kind):
        if kind != self.kind:
            return -1
        for i, s in enumerate(self.slots):
            if s.phase == "free":
                return i
        return -1

    def busy(self):
        return any(s.phase != "free" for s in self.slots)

    def launch(self):
        started = False
        for i, s in enumerate(self.slots):
            if s.phase == "fwd":
                self.backend.start(i, s.req)
                s.phase = "run"
                started = True
        if self.busy():
            self.plan = True
        return started

    def ready(self):
        return any(s.phase == "run" and self.backend.done(i) for i, s in enumerate(self.slots))

    def complete(self, server):
        """Collects the finished slots; when none has finished yet, waits for
        the first running one (so a synchronous tick always progresses)."""
        running = [i for i, s in enumerate(self.slots) if s.phase == "run"]
        fin = [i for i in running if self.backend.done(i)]
        if not fin and running:
            fin = running[:1]
        out = []
        for i in fin:
            s = self.slots[i]
            loss, x, grads = self.backend.result(i, s.req)
            server.substeps_done += int(s.req.steps)
            s.loss, s.fx = loss, x
            s.terms = {"total": loss}
            out.append(server._finish(self, i, grads))
        self.plan = True if self.busy() else None
        return out


class SlotBackend:
    """GPU backend of one pool: a ``MassSpringBatch`` whose envs are the
    slots, each with a robot entry (controller) of its own."""

    def __init__(self, slot_types: Sequence[str], types: Dict[str, RobotType], params, stream=None,
                 weights_seed=0):
        from .batch import MassSpringBatch
        self.slot_types = list(slot_types)
        robots = [types[k].robot for k in self.slot_types]
        self.batch = MassSpringBatch(robots, list(range(len(robots))), params)
        self.stream = stream          # a torch.cuda.Stream (or None: default stream)
        if stream is not None:
            self.batch.set_stream(stream.cuda_stream)
        self.T = self.batch.T
        self.K = int(params.checkpoint_every)
        self.turn_period = int(params.turn_period)
        self.loaded = [None] * len(robots)   # type whose weights a slot holds
        for e, k in enumerate(self.slot_types):
            if types[k].weights is None:
                types[k].weights = self._type_weights(e, k, weights_seed)
            self.load_weights(e, k, types[k].weights)

    def _type_weights(self, slot, kind, seed):
        """Weights of a type without given ones: U(-1, 1) sqrt(6 / fan_in), zero
        bias (multitask/nn.py:59-67), drawn from (seed, type name) so that every
        slot and every server holds the same controller for the type."""
        rng = np.random.default_rng([seed, zlib.crc32(kind.encode())])
        out = []
        for l in range(self.batch.n_layers(slot)):
            rows, cols = self.batch.layer_shape(slot, l)
            out.append(((rng.random((rows, cols)) * 2 - 1) * math.sqrt(6.0 / cols), np.zeros(rows)))
        return out

    def load_weights(self, slot, kind, weights):
        if weights is not None:
            for l, (W, b) in enumerate(weights):
                self.batch.set_weights(slot, l, W, b)
        self.loaded[slot] = kind

    def reset(self, slot, req: Request, robot):
        x0 = robot.objects if req.x0 is None else req.x0
        tv, th = request_targets(req.seed, self.T, req.steps, self.turn_period)
        self.batch.serve_reset_env(slot, x0, None, tv, th)

    def forward(self, windows, steps):
        self.batch.serve_forward(windows, steps)

    def backward(self, windows, steps):
        self.batch.serve_backward(windows, steps)

    def loss(self, steps):
        return self.batch.serve_loss(steps)

    def final_x(self, slot):
        return self.batch.serve_env_state(slot)[0]

    def grads(self, slot):
        return [self.batch.get_grads(slot, l) for l in range(self.batch.n_layers(slot))]

    def sync(self):
        self.batch.synchronize()

    def query(self):
        """True when the pool's stream has finished its work."""
        return self.stream.query() if self.stream is not None else True

    def close(self):
        self.batch.close()


class _Slot:
    __slots__ = ("kind", "req", "phase", "pos", "seg", "loss", "terms", "fx", "admitted", "bytes")

    def __init__(self, kind):
        self.kind = kind
        self.req = None
        self.phase = "free"     # free | fwd | rev
        self.pos = 0            # forward: next step to run
        self.seg = 0            # reverse: next segment to run
        self.loss = None
        self.terms = None
        self.fx = None
        self.admitted = 0.0
        self.bytes = 0


class Pool:
    """The slots of one robot type, served by one backend (one batch on its
    own stream).  A pool advances by ticks: launch() issues one tick's
    windows, complete() collects its effects once the stream is done."""

    def __init__(self, slot_types, backend, K, T, rounds):
        self.slots = [_Slot(k) for k in slot_types]
        self.backend = backend
        self.K = K
        self.T = T
        self.rounds = rounds
        self.plan = None          # the tick in flight

    def free_slot(self, kind):
        for i, s in enumerate(self.slots):
            if s.phase == "free" and s.kind == kind:
                return i
        return -1

    def busy(self):
        return self.plan is not None or any(s.phase != "free" for s in self.slots)

    def steps(self):
        st = np.full(len(self.slots), 2, dtype=np.int32)
        for i, s in enumerate(self.slots):
            if s.phase != "free":
                st[i] = s.req.steps
        return st

    def forward_windows(self, span):
        """Forward window table of this tick ({t_begin, t_end, checkpoint, 0}
        per slot): `span` substeps from each forward-phase slot's position."""
        fw = np.zeros((len(self.slots), 4), dtype=np.int32)
        any_f = False
        for i, s in enumerate(self.slots):
            if s.phase == "fwd":
                t0, t_last = s.pos, s.req.steps - 1   # the first pass runs steps [0, steps - 1)
                fw[i] = (t0, min(t0 + span, t_last), t0 // self.K, 0)
                any_f = True
        return fw if any_f else None

    def reverse_windows(self, r):
        """Reverse window table of round r of this tick: segment seg - r of
        each reverse-phase slot ({t_begin, t_end, segment, first})."""
        K = self.K
        bw = np.zeros((len(self.slots), 4), dtype=np.int32)
        any_b = False
        for i, s in enumerate(self.slots):
            if s.phase == "rev" and s.seg - r >= 0:
                t_last = s.req.steps - 1
                n_seg = (t_last + K - 1) // K
                seg = s.seg - r
                bw[i] = (seg * K, min(seg * K + K, t_last), seg, 1 if seg == n_seg - 1 else 0)
                any_b = True
        return bw if any_b else None

    def launch(self):
        """Issue one tick (forward windows of rounds * K substeps, `rounds`
        reverse segments); False when no slot is active."""
        steps = self.steps()
        fw = self.forward_windows(self.rounds * self.K)
        if fw is not None:
            self.backend.forward(fw, steps)
        any_b = False
        for r in range(self.rounds):
            bw = self.reverse_windows(r)
            if bw is None:
                break
            self.backend.backward(bw, steps)
            any_b = True
        if fw is None and not any_b:
            return False
        self.plan = (fw, steps)
        return True

    def ready(self):
        return self.plan is not None and self.backend.query()

    def complete(self, server):
        """Effects of the tick in flight: positions, finished first passes
        (losses), finished requests.  Returns the finished requests."""
        fw, steps = self.plan
        self.plan = None
        self.backend.sync()
        done, fwd_finished = [], []
        for i, s in enumerate(self.slots):
            if s.phase == "fwd":
                server.substeps_done += int(fw[i, 1] - fw[i, 0])
                s.pos = int(fw[i, 1])
                if s.pos >= s.req.steps - 1:
                    fwd_finished.append(i)
            elif s.phase == "rev":
                s.seg -= self.rounds
        if fwd_finished:
            lsteps = np.zeros_like(steps)
            lsteps[fwd_finished] = steps[fwd_finished]
            env = self.backend.loss(lsteps)
            for i in fwd_finished:
                s = self.slots[i]
                s.terms = dict(zip(LOSS_SLOTS, env[:, i].tolist()))
                s.loss = s.terms["total"]
                s.fx = self.backend.final_x(i)
                if s.req.grad:
                    t_last = s.req.steps - 1
                    s.phase, s.seg = "rev", (t_last + self.K - 1) // self.K - 1
                else:
                    done.append(server._finish(self, i, None))
        for i, s in enumerate(self.slots):
            if s.phase == "rev" and s.seg < 0:
                done.append(server._finish(self, i, self.backend.grads(i)))
        return done


class Server:
    """Continuous-batching request loop over resident env slots.

    types:         {name: RobotType or MpmType}
    slots:         {name: number of slots of that type}; each mass-spring type
                   is a pool (one batch on its own CUDA stream) that ticks at
                   its own pace, each MPM type a pool of one-env handles
    params:        ``batch.default_params`` of the served batches (max_steps
                   is the longest episode, checkpoint_every the segment length)
    hbm_budget:    bytes of request footprints admitted at once (None: no
                   limit beyond the slots)
    tick_segments: checkpoint segments a tick advances every request by
    """

    def __init__(self, types: Dict[str, RobotType], slots: Dict[str, int], params, hbm_budget=None,
                 backend_factory=None, streams=True, clock=time.perf_counter, tick_segments=1,
                 mpm_backend_factory=None):
        self.types = types
        self.K = int(params.checkpoint_every)
        self.rounds = max(1, int(tick_segments))
        self.T = int(params.max_steps)
        self.hbm_budget = hbm_budget
        self.used_bytes = 0
        self.clock = clock
        self.t0 = clock()
        self.queue: List[Request] = []
        self.results: List[Result] = []
        self.next_rid = 0
        self.substeps_done = 0
        self.ticks = 0
        self.pools: List[Pool] = []
        self._streams = []
        for name, n in slots.items():
            slot_types = [name] * n
            if isinstance(types[name], MpmType):
                mb = (mpm_backend_factory(types[name], n, self.T, self.K) if mpm_backend_factory is not None
                      else MpmSlotBackend(types[name], n, self.T, self.K, streams))
                self.pools.append(MpmPool(name, n, mb))
                continue
            if backend_factory is not None:
                backend = backend_factory(slot_types, types, params)
            else:
                stream = None
                if streams:
                    import torch
                    stream = torch.cuda.Stream()
                    self._streams.append(stream)
                backend = SlotBackend(slot_types, types, params, stream=stream)
            self.pools.append(Pool(slot_types, backend, self.K, self.T, self.rounds))

    def now(self):
        return self.clock() - self.t0

    def close(self):
        for p in self.pools:
            p.backend.close()

    # ---------------------------------------------------------------- requests
    def submit(self, req: Request) -> int:
        if req.kind not in self.types:
            raise KeyError("unknown robot type %r" % req.kind)
        if not 2 <= req.steps <= self.T:
            raise ValueError("steps must be in [2, %d]" % self.T)
        req.rid = self.next_rid
        self.next_rid += 1
        self.queue.append(req)
        return req.rid

    def footprint(self, req):
        t = self.types[req.kind]
        if isinstance(t, MpmType):
            return mpm_footprint_bytes(t, self.T, self.K)
        return footprint_bytes(t.robot, req.steps, req.grad, self.K)

    def _admit(self, pools):
        """FIFO admission into idle pools: a request waits for a free slot of
        its type and for HBM budget; later requests may pass it."""
        waiting = []
        for req in self.queue:
            fp = self.footprint(req)
            if self.hbm_budget is not None and self.used_bytes + fp > self.hbm_budget:
                waiting.append(req)
                continue
            placed = False
            for pool in pools:
                i = pool.free_slot(req.kind)
                if i < 0:
                    continue
                s = pool.slots[i]
                if isinstance(pool, Pool):
                    if pool.backend.loaded[i] != req.kind:
                        pool.backend.load_weights(i, req.kind, self.types[req.kind].weights)
                    pool.backend.reset(i, req, self.types[req.kind].robot)
                s.req, s.phase, s.pos, s.seg = req, "fwd", 0, 0
                s.admitted, s.bytes = self.now(), fp
                self.used_bytes += fp
                placed = True
                break
            if not placed:
                waiting.append(req)
        self.queue = waiting

    # -------------------------------------------------------------------- tick
    def tick(self) -> List[Result]:
        """One synchronous round: admit what fits, launch a tick in every pool,
        wait for them and return the requests that finished."""
        self._admit(self.pools)
        for pool in self.pools:
            pool.launch()
        done = []
        for pool in self.pools:
            if pool.plan is not None:
                done.extend(pool.complete(self))
        self.ticks += 1
        self.results.extend(done)
        return done

    def _finish(self, pool, i, grads):
        s = pool.slots[i]
        r = Result(rid=s.req.rid, kind=s.req.kind, steps=s.req.steps, grad=s.req.grad, loss=s.loss,
                   loss_terms=s.terms, final_x=s.fx, grads=grads, arrival=s.req.arrival,
                   admitted=s.admitted, done=self.now())
        self.used_bytes -= s.bytes
        s.req, s.phase, s.bytes = None, "free", 0
        return r

    def busy(self):
        return bool(self.queue) or any(p.busy() for p in self.pools)

    def drain(self):
        while self.busy():
            self.tick()
        return self.results

    # ------------------------------------------------------------ open loop
    def run(self, requests: Sequence[Request], max_seconds=None, poll=2e-4):
        """Serve requests at their arrival times (seconds from now), every
        pool ticking at its own pace: a pool whose tick is done collects its
        results, takes in waiting requests and launches its next tick while
        the other pools' ticks are still on the GPU.  Returns the results and
        latency / throughput statistics."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        self.t0 = self.clock()
        k = 0
        while k < len(reqs) or self.busy():
            t = self.now()
            while k < len(reqs) and reqs[k].arrival <= t:
                self.submit(reqs[k])
                k += 1
            progressed = False
            for pool in self.pools:
                if isinstance(pool, MpmPool):
                    # whole-rollout slots: collect what finished, refill free slots
                    if pool.ready():
                        self.results.extend(pool.complete(self))
                        progressed = True
                    self._admit([pool])
                    if pool.launch():
                        progressed = True
                    continue
                if pool.plan is not None:
                    if not pool.ready():
                        continue
                    self.results.extend(pool.complete(self))
                    progressed = True
                self._admit([pool])
                if pool.launch():
                    self.ticks += 1
                    progressed = True
            if not progressed:
                if self.busy():
                    time.sleep(poll)
                elif k < len(reqs):
                    time.sleep(max(0.0, min(reqs[k].arrival - self.now(), 0.01)))
            if max_seconds is not None and self.now() > max_seconds:
                break
        return self.results, self.stats()

    def stats(self):
        """Latency percentiles over the finished requests, split into the wait
        for admission (arrival -> admitted) and the service time (admitted ->
        done), overall and per robot type."""
        def pct(v):
            v = np.asarray(v) if len(v) else np.zeros(1)
            return {"p50": float(np.percentile(v, 50) * 1e3), "p99": float(np.percentile(v, 99) * 1e3)}

        lat = np.array([r.latency for r in self.results]) if self.results else np.zeros(1)
        wall = max(self.now(), 1e-9)
        per_kind = {}
        for k in sorted({r.kind for r in self.results}):
            rs = [r for r in self.results if r.kind == k]
            per_kind[k] = dict(pct([r.latency for r in rs]), n=len(rs))
        return {"requests": len(self.results), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3),
                "queue_ms": pct([r.admitted - r.arrival for r in self.results]),
                "service_ms": pct([r.done - r.admitted for r in self.results]),
                "per_kind_ms": per_kind,
                "env_substeps_per_s": self.substeps_done / wall, "ticks": self.ticks,
                "wall_s": wall}


def poisson_requests(rng, rate, duration, kinds, p_kinds, steps_lo=100, steps_hi=2000, p_grad=0.2):
    """Open-loop arrivals: Poisson at `rate` per second over `duration`
    seconds, robot types drawn with probabilities p_kinds, episode steps
    U{steps_lo..steps_hi}, a fraction p_grad of gradient queries."""
    out = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        k = kinds[int(rng.choice(len(kinds), p=p_kinds))]
        out.append(Request(kind=k, steps=int(rng.integers(steps_lo, steps_hi + 1)),
                           grad=bool(rng.random() < p_grad), seed=int(rng.integers(1 << 30)),
                           arrival=t))
    return out
