"""Served request stream: continuous batching of independent solves on one GPU.

No counterpart in the reference (one solve per program).  Requests (a periodic-box Euler or
Navier-Stokes solve: mesh arrays, initial state, end time) arrive over time; the server keeps
their state on the device inside one ``Batch`` and advances all admitted requests together, one
graph replay per time step.  A request is admitted when its device bytes fit the HBM budget next to
the requests already running (first come, first served: a request that does not fit holds the ones
behind it), and leaves the batch as soon as it reaches its end time, which frees its bytes for
the next ones.  Each result is what the same solve gives alone (``DGOperator.time_disc``).

The step loop itself runs on the device (``Batch.loop_start``, a conditional while-node of a CUDA
graph): the GPU repeats the time step of all admitted requests and returns to the host only when a
request finishes, when the host wakes it because a newly arrived request fits the budget, or at a
step limit.  While it runs, the host takes in arrivals and prepares the admitted ones (``Batch.add``
is host-only), so that preparation overlaps the GPU's steps.  ``device_loop=False`` keeps the older
host-polled form (``steps_per_poll`` steps per ``Batch.run`` call).

The host work of an admission (configuration checks, the mesh repacked into the device layout:
about 0.4 s for a 24^3-element request at N=7) runs ahead of it on a worker thread
(``Batch.prepare``) as soon as a request is queued, for the queue's head up to ``prepare_budget``
bytes; the admission itself then only hands the prepared request to the batch.
"""
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Request:
    """One solve: kernel configuration (a ``FluxoCfg``), reference-layout mesh arrays, initial U."""
    rid: int
    cfg: object
    mesh: dict
    U: np.ndarray
    t_end: float
    arrival: float = 0.0            # seconds after the start of the stream
    dofs: int = 0
    nbytes: int = 0
    prepared: object = None         # future of Batch.prepare, started while the request is queued


@dataclass
class Result:
    rid: int
    U: np.ndarray
    t: float
    steps: int
    err: int
    arrival: float
    admitted: float
    finished: float
    dofs: int

    @property
    def time_to_solution(self):
        return self.finished - self.arrival


@dataclass
class ServeStats:
    results: list = field(default_factory=list)
    wall: float = 0.0
    rebuilds: int = 0
    loops: int = 0                  # device-resident loops started
    wakes: int = 0                  # loops the host woke for an admission
    start_s: float = 0.0            # host time in loop starts (placing admitted requests, graph launch)
    harvest_s: float = 0.0          # host time reading back and removing finished requests
    max_running: int = 0
    max_bytes: int = 0
    waited_for_memory: set = field(default_factory=set)  # requests that queued because the budget was full

    def dof_updates(self):
        """DOFs x RHS evaluations of all finished requests (5 stages per LSERK4-5 step)."""
        return sum(r.dofs * r.steps * 5 for r in self.results)

    def summary(self):
        tts = np.array([r.time_to_solution for r in self.results]) if self.results else np.zeros(1)
        return {"requests": len(self.results), "wall_s": self.wall,
                "dof_updates_per_s": self.dof_updates() / self.wall if self.wall > 0 else None,
                "p50_s": float(np.percentile(tts, 50)), "p99_s": float(np.percentile(tts, 99)),
                "mean_s": float(tts.mean()), "max_running": self.max_running, "max_device_bytes": self.max_bytes,
                "failed": sum(1 for r in self.results if r.err), "waited_for_memory": len(self.waited_for_memory)}


class Server:
    """Continuous batching over a ``Batch``: admission by HBM budget, eviction on completion.

    ``batch`` is a ``fluxo_b200.batch.Batch`` (or an object with its methods); ``instance_bytes``
    gives a request's device bytes; ``steps_per_poll`` time steps run between two admission rounds.
    """

    def __init__(self, batch, hbm_budget, instance_bytes, steps_per_poll=2, clock=time.perf_counter,
                 device_loop=True, max_loop_steps=1 << 20, poll_interval=2e-4, sleep=time.sleep,
                 prepare_ahead=True, prepare_budget=None):
        self.batch = batch
        self.budget = int(hbm_budget)
        self.instance_bytes = instance_bytes
        self.steps_per_poll = int(steps_per_poll)
        self.clock = clock
        self.device_loop = bool(device_loop)
        self.max_loop_steps = int(max_loop_steps)
        self.poll_interval = float(poll_interval)
        self.sleep = sleep
        self.prepare_ahead = bool(prepare_ahead) and hasattr(batch, "prepare")
        self.prepare_budget = int(prepare_budget if prepare_budget is not None else hbm_budget)
        self._pool = ThreadPoolExecutor(max_workers=1) if self.prepare_ahead else None
        self.queue = deque()
        self.running = {}           # batch id -> (request, admitted time)
        self.used = 0

    def close(self):
        """Stops the preparation worker (requests still queued keep their preparations)."""
        if self._pool is not None:
            self._pool.shutdown(wait=True)
            self._pool = None
            self.prepare_ahead = False

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, req):
        if not req.nbytes:
            nE = req.mesh["ElemToSide"].shape[0]
            req.nbytes = self.instance_bytes(req.cfg, nE, req.mesh["SideToElem"].shape[0])
            req.dofs = nE * (req.cfg.N + 1) ** 3
        if req.nbytes > self.budget:
            raise ValueError("request %d needs %d device bytes, more than the budget %d" %
                             (req.rid, req.nbytes, self.budget))
        self.queue.append(req)

    def prepare(self):
        """Starts the host-side preparation of the queue's head, in arrival order, while the requests
        prepared but not yet admitted stay within ``prepare_budget`` bytes."""
        if not self.prepare_ahead:
            return
        held = 0
        for req in self.queue:
            if req.prepared is None:
                if held and held + req.nbytes > self.prepare_budget:
                    return
                req.prepared = self._pool.submit(self.batch.prepare, req.mesh, req.U, 0.0, req.t_end, cfg=req.cfg)
            held += req.nbytes

    def admit(self, now, stats=None, ready_only=False):
        """Adds queued requests in arrival order while they fit the budget; returns how many.  A request
        left at the head of the queue waits for memory (recorded in stats.waited_for_memory).  With
        ``ready_only`` the admission also stops at a request whose preparation is still running."""
        n = 0
        while self.queue and self.used + self.queue[0].nbytes <= self.budget:
            if ready_only and self.queue[0].prepared is not None and not self.queue[0].prepared.done():
                break
            req = self.queue.popleft()
            if req.prepared is not None:
                iid = self.batch.add_prepared(req.prepared.result())
                req.prepared = None
            else:
                iid = self.batch.add(req.mesh, req.U, 0.0, req.t_end, cfg=req.cfg)
            self.running[iid] = (req, now)
            self.used += req.nbytes
            n += 1
        if self.queue and stats is not None:
            stats.waited_for_memory.add(self.queue[0].rid)
        return n

    def harvest(self, now, stats):
        """Moves finished requests out of the batch (their result to the host)."""
        for iid in list(self.running):
            t, steps, done, err = self.batch.status(iid)
            if not done:
                continue
            req, admitted = self.running.pop(iid)
            U = self.batch.get_state(iid)
            self.batch.remove(iid)
            self.used -= req.nbytes
            stats.results.append(Result(req.rid, U, t, steps, err, req.arrival, admitted, self.clock() - self._t0,
                                        req.dofs))

    def serve(self, requests, stats=None):
        """Runs a stream to the end: each request becomes visible at its arrival time (seconds after
        the call), all of them finish.  Returns ServeStats with per-request results."""
        stats = stats or ServeStats()
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        self._t0 = self.clock()
        while pending or self.queue or self.running:
            now = self.clock() - self._t0
            while pending and pending[0].arrival <= now:
                self.submit(pending.popleft())
            if self.admit(now, stats):
                stats.rebuilds += 1
            self._track(stats)
            self.prepare()
            if self.running:
                if self.device_loop:
                    self._device_loop(pending, stats)
                else:
                    self.batch.run(self.steps_per_poll)
                h0 = self.clock()
                self.harvest(h0 - self._t0, stats)
                stats.harvest_s += self.clock() - h0
            elif pending:
                self.sleep(max(0.0, pending[0].arrival - (self.clock() - self._t0)))
        stats.wall = self.clock() - self._t0
        return stats

    def _track(self, stats):
        stats.max_running = max(stats.max_running, len(self.running))
        stats.max_bytes = max(stats.max_bytes, self.used)

    def _device_loop(self, pending, stats):
        """One device-resident loop: the GPU steps all admitted requests until one finishes.  Meanwhile
        arrivals are queued and admitted while they fit the budget (their host-side preparation runs
        during the GPU's steps); the first admission wakes the loop so that they join at the next start."""
        s0 = self.clock()
        self.batch.loop_start(self.max_loop_steps)
        stats.start_s += self.clock() - s0
        stats.loops += 1
        woken = False
        while True:
            r = self.batch.loop_poll()
            if r is not None:
                return r
            now = self.clock() - self._t0
            while pending and pending[0].arrival <= now:
                self.submit(pending.popleft())
            self.prepare()
            if self.queue and self.admit(now, stats, ready_only=True):
                stats.rebuilds += 1
                self._track(stats)
                if not woken:
                    self.batch.loop_wake()
                    stats.wakes += 1
                    woken = True
            self.sleep(self.poll_interval)


def serve_one_at_a_time(requests, make_operator, clock=time.perf_counter):
    """The plain path on the same stream: one solve at a time in arrival order (first come, first
    served), each through its own operator (``DGOperator``: set_mesh, set_state, time_disc)."""
    stats = ServeStats()
    t0 = clock()
    for req in sorted(requests, key=lambda r: r.arrival):
        now = clock() - t0
        if req.arrival > now:
            time.sleep(req.arrival - now)
        start = clock() - t0
        op = make_operator(req.cfg)
        op.set_mesh(req.mesh)
        op.set_state(req.U)
        t, steps, err = op.time_disc(0.0, req.t_end)
        U = op.get_state()
        op.close()
        nE = req.mesh["ElemToSide"].shape[0]
        stats.results.append(Result(req.rid, U, t, steps, err, req.arrival, start, clock() - t0,
                                    nE * (req.cfg.N + 1) ** 3))
    stats.wall = clock() - t0
    return stats
