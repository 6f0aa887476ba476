"""Host logic of the served request stream (fluxo_b200.serve) on a fake batch, no GPU:
admission by HBM budget in arrival order, eviction on completion, result bookkeeping."""
import numpy as np
import pytest

from fluxo_b200.serve import Request, Server, ServeStats


class FakeCfg:
    def __init__(self, N):
        self.N = N


class FakeBatch:
    """Each instance takes ceil(t_end / dt) steps; records the admission order."""

    def __init__(self, dt=0.1):
        self.dt = dt
        self.inst = {}
        self.next = 1
        self.order = []
        self.live_bytes = []

    def add(self, mesh, U, t, t_end, cfg=None):
        self.added_during_loop = getattr(self, "added_during_loop", 0) + (getattr(self, "loop", None) is not None)
        iid = self.next
        self.next += 1
        self.inst[iid] = dict(U=U.copy(), t=t, t_end=t_end, steps=0, done=False)
        self.order.append(int(U.ravel()[0]))
        return iid

    def run(self, k):
        for s in self.inst.values():
            for _ in range(k):
                if s["done"]:
                    break
                s["t"] = min(s["t"] + self.dt, s["t_end"])
                s["steps"] += 1
                s["U"] += 1.0
                s["done"] = s["t"] >= s["t_end"]
        return sum(not s["done"] for s in self.inst.values())

    # device-resident loop: one poll advances one step (a stand-in for the GPU's progress between polls)
    def loop_start(self, max_steps):
        assert getattr(self, "loop", None) is None, "loop_start while a loop runs"
        self.loop = dict(max=max_steps, steps=0, woken=False,
                         running0=sum(not s["done"] for s in self.inst.values()))
        self.loops = getattr(self, "loops", 0) + 1

    def loop_wake(self):
        self.loop["woken"] = True

    def loop_poll(self):
        lp = self.loop
        running = self.run(1)
        lp["steps"] += 1
        why = 1 if running < lp["running0"] else 2 if lp["woken"] else 3 if lp["steps"] >= lp["max"] else 0
        if why == 0:
            return None
        self.loop = None
        return lp["steps"], why, running

    def status(self, iid):
        s = self.inst[iid]
        return s["t"], s["steps"], s["done"], 0

    def get_state(self, iid):
        return self.inst[iid]["U"].copy()

    def remove(self, iid):
        del self.inst[iid]


def mesh(nE):
    return {"ElemToSide": np.zeros((nE, 6, 2), np.int32), "SideToElem": np.zeros((3 * nE, 5), np.int32)}


def fake_bytes(cfg, nE, nS):
    return 1000 * nE


def make_requests(n, seed=0):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        nE = int(rng.integers(1, 9))
        reqs.append(Request(rid=i, cfg=FakeCfg(3), mesh=mesh(nE), U=np.full(4, float(i)),
                            t_end=float(rng.uniform(0.1, 1.0)), arrival=float(i) * 1e-7))
    return reqs


class CountingServer(Server):
    def admit(self, now, stats=None, ready_only=False):
        n = super().admit(now, stats, ready_only)
        assert self.used <= self.budget
        return n


@pytest.mark.parametrize("device_loop", [True, False])
def test_admission_respects_budget_and_order(device_loop):
    fb = FakeBatch()
    srv = CountingServer(fb, hbm_budget=12000, instance_bytes=fake_bytes, steps_per_poll=1,
                         device_loop=device_loop, sleep=lambda s: None)
    reqs = make_requests(40)
    stats = srv.serve(reqs)
    assert len(stats.results) == 40
    assert fb.order == list(range(40))                 # first come, first served
    assert stats.max_bytes <= 12000 and stats.max_running >= 2
    assert not fb.inst and srv.used == 0               # every request left the batch
    for r in stats.results:
        req = reqs[r.rid]
        steps = int(np.ceil(req.t_end / 0.1 - 1e-12))
        assert r.steps == steps and r.t == pytest.approx(req.t_end)
        assert np.array_equal(r.U, req.U + steps)      # the result is the request's own state
        assert r.finished >= r.admitted >= r.arrival - 1e-9
        assert r.dofs == req.mesh["ElemToSide"].shape[0] * 64
    s = stats.summary()
    assert s["requests"] == 40 and s["p99_s"] >= s["p50_s"] >= 0 and s["failed"] == 0
    # the budget holds a few requests at a time: later ones waited for memory, and the count says so
    assert 0 < s["waited_for_memory"] < 40 and stats.max_running < 40


def test_request_larger_than_budget_is_refused():
    srv = Server(FakeBatch(), hbm_budget=5000, instance_bytes=fake_bytes)
    with pytest.raises(ValueError):
        srv.submit(Request(rid=0, cfg=FakeCfg(3), mesh=mesh(6), U=np.zeros(4), t_end=1.0))


def test_stats_throughput_counts_rhs_evaluations():
    st = ServeStats()
    srv = Server(FakeBatch(dt=0.25), hbm_budget=10 ** 9, instance_bytes=fake_bytes)
    stats = srv.serve([Request(rid=0, cfg=FakeCfg(3), mesh=mesh(2), U=np.zeros(4), t_end=1.0)], st)
    assert stats.dof_updates() == 2 * 64 * 4 * 5


class StepClock:
    """A clock that advances by a fixed amount per reading (the stream's arrivals then fall inside
    device loops, as they do on the GPU)."""

    def __init__(self, dt):
        self.t, self.dt = 0.0, dt

    def __call__(self):
        self.t += self.dt
        return self.t


def test_device_loop_wakes_for_arrivals_that_fit():
    """Requests arriving while a loop runs are admitted during the loop (prepared on the host while
    the device steps) and wake it; a loop ends otherwise only when a request finishes."""
    fb = FakeBatch(dt=0.05)
    rng = np.random.default_rng(3)
    reqs = [Request(rid=i, cfg=FakeCfg(3), mesh=mesh(int(rng.integers(1, 4))), U=np.full(4, float(i)),
                    t_end=float(rng.uniform(0.5, 1.5)), arrival=0.01 * i) for i in range(30)]
    srv = Server(fb, hbm_budget=10 ** 9, instance_bytes=fake_bytes, clock=StepClock(1e-3), sleep=lambda s: None)
    stats = srv.serve(reqs)
    assert len(stats.results) == 30 and not fb.inst
    assert stats.loops >= 2 and stats.wakes >= 1
    assert fb.added_during_loop >= 1                   # admitted while the device stepped
    for r in stats.results:
        steps = int(np.ceil(reqs[r.rid].t_end / 0.05 - 1e-12))
        assert r.steps == steps and np.array_equal(r.U, reqs[r.rid].U + steps)
    # with a budget that holds one request, arrivals never wake the loop: they wait for memory
    fb = FakeBatch(dt=0.05)
    one = [Request(rid=r.rid, cfg=r.cfg, mesh=mesh(3), U=r.U, t_end=r.t_end, arrival=r.arrival) for r in reqs[:10]]
    srv = Server(fb, hbm_budget=3000, instance_bytes=fake_bytes, clock=StepClock(1e-3), sleep=lambda s: None)
    stats = srv.serve(one)
    assert len(stats.results) == 10 and stats.wakes == 0 and stats.max_running == 1


class PreparingBatch(FakeBatch):
    """A fake batch with the two-part admission: prepare (host work, any thread) and add_prepared."""

    def prepare(self, mesh, U, t, t_end, cfg=None):
        self.prepared = getattr(self, "prepared", 0) + 1
        return ("prepared", mesh, U.copy(), t, t_end, cfg)

    def add_prepared(self, p):
        assert p[0] == "prepared"
        return self.add(p[1], p[2], p[3], p[4], cfg=p[5])


def test_requests_are_prepared_ahead_of_admission():
    """Requests queued behind others are prepared on the worker thread before their admission, and
    the results are those of plain admissions."""
    fb = PreparingBatch(dt=0.05)
    reqs = make_requests(25, seed=5)
    srv = Server(fb, hbm_budget=12000, instance_bytes=fake_bytes, clock=StepClock(1e-3), sleep=lambda s: None)
    stats = srv.serve(reqs)
    assert len(stats.results) == 25 and fb.prepared >= 20 and fb.order == list(range(25))
    for r in stats.results:
        steps = int(np.ceil(reqs[r.rid].t_end / 0.05 - 1e-12))
        assert r.steps == steps and np.array_equal(r.U, reqs[r.rid].U + steps)
    # the preparation holds at most prepare_budget bytes beyond the admitted requests (the first one
    # always starts)
    srv = Server(PreparingBatch(), hbm_budget=12000, instance_bytes=fake_bytes, prepare_budget=3000)
    for r in make_requests(10, seed=6):
        srv.submit(r)
    srv.prepare()
    started = [r for r in srv.queue if r.prepared is not None]
    assert len(started) >= 1 and (len(started) == 1 or sum(r.nbytes for r in started) <= 3000)


def test_close_stops_the_preparation_worker():
    srv = Server(PreparingBatch(), hbm_budget=12000, instance_bytes=fake_bytes)
    with srv:
        stats = srv.serve(make_requests(5, seed=9))
    assert len(stats.results) == 5 and srv._pool is None and not srv.prepare_ahead
