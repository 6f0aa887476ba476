"""Served request stream on the GPU: continuous batching (requests join and leave the batch while
others run, under an HBM budget that holds only part of the stream) gives every request exactly
the result of its solo run (same steps, same final time, identical state)."""
import numpy as np
import pytest

import fluxo_b200 as fb
from fluxo_b200.batch import Batch, instance_bytes
from fluxo_b200.serve import Request, Server, serve_one_at_a_time
from fluxo_b200.workloads import build_instance, instance_fields, serve_request_specs

pytestmark = pytest.mark.gpu


def requests(n_max=12):
    specs = serve_request_specs(rate=2000.0, duration=0.006, seed=7, elems=(2, 5), N=(2, 5),
                                t_end=(0.2, 1.0))[:n_max]
    cache, reqs = {}, []
    for s in specs:
        mesh, U = build_instance(s, cache)
        reqs.append(Request(rid=s["index"], cfg=fb.make_cfg(**instance_fields(s)), mesh=mesh, U=U, t_end=s["t_end"],
                            arrival=s["arrival"]))
    return reqs


@pytest.mark.parametrize("device_loop", [True, False])
def test_served_results_equal_solo_runs(gpu_lib, device_loop):
    reqs = requests()
    assert len(reqs) >= 8
    sizes = [instance_bytes(r.cfg, r.mesh["ElemToSide"].shape[0], r.mesh["SideToElem"].shape[0]) for r in reqs]
    budget = max(sizes) + sorted(sizes)[len(sizes) // 2]   # room for only a few requests at a time
    b = Batch()
    srv = Server(b, hbm_budget=budget, instance_bytes=instance_bytes, steps_per_poll=1, device_loop=device_loop)
    stats = srv.serve(reqs)
    if device_loop:
        assert stats.loops >= 3
    b.close()
    assert len(stats.results) == len(reqs) and stats.rebuilds >= 3
    assert 2 <= stats.max_running < len(reqs) and stats.max_bytes <= budget
    solo = serve_one_at_a_time(reqs, lambda cfg: fb.DGOperator(cfg=cfg))
    alone = {r.rid: r for r in solo.results}
    for r in stats.results:
        a = alone[r.rid]
        assert r.err == a.err == 0 and r.steps == a.steps > 1 and r.t == a.t
        assert np.array_equal(r.U, a.U)
    s = stats.summary()
    assert s["p99_s"] >= s["p50_s"] > 0 and s["dof_updates_per_s"] > 0


def test_device_loop_ends_and_matches_run(gpu_lib):
    """fluxo_batch_loop_*: the while-graph stops at its step limit, when an instance finishes and when
    woken; the states equal those of fluxo_batch_run over the same steps, bit for bit; the batch
    refuses run / get_state while a loop is in flight."""
    from fluxo_b200 import _lib

    reqs = requests(4)
    b1, b2 = Batch(), Batch()
    ids1 = [b1.add(r.mesh, r.U, 0.0, r.t_end, cfg=r.cfg) for r in reqs]
    ids2 = [b2.add(r.mesh, r.U, 0.0, r.t_end, cfg=r.cfg) for r in reqs]
    b1.loop_start(3)
    with pytest.raises(_lib.FluxoError):
        b1.run(1)
    steps, why, running = b1.loop_wait()
    assert (steps, why, running) == (3, _lib.LOOP_STEP_LIMIT, 4)
    b2.run(3)
    for i1, i2 in zip(ids1, ids2):
        assert b1.status(i1) == b2.status(i2) and b1.status(i1)[1] == 3
        assert np.array_equal(b1.get_state(i1), b2.get_state(i2))
    # run to the first completion: the loop returns right after the step that finished an instance
    b1.loop_start(1 << 20)
    steps, why, running = b1.loop_wait()
    assert why == _lib.LOOP_FINISHED and running < 4
    assert any(b1.status(i)[2] for i in ids1)
    b2.run(steps)
    for i1, i2 in zip(ids1, ids2):
        assert b1.status(i1) == b2.status(i2)
        assert np.array_equal(b1.get_state(i1), b2.get_state(i2))
    # a woken loop returns after the step in flight
    b1.loop_start(1 << 20)
    b1.loop_wake()
    steps, why, _ = b1.loop_wait()
    assert why in (_lib.LOOP_WOKEN, _lib.LOOP_FINISHED) and steps >= 1
    b2.run(steps)
    for i1, i2 in zip(ids1, ids2):
        assert np.array_equal(b1.get_state(i1), b2.get_state(i2))
    # nothing running: the loop ends at once without a step
    for i in ids1:
        b1.remove(i)
    b1.loop_start(10)
    assert b1.loop_wait() == (0, _lib.LOOP_IDLE, 0)
    b1.close()
    b2.close()


def test_prepared_admission_equals_add(gpu_lib):
    """fluxo_batch_prepare (run on another thread) + fluxo_batch_add_prepared gives the same instance as
    fluxo_batch_add: same steps and identical states."""
    from concurrent.futures import ThreadPoolExecutor

    reqs = requests(3)
    b1, b2 = Batch(), Batch()
    with ThreadPoolExecutor(1) as ex:
        preps = [ex.submit(b1.prepare, r.mesh, r.U, 0.0, r.t_end, cfg=r.cfg) for r in reqs]
        ids1 = [b1.add_prepared(f.result()) for f in preps]
    ids2 = [b2.add(r.mesh, r.U, 0.0, r.t_end, cfg=r.cfg) for r in reqs]
    b1.run_to_end()
    b2.run_to_end()
    for i1, i2 in zip(ids1, ids2):
        assert b1.status(i1) == b2.status(i2) and b1.status(i1)[2]
        assert np.array_equal(b1.get_state(i1), b2.get_state(i2))
    b1.close()
    b2.close()
