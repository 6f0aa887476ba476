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


def test_served_results_equal_solo_runs(gpu_lib):
    reqs = requests()
    assert len(reqs) >= 8
    sizes = [instance_bytes(r.cfg, r.mesh["ElemToSide"].shape[0], r.mesh["SideToElem"].shape[0]) for r in reqs]
    budget = max(sizes) + sorted(sizes)[len(sizes) // 2]   # room for only a few requests at a time
    b = Batch()
    srv = Server(b, hbm_budget=budget, instance_bytes=instance_bytes, steps_per_poll=1)
    stats = srv.serve(reqs)
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
