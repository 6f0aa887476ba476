"""The multi-GPU path of bench.py is replicas only (each rank solves its own instances, no data-path
collective); its host side, the barrier and the max-over-ranks timing reduction, runs here on two
gloo ranks on the CPU, and the per-rank workloads are checked: the batched mix is the same on every
rank (weak scaling), the served stream is each rank's own."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch

    import bench
    from fluxo_b200.workloads import SEED, batch_instance_specs, serve_request_specs

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.barrier(world)
        local_ms = 10.0 + 5.0 * rank
        out[rank] = (bench.max_over_ranks(local_ms, world, torch.device("cpu")),
                     [s["seed"] for s in batch_instance_specs(8)],
                     [round(s["arrival"], 9) for s in serve_request_specs(20.0, 1.0, seed=SEED + rank)])
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_replica_timing():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 15.0          # max over ranks
    assert res[0][1] == res[1][1]                  # same batched mix on every rank
    assert res[0][2] != res[1][2]                  # each rank serves its own stream
