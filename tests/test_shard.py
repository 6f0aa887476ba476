"""One solve over several ranks, host side on the CPU: the element partition of the reference
(offsetElemMPI), each rank's local mesh with its ghost elements, the exchange lists (every rank's send
list is its peer's receive list, in the same order), and the exchanges themselves on 2 and 3 gloo
ranks (torch.distributed point-to-point on CPU tensors, the code that runs over NCCL between GPUs):
after them every ghost row holds its owner's values and dt / the error key are the minima over ranks."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import fluxo_b200 as fb
from fluxo_b200 import _lib, hopr
from fluxo_b200.shard import DistExchange, Partition, element_offsets

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def box(ne=(3, 2, 2), N=2):
    return fb.box_mesh(N, ne, (-1, -1, -1), (1, 1, 1), NGeo=2, deform_amp=0.1)


def test_element_offsets_follow_the_reference():
    # mesh_readin.f90:270-276: nElems/nProcs each, the first MOD(nElems,nProcs) ranks one more
    for nE, nR in [(27, 2), (27, 4), (12, 3), (10, 10), (7, 1)]:
        off = element_offsets(nE, nR)
        base, extra = divmod(nE, nR)
        assert off[0] == 0 and off[-1] == nE
        assert list(np.diff(off)) == [base + (r < extra) for r in range(nR)]


@pytest.mark.parametrize("mesh_name,n_ranks", [("box", 2), ("box", 3), ("box", 5), ("warped", 2), ("warped", 4)])
def test_partition_consistency(mesh_name, n_ranks):
    mesh = box() if mesh_name == "box" else hopr.load_mesh(
        os.path.join(GOLDEN, "hopr_ConformBoxHeavilyWarped_Ngeo3_03_03_03.h5"), 2)
    S2E, E2S = mesh["SideToElem"], mesh["ElemToSide"]
    parts = [Partition(mesh, n_ranks, r) for r in range(n_ranks)]
    owned = np.concatenate([p.owned for p in parts])
    assert np.array_equal(owned, np.arange(E2S.shape[0]))
    for p in parts:
        m = p.mesh
        nl = len(p.elems)
        # every side of an owned element is local and both its elements are present
        for k, g in enumerate(p.owned):
            for ls in range(6):
                sid = m["ElemToSide"][k, ls, 0] - 1
                assert p.sides[sid] == E2S[g, ls, 0] - 1 and m["ElemToSide"][k, ls, 1] == E2S[g, ls, 1]
        s2e = m["SideToElem"]
        assert s2e[:, :2].min() >= 1 and s2e[:, :2].max() <= nl
        assert np.array_equal(p.elems[s2e[:, 0] - 1], S2E[p.sides, 0] - 1)
        assert np.array_equal(p.elems[s2e[:, 1] - 1], S2E[p.sides, 1] - 1)
        assert np.array_equal(s2e[:, 2:], S2E[p.sides, 2:])
        for k in ("NormVec", "SurfElem"):
            assert np.array_equal(m[k], mesh[k][p.sides])
        assert np.array_equal(m["sJ"], mesh["sJ"][p.elems])
        # the ghosts are exactly the rows received from the peers
        recv = np.sort(np.concatenate([p.elems[d["state_recv"]] for d in p.peers.values()]))
        assert np.array_equal(recv, p.ghosts)
    # send lists equal the peers' receive lists (global element ids; global side and role)
    for p in parts:
        for q, d in p.peers.items():
            e = parts[q].peers[p.rank]
            assert np.array_equal(p.elems[d["state_send"]], parts[q].elems[e["state_recv"]])
            mine = [(p.sides[r // 2], r % 2) for r in d["gt_send"]]
            theirs = [(parts[q].sides[r // 2], r % 2) for r in e["gt_recv"]]
            assert mine == theirs and len(mine) > 0


def test_partition_of_one_rank_is_the_mesh():
    mesh = box()
    p = Partition(mesh, 1, 0)
    assert len(p.ghosts) == 0 and p.peers == {}
    for k in ("SideToElem", "ElemToSide", "sJ", "NormVec"):
        assert np.array_equal(np.asarray(p.mesh[k]), np.asarray(mesh[k]))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        N, nvar = 2, 5
        mesh = box((4, 3, 2), N)
        part = Partition(mesh, world, rank)
        ex = DistExchange(part, "cpu", nvar, N + 1)
        np3, npt = (N + 1) ** 3, (N + 1) ** 2
        nl, ns = len(part.elems), len(part.sides)
        # state: owned rows carry their global id, ghost rows NaN
        U = torch.full((nl * np3 * nvar,), float("nan"), dtype=torch.float64)
        Uv = U.view(nl, -1)
        for k in range(part.n_owned):
            Uv[k] = float(part.elems[k]) + torch.arange(np3 * nvar, dtype=torch.float64) * 1e-3
        ex.apply(_lib.FLUXO_XCHG_STATE, U, None)
        ok_state = all(torch.equal(Uv[k], float(part.elems[k]) + torch.arange(np3 * nvar, dtype=torch.float64) * 1e-3)
                       for k in range(nl))
        # traces: each rank fills the shares of its owned elements with (global side, role)
        G = torch.full((ns * 2 * 4 * npt,), float("nan"), dtype=torch.float64)
        Gv = G.view(2 * ns, -1)
        s2e = part.mesh["SideToElem"]
        for s in range(ns):
            for role in (0, 1):
                if s2e[s, role] - 1 < part.n_owned:
                    Gv[2 * s + role] = 10.0 * part.sides[s] + role
        ex.apply(_lib.FLUXO_XCHG_GTRACE, G, None)
        ok_trace = all(torch.all(Gv[2 * s + role] == 10.0 * part.sides[s] + role)
                       for s in range(ns) for role in (0, 1))
        # dt bits and error key: minima over the ranks
        a = torch.tensor([1000 + 7 * rank], dtype=torch.int64)
        b = torch.tensor([2147483647 if rank != world - 1 else 42], dtype=torch.int32)
        ex.apply(_lib.FLUXO_XCHG_DT, a, b)
        out[rank] = (ok_state, ok_trace, int(a.item()), int(b.item()), len(part.ghosts))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(180)
@pytest.mark.parametrize("world", [2, 3])
def test_gloo_exchange(world):
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        ok_state, ok_trace, a, b, nghost = res[r]
        assert ok_state and ok_trace and nghost > 0
        assert a == 1000 and b == 42
