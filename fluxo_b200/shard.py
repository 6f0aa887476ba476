"""One solve over several handles: the element partition, the ghost-element halo and its exchanges.

The reference splits the elements of a mesh into contiguous ranges, one per MPI rank
(mesh_readin.f90:246-292, offsetElemMPI), and exchanges the face data of the sides between ranks
inside DGTimeDerivative (dg.f90:342-442: U_slave, the gradient traces, Flux_slave) and the time step
with MPI_ALLREDUCE (calctimestep.f90:159-167).  Here every rank's handle holds its owned elements and
whole ghost copies of the neighbouring elements of other ranks; both ranks of a partition side compute
its flux from the same two states, so the exchanges are

* FLUXO_XCHG_STATE  - the ghost elements' U (before each right-hand side),
* FLUXO_XCHG_GTRACE - the ghost side's viscous face share of each partition side (after the lifting),
* FLUXO_XCHG_DT     - MIN over the ranks of the dt bits and the error key (after CALCTIMESTEP),
* FLUXO_XCHG_ALPHA  - the ghost elements' NFVSE blending coefficients (before each propagation sweep),

driven by the library through the callback of ``fluxo_gpu_set_partition``.  ``Partition`` builds a
rank's local mesh and its exchange lists (host logic only); ``DistExchange`` moves the data with
``torch.distributed`` point-to-point operations (NCCL between GPUs, also gloo on CPU tensors) and
``ThreadExchange`` between several handles of one process (one host thread each, no device-side waits
between the handles' kernels).
"""

from __future__ import annotations

import threading
import traceback

import numpy as np

from . import _lib
from .solver import DGOperator

VOLUME_KEYS = ("Metrics_fTilde", "Metrics_gTilde", "Metrics_hTilde", "sJ", "Elem_xGP")
FACE_KEYS = ("NormVec", "TangVec1", "TangVec2", "SurfElem")


def element_offsets(n_elems, n_ranks):
    """offsetElemMPI of the reference (mesh_readin.f90:270-276): the first nElems mod nRanks ranks hold one
    element more than the others."""
    base, extra = divmod(int(n_elems), int(n_ranks))
    return np.array([base * r + min(r, extra) for r in range(n_ranks)] + [int(n_elems)], dtype=np.int64)


class Partition:
    """Rank ``rank`` of ``n_ranks`` of a mesh in the reference layout (the keys of ``solver.box_mesh``).

    ``mesh``: the rank's local mesh (owned elements first, then ghosts sorted by global id; every side of an
    owned element, in global side order).  ``owned`` / ``ghosts`` / ``sides``: their global (0-based) ids.
    ``peers``: {rank q: dict(state_send, state_recv, gt_send, gt_recv)} of local row indices, the state rows
    being local elements and the trace rows 2 * local side + role (0 master, 1 slave), all in ascending
    global order so that each send list matches the peer's receive list."""

    def __init__(self, mesh, n_ranks, rank):
        S2E = np.asarray(mesh["SideToElem"], dtype=np.int64)
        E2S = np.asarray(mesh["ElemToSide"], dtype=np.int64)
        nE = E2S.shape[0]
        if not 1 <= n_ranks <= nE:
            raise ValueError("need 1 <= n_ranks <= nElems")
        off = element_offsets(nE, n_ranks)
        self.n_ranks, self.rank, self.offsets = int(n_ranks), int(rank), off
        e0, e1 = int(off[rank]), int(off[rank + 1])
        owner = np.searchsorted(off, np.arange(nE), side="right") - 1
        self.owned = np.arange(e0, e1, dtype=np.int64)
        self.sides = np.unique(E2S[self.owned, :, 0].ravel() - 1)
        em, es = S2E[self.sides, 0] - 1, S2E[self.sides, 1] - 1
        ends = np.concatenate([em, es])
        self.ghosts = np.unique(ends[(ends < e0) | (ends >= e1)])
        self.n_owned = len(self.owned)
        elems = np.concatenate([self.owned, self.ghosts])
        g2l = np.full(nE, -1, dtype=np.int64)
        g2l[elems] = np.arange(len(elems))
        g2s = np.full(S2E.shape[0], -1, dtype=np.int64)
        g2s[self.sides] = np.arange(len(self.sides))
        # local connectivity (1-based ids, flips and local sides unchanged)
        s2e = S2E[self.sides].copy()
        s2e[:, 0] = g2l[em] + 1
        s2e[:, 1] = g2l[es] + 1
        e2s = np.zeros((len(elems), 6, 2), dtype=np.int64)
        e2s[: self.n_owned, :, 0] = g2s[E2S[self.owned, :, 0] - 1] + 1
        e2s[: self.n_owned, :, 1] = E2S[self.owned, :, 1]
        for k, g in enumerate(self.ghosts):  # ghosts: their local sides; the others any valid entry (unused)
            loc = g2s[E2S[g, :, 0] - 1]
            first = int(loc[loc >= 0][0])
            e2s[self.n_owned + k, :, 0] = np.where(loc >= 0, loc, first) + 1
            e2s[self.n_owned + k, :, 1] = np.where(loc >= 0, E2S[g, :, 1], 0)
        m = {"SideToElem": s2e.astype(np.int32), "ElemToSide": e2s.astype(np.int32)}
        for k in VOLUME_KEYS:
            if k in mesh:
                m[k] = np.ascontiguousarray(np.asarray(mesh[k])[elems])
        for k in FACE_KEYS:
            m[k] = np.ascontiguousarray(np.asarray(mesh[k])[self.sides])
        self.mesh = m
        self.elems = elems
        # exchange lists
        self.peers = {}
        ghost_owner = owner[self.ghosts]
        nb = {}  # owned element -> ranks of its neighbours
        for s_loc, (a, b) in enumerate(zip(em, es)):
            ra, rb = owner[a], owner[b]
            if ra == rank and rb != rank:
                nb.setdefault(int(rb), set()).add(int(a))
            if rb == rank and ra != rank:
                nb.setdefault(int(ra), set()).add(int(b))
        for q in sorted(set(ghost_owner.tolist()) | set(nb)):
            send_e = np.array(sorted(nb.get(q, ())), dtype=np.int64)
            recv_e = self.ghosts[ghost_owner == q]
            gt_send, gt_recv = [], []
            for s_loc, (a, b) in enumerate(zip(em, es)):
                ra, rb = owner[a], owner[b]
                if (ra == rank and rb == q) or (rb == rank and ra == q):
                    mine = 0 if ra == rank else 1
                    gt_send.append(2 * s_loc + mine)
                    gt_recv.append(2 * s_loc + 1 - mine)
            self.peers[q] = dict(state_send=g2l[send_e], state_recv=g2l[recv_e],
                                 gt_send=np.array(gt_send, dtype=np.int64), gt_recv=np.array(gt_recv, dtype=np.int64))

    def local_state(self, U_global):
        """The rank's local state (owned, then ghosts) from a global U (C view [elem][k][j][i][var])."""
        return np.ascontiguousarray(np.asarray(U_global)[self.elems])


class _DeviceArray:
    """A device pointer as a __cuda_array_interface__ object (no copy, no ownership)."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2, "strides": None}


class _Exchange:
    """Index tensors of a partition and the three exchanges on torch tensors; subclasses move the rows."""

    def __init__(self, part, device, nvar, npts):
        import torch

        self.part, self.device, self.nvar, self.npts = part, device, int(nvar), int(npts)
        self.n_local = len(part.elems)
        self.n_sides = len(part.sides)
        self.idx = {q: {k: torch.as_tensor(v, dtype=torch.int64, device=device) for k, v in d.items()}
                    for q, d in part.peers.items()}

    def apply(self, what, a, b):
        if what == _lib.FLUXO_XCHG_STATE:
            self._swap(a.view(self.n_local, -1), "state_send", "state_recv")
        elif what == _lib.FLUXO_XCHG_GTRACE:
            if a is not None:
                self._swap(a.view(2 * self.n_sides, -1), "gt_send", "gt_recv")
        elif what == _lib.FLUXO_XCHG_DT:
            self._min(a, b)
        elif what == _lib.FLUXO_XCHG_ALPHA:
            self._swap(a.view(self.n_local, 1), "state_send", "state_recv")
        else:
            raise ValueError("unknown exchange %d" % what)

    # the library's callback: device pointers -> tensor views on the handle's stream
    def callback(self, op):
        import torch

        np3 = self.npts ** 3
        nvisc = 7 if self.nvar == 9 else 4  # n.F_v components per face point (MHD: variables 2..8)
        nst, ngt = self.n_local * self.nvar * np3, 2 * self.n_sides * nvisc * self.npts ** 2

        def cb(ctx, what, stream, a, b):
            try:
                dev = torch.device(self.device)
                with torch.cuda.device(dev), torch.cuda.stream(torch.cuda.ExternalStream(stream, device=dev)):
                    if what == _lib.FLUXO_XCHG_STATE:
                        A = torch.as_tensor(_DeviceArray(a, nst, "<f8"), device=dev)
                        self.apply(what, A, None)
                    elif what == _lib.FLUXO_XCHG_GTRACE:
                        A = torch.as_tensor(_DeviceArray(a, ngt, "<f8"), device=dev) if a else None
                        self.apply(what, A, None)
                    elif what == _lib.FLUXO_XCHG_ALPHA:
                        A = torch.as_tensor(_DeviceArray(a, self.n_local, "<f8"), device=dev)
                        self.apply(what, A, None)
                    else:
                        A = torch.as_tensor(_DeviceArray(a, 1, "<i8"), device=dev)
                        B = torch.as_tensor(_DeviceArray(b, 1, "<i4"), device=dev)
                        self.apply(what, A, B)
                return 0
            except Exception:  # reported as FLUXO_EXCHANGE by the library
                traceback.print_exc()
                return 1

        return _lib.EXCHANGE_FN(cb)


class DistExchange(_Exchange):
    """torch.distributed point-to-point exchange (rank = the process group's rank; NCCL or gloo)."""

    def _swap(self, X, send_key, recv_key):
        import torch
        import torch.distributed as dist

        # one group of all sends and receives (ncclGroupStart/End under NCCL: separate point-to-point calls
        # between two ranks that both send first would wait on each other)
        ops, recvs = [], []
        for q, ix in self.idx.items():
            if ix[send_key].numel():
                ops.append(dist.P2POp(dist.isend, X.index_select(0, ix[send_key]).contiguous(), q))
            if ix[recv_key].numel():
                buf = torch.empty((ix[recv_key].numel(), X.shape[1]), dtype=X.dtype, device=X.device)
                ops.append(dist.P2POp(dist.irecv, buf, q))
                recvs.append((ix[recv_key], buf))
        if ops:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
        for rows, buf in recvs:
            X.index_copy_(0, rows, buf)

    def _min(self, a, b):
        import torch.distributed as dist

        dist.all_reduce(a, op=dist.ReduceOp.MIN)
        dist.all_reduce(b, op=dist.ReduceOp.MIN)


class ThreadExchange:
    """The exchanges of several handles of one process, one host thread per handle: each rank packs its
    rows into a buffer on its own stream, waits for its stream, meets the others at a barrier (with a
    timeout), and copies the others' buffers into its ghost rows.  No kernel waits for another handle's."""

    class _Rank(_Exchange):
        def __init__(self, hub, part, device, nvar, npts):
            super().__init__(part, device, nvar, npts)
            self.hub = hub

        def _wait(self):
            import torch

            torch.cuda.current_stream().synchronize()
            self.hub.barrier.wait()

        def _swap(self, X, send_key, recv_key):
            r = self.part.rank
            self.hub.box[r] = {q: X.index_select(0, ix[send_key]) for q, ix in self.idx.items()}
            self._wait()
            for q, ix in self.idx.items():
                if ix[recv_key].numel():
                    X.index_copy_(0, ix[recv_key], self.hub.box[q][r])
            self._wait()

        def _min(self, a, b):
            r = self.part.rank
            self.hub.box[r] = (int(a.item()), int(b.item()))
            self._wait()
            da = min(v[0] for v in self.hub.box.values())
            db = min(v[1] for v in self.hub.box.values())
            a.fill_(da)
            b.fill_(db)
            self._wait()

    def __init__(self, n_ranks, timeout=120.0):
        self.barrier = threading.Barrier(n_ranks, timeout=timeout)
        self.box = {}

    def rank(self, part, device, nvar, npts):
        return ThreadExchange._Rank(self, part, device, nvar, npts)


class ShardedOperator:
    """One rank of a partitioned solve: a DGOperator on the rank's local mesh with its exchange callback."""

    def __init__(self, mesh, n_ranks, rank, exchange_factory, device=0, **fields):
        self.part = Partition(mesh, n_ranks, rank)
        self.op = DGOperator(device=device, **fields)
        self.op.set_mesh(self.part.mesh)
        self.exchange = exchange_factory(self.part, "cuda:%d" % device, self.op.nVar, self.op.N + 1)
        self._cb = self.exchange.callback(self)  # kept alive as long as the handle
        _lib.check(self.op.lib.fluxo_gpu_set_partition(self.op.h, self.part.n_owned, self._cb, None), self.op.h)

    def set_state(self, U_global):
        self.op.set_state(self.part.local_state(U_global))

    def get_state(self):
        """This rank's owned elements of U (global ids ``part.owned``)."""
        return self.op.get_state()[: self.part.n_owned]

    def get_ut(self):
        return self.op.get_ut()[: self.part.n_owned]

    def close(self):
        self.op.close()
