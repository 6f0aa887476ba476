"""Batched solves: many independent Euler / Navier-Stokes instances advanced together on one GPU.

The reference runs one mesh per program (src/fluxo.f90); ``Batch`` wraps the ``fluxo_batch`` C ABI,
which concatenates instances of the same kernel configuration into one launch per kernel and
replays one CUDA graph per time step of all instances.  Each instance advances exactly as
``DGOperator.time_disc`` would advance it alone: per-instance CALCTIMESTEP, dt clipped to its own
end time (src/timedisc/timedisc.f90:274-359).
"""
import ctypes

import numpy as np

from . import _lib
from .solver import MESH_KEYS, _c, _ptr, make_cfg


def instance_bytes(cfg, n_elems, n_sides):
    """Device bytes one instance of ``cfg`` with this mesh size occupies inside a batch."""
    b = ctypes.c_size_t()
    _lib.check(_lib.load().fluxo_batch_instance_bytes(ctypes.byref(cfg), int(n_elems), int(n_sides),
                                                      ctypes.byref(b)))
    return b.value


class Prepared:
    """A request repacked on the host (``fluxo_batch_prepare``), waiting for ``Batch.add_prepared``."""

    def __init__(self, lib, p, shape):
        self.lib, self.p, self.shape = lib, p, shape

    def __del__(self):
        if getattr(self, "p", None) is not None:
            self.lib.fluxo_batch_prepared_free(self.p)
            self.p = None


class Batch:
    """A set of independent solves on one device (``fluxo_batch_*``)."""

    def __init__(self, device=0):
        self.lib = _lib.load()
        b = ctypes.c_void_p()
        _lib.check(self.lib.fluxo_batch_create(int(device), ctypes.byref(b)), None)
        self.b = b
        self._shapes = {}

    def close(self):
        if getattr(self, "b", None):
            self.lib.fluxo_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        self.close()

    def _check(self, r):
        if r != _lib.FLUXO_OK:
            buf = ctypes.create_string_buffer(1024)
            self.lib.fluxo_batch_last_error(self.b, buf, 1024)
            raise _lib.FluxoError(r, buf.value.decode(errors="replace"))

    def add(self, mesh, U, t, t_end, cfg=None, max_iter=-1, **fields):
        """Adds an instance (reference-layout mesh arrays, initial U); returns its id."""
        cfg = cfg if cfg is not None else make_cfg(**fields)
        S2E = _c(mesh["SideToElem"], np.int32)
        E2S = _c(mesh["ElemToSide"], np.int32)
        arrs = [_c(mesh[k]) for k in MESH_KEYS[2:10]]
        U = _c(U)
        nE, nS = E2S.shape[0], S2E.shape[0]
        n = cfg.N + 1
        if U.size != nE * n ** 3 * 5:
            raise ValueError("U has the wrong size")
        iid = ctypes.c_int()
        r = self.lib.fluxo_batch_add(self.b, ctypes.byref(cfg), nE, nS, _ptr(S2E), _ptr(E2S), *[_ptr(a) for a in arrs],
                                     _ptr(U), float(t), float(t_end), int(max_iter), ctypes.byref(iid))
        self._check(r)
        self._shapes[iid.value] = (nE, n, n, n, 5)
        return iid.value

    def prepare(self, mesh, U, t, t_end, cfg=None, max_iter=-1, **fields):
        """The host work of ``add`` (checks, mesh repack) without touching the batch: returns a
        ``Prepared`` for ``add_prepared``.  Safe to call from another thread while the batch runs."""
        cfg = cfg if cfg is not None else make_cfg(**fields)
        S2E = _c(mesh["SideToElem"], np.int32)
        E2S = _c(mesh["ElemToSide"], np.int32)
        arrs = [_c(mesh[k]) for k in MESH_KEYS[2:10]]
        U = _c(U)
        nE, nS = E2S.shape[0], S2E.shape[0]
        n = cfg.N + 1
        if U.size != nE * n ** 3 * 5:
            raise ValueError("U has the wrong size")
        p = ctypes.c_void_p()
        _lib.check(self.lib.fluxo_batch_prepare(ctypes.byref(cfg), nE, nS, _ptr(S2E), _ptr(E2S),
                                                *[_ptr(a) for a in arrs], _ptr(U), float(t), float(t_end),
                                                int(max_iter), ctypes.byref(p)), None)
        return Prepared(self.lib, p, (nE, n, n, n, 5))

    def add_prepared(self, prep):
        """Adds a prepared instance (ownership passes to the batch); returns its id."""
        if prep.p is None:
            raise ValueError("prepared instance already added")
        iid = ctypes.c_int()
        self._check(self.lib.fluxo_batch_add_prepared(self.b, prep.p, ctypes.byref(iid)))
        prep.p = None
        self._shapes[iid.value] = prep.shape
        return iid.value

    def run(self, n_steps):
        """Advances every unfinished instance by up to n_steps steps; returns how many are unfinished."""
        running = ctypes.c_int()
        self._check(self.lib.fluxo_batch_run(self.b, int(n_steps), ctypes.byref(running)))
        return running.value

    def run_to_end(self, max_steps=1 << 30):
        while max_steps > 0:
            k = min(max_steps, 1024)
            if self.run(k) == 0:
                return
            max_steps -= k

    def loop_start(self, max_steps):
        """Starts the device-resident loop (``fluxo_batch_loop_start``) and returns at once: the GPU
        repeats the time step of all instances until one finishes, ``loop_wake`` is called, or
        ``max_steps`` steps ran."""
        self._check(self.lib.fluxo_batch_loop_start(self.b, int(max_steps)))

    def loop_wake(self):
        """Asks the running loop to return after its current step."""
        self._check(self.lib.fluxo_batch_loop_wake(self.b))

    def loop_poll(self):
        """None while the loop runs; else (steps run, end reason, instances still running)."""
        fin, n, why, run = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.fluxo_batch_loop_poll(self.b, ctypes.byref(fin), ctypes.byref(n), ctypes.byref(why),
                                                   ctypes.byref(run)))
        return (n.value, why.value, run.value) if fin.value else None

    def loop_wait(self):
        """Waits for the loop's end; returns (steps run, end reason, instances still running)."""
        n, why, run = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.fluxo_batch_loop_wait(self.b, ctypes.byref(n), ctypes.byref(why), ctypes.byref(run)))
        return n.value, why.value, run.value

    def status(self, iid):
        """(t, steps taken, finished, errType) of an instance."""
        t, n, done, err = ctypes.c_double(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.fluxo_batch_status(self.b, int(iid), ctypes.byref(t), ctypes.byref(n),
                                                ctypes.byref(done), ctypes.byref(err)))
        return t.value, n.value, bool(done.value), err.value

    def get_state(self, iid):
        U = np.empty(self._shapes[iid])
        self._check(self.lib.fluxo_batch_get_state(self.b, int(iid), _ptr(U)))
        return U

    def set_state(self, iid, U):
        """Overwrites the instance's U (``fluxo_batch_set_state``; its time and step count stay)."""
        U = _c(U)
        if U.size != int(np.prod(self._shapes[iid])):
            raise ValueError("U has the wrong size")
        self._check(self.lib.fluxo_batch_set_state(self.b, int(iid), _ptr(U)))

    def remove(self, iid):
        self._check(self.lib.fluxo_batch_remove(self.b, int(iid)))
        self._shapes.pop(iid, None)

    def stream(self):
        """The CUDA stream (as an integer handle) all of the batch's GPU work runs on."""
        s = ctypes.c_void_p()
        self._check(self.lib.fluxo_batch_stream(self.b, ctypes.byref(s)))
        return s.value

    def info(self):
        """(groups, placed instances, device bytes of the placed instances)."""
        g, n, d = ctypes.c_int(), ctypes.c_int(), ctypes.c_size_t()
        self._check(self.lib.fluxo_batch_info(self.b, ctypes.byref(g), ctypes.byref(n), ctypes.byref(d)))
        return g.value, n.value, d.value
