"""Large host <-> device copies of the C ABI (fluxo_gpu_set_state / get_state / set_mesh, fluxo_batch_add /
get_state): pageable host arrays of several 32 MiB chunks and a ragged last chunk go through the staged
path (page-locked bounce buffers, parallel host copy), page-locked ones directly; both give back every
bit."""
import numpy as np
import pytest

import fluxo_b200 as fb
from fluxo_b200.batch import Batch
from fluxo_b200.solver import box_mesh, get_state_ptr, set_state_ptr

pytestmark = pytest.mark.gpu

# N=7 on 17 x 16 x 9 elements: U is 2448 * 512 * 5 doubles = 50.1 MB (one full 32 MiB chunk and a ragged
# one), the metrics 90 MB
ELEMS = (17, 16, 9)


@pytest.fixture(scope="module")
def big():
    mesh = box_mesh(7, ELEMS, (0.0,) * 3, (2.0,) * 3, NGeo=1)
    nE = mesh["ElemToSide"].shape[0]
    rng = np.random.default_rng(11)
    U = 1.0 + 0.01 * rng.standard_normal((nE, 8, 8, 8, 5))
    U[..., 4] += 2.5  # positive pressure
    return mesh, U


def test_state_roundtrip_pageable_and_pinned(gpu_lib, big):
    import torch

    mesh, U = big
    op = fb.DGOperator(N=7, eqn=0, riemann=1, volume_flux=5, device=0)
    op.set_mesh(mesh)
    op.set_state(U)
    assert np.array_equal(op.get_state(), U)
    # a second state through page-locked host memory (the direct path)
    V = U[::-1].copy()
    pin = torch.empty(V.size, dtype=torch.float64, pin_memory=True)
    pin.numpy()[:] = V.ravel()
    set_state_ptr(op, pin.data_ptr())
    out = torch.zeros_like(pin).pin_memory()
    get_state_ptr(op, out.data_ptr())
    assert np.array_equal(out.numpy(), V.ravel())
    assert np.array_equal(op.get_state(), V)
    op.close()


def test_batch_placement_and_readback(gpu_lib, big):
    """An instance placed from pageable host arrays (staged uploads of U, metrics, face data) and read
    back equals the same state set on a handle; one step advances both alike."""
    mesh, U = big
    b = Batch(device=0)
    cfg = fb.make_cfg(N=7, eqn=0, riemann=1, volume_flux=5, device=0)
    iid = b.add(mesh, U, 0.0, 1.0, cfg=cfg, max_iter=1)
    b.run(1)
    op = fb.DGOperator(cfg=cfg)
    op.set_mesh(mesh)
    op.set_state(U)
    t, n, err = op.time_disc(0.0, 1.0, 1)
    assert err == 0 and n == 1 and b.status(iid)[1] == 1
    assert np.array_equal(b.get_state(iid), op.get_state())
    W = U[:, ::-1].copy()
    b.set_state(iid, W)  # staged upload into the placed instance
    assert np.array_equal(b.get_state(iid), W)
    op.close()
    b.close()
