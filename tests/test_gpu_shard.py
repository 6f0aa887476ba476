"""One solve partitioned over several handles, run on one GPU: each handle owns a contiguous element range
(the reference's offsetElemMPI) plus ghost copies of its neighbours, and the library calls the exchange
callback for the ghost states, the viscous face shares of the partition sides and the global dt.  Here
the handles share one GPU and exchange through host threads (ThreadExchange: each handle's thread waits
for its own stream and meets the others at a barrier; no kernel waits for another handle).  The owned
rows of Ut and of the states after device-resident time steps equal those of one handle on the whole
mesh (same arithmetic on the same data: to 1e-15)."""
import os
import socket
import threading

import numpy as np
import pytest

import fluxo_b200 as fb
from fluxo_b200 import _lib
from fluxo_b200.shard import ShardedOperator, ThreadExchange

pytestmark = pytest.mark.gpu


def run_threads(n, fn, timeout=600):
    errs = [None] * n

    def work(i):
        try:
            fn(i)
        except Exception as ex:  # re-raised in the test thread
            errs[i] = ex

    th = [threading.Thread(target=work, args=(i,)) for i in range(n)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout)
    assert not any(t.is_alive() for t in th), "a rank did not finish"
    for e in errs:
        if e is not None:
            raise e


MHD_FIELDS = dict(eqn=3, riemann=14, volume_flux=10, kappa=5 / 3, mu0=0.005, eta=0.01, lifting=1, lifting_var=3,
                  noncons=1, glm_scale=0.5)


def setup(n_ranks, ne=(4, 3, 3), N=3, mhd=False, **kw):
    fields = dict(N=N, eqn=1, riemann=44, volume_flux=5, lifting=1, lifting_var=3, mu0=0.01, kappa=1.4,
                  cfl_scale=0.6, dfl_scale=0.5, time_disc=0, ini_exact_func=1)
    if mhd:
        fields.update(MHD_FIELDS)
    fields.update(kw)
    mesh = fb.box_mesh(N, ne, (-1, -1, -1), (1, 1, 1), NGeo=2, deform_amp=0.1)
    if mhd:
        from fluxo_b200.workloads import mhd_orszag_tang_state

        U0 = mhd_orszag_tang_state(mesh["Elem_xGP"], kappa=5 / 3)
    else:
        U0 = fb.exact_func(2, 0.0, mesh["Elem_xGP"], adv_vel=(0.3, -0.2, 0.5), amplitude=0.3)
    U0 = U0 * (1 + 0.02 * np.random.default_rng(3).standard_normal(U0.shape))
    ref = fb.DGOperator(**fields)
    ref.set_mesh(mesh)
    ref.set_state(U0)
    hub = ThreadExchange(n_ranks)
    shards = [None] * n_ranks

    def make(r):  # MHD: set_partition reduces GLM_dtch1 over the ranks, so the ranks build together
        shards[r] = ShardedOperator(mesh, n_ranks, r, hub.rank, **fields)
        shards[r].set_state(U0)

    run_threads(n_ranks, make)
    return ref, shards, U0


def gather(shards, what):
    return np.concatenate([getattr(s, what)() for s in shards])


CASES = [dict(n=2), dict(n=3), dict(n=2, eqn=0), dict(n=4, lifting=2, lifting_var=2), dict(n=3, riemann=1, volume_flux=10),
         dict(n=2, N=7, ne=(3, 2, 2)), dict(n=5, N=2, ne=(5, 2, 2), time_disc=8),
         dict(n=2, mhd=True), dict(n=3, mhd=True, N=4, lifting=2), dict(n=2, mhd=True, eqn=2, riemann=10),
         dict(n=3, nfvse=1, compute_alpha=1, space_prop_sweeps=2, alpha_min=1e-4, riemann=44, sub_fv_method=2,
              recons_boundaries=3),
         dict(n=2, nfvse=1, compute_alpha=3, shock_blend_coef=0.4, sub_fv_method=4, recons_boundaries=3, eqn=0),
         dict(n=2, mhd=True, N=4, nfvse=1, compute_alpha=1, space_prop_sweeps=1, alpha_min=1e-4),
         dict(n=3, nfvse=1, compute_alpha=3, shock_blend_coef=0.3, nfvse_corr=1, time_disc=8, eqn=0)]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "_".join("%s%s" % kv for kv in c.items()))
def test_partitioned_rhs_and_steps_match_one_handle(gpu_lib, case):
    case = dict(case)
    n = case.pop("n")
    ref, shards, U0 = setup(n, **case)
    ref.dg_time_derivative(0.0)
    Ut = ref.get_ut()
    run_threads(n, lambda i: shards[i].op.dg_time_derivative(0.0))
    Uts = gather(shards, "get_ut")
    assert np.abs(Uts - Ut).max() <= 1e-15 * np.abs(Ut).max(), np.abs(Uts - Ut).max()
    if case.get("nfvse"):  # the blending coefficients after the propagation sweeps over the partition sides
        a_ref = ref.alpha()
        a_sh = np.concatenate([s.op.alpha()[: s.part.n_owned] for s in shards])
        assert (a_ref > 0).any() and np.array_equal(a_sh, a_ref)
    # CALCTIMESTEP with the dt reduction, then device-resident steps of the TimeDisc loop
    dt_ref, _ = ref.calc_timestep()
    dts = [None] * n
    run_threads(n, lambda i: dts.__setitem__(i, shards[i].op.calc_timestep()))
    assert all(d[0] == dt_ref and d[1] == 0 for d in dts)
    if case.get("mhd"):
        assert all(s.op.glm_ch == ref.glm_ch for s in shards)
    t_ref, n_ref, e_ref = ref.time_disc(0.0, 1e30, 12)
    res = [None] * n
    run_threads(n, lambda i: res.__setitem__(i, shards[i].op.time_disc(0.0, 1e30, 12)))
    assert e_ref == 0 and n_ref == 12
    assert all(r == (t_ref, n_ref, e_ref) for r in res), (t_ref, n_ref, res)
    U = ref.get_state()
    Us = gather(shards, "get_state")
    assert np.abs(Us - U).max() <= 1e-14 * np.abs(U).max()
    for s in shards:
        s.close()


def test_partition_restrictions(gpu_lib):
    mesh = fb.box_mesh(3, (2, 2, 2), (-1, -1, -1), (1, 1, 1), node_type=1)
    op = fb.DGOperator(N=3, eqn=0, riemann=44, volume_flux=5, node_type=1)
    op.set_mesh(mesh)
    with pytest.raises(fb.FluxoError):
        _lib.check(op.lib.fluxo_gpu_set_partition(op.h, 4, _lib.EXCHANGE_FN(lambda *a: 0), None), op.h)


def _nccl_rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    from fluxo_b200.shard import DistExchange

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    import datetime

    dist.init_process_group("nccl", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ref, _, U0 = setup(1, ne=(3, 2, 2))
        mesh = fb.box_mesh(3, (3, 2, 2), (-1, -1, -1), (1, 1, 1), NGeo=2, deform_amp=0.1)
        sh = ShardedOperator(mesh, world, rank, DistExchange, N=3, eqn=1, riemann=44, volume_flux=5, lifting=1,
                             lifting_var=3, mu0=0.01, kappa=1.4, cfl_scale=0.6, dfl_scale=0.5, time_disc=0,
                             ini_exact_func=1)
        sh.set_state(U0)
        t1, n1, e1 = sh.op.time_disc(0.0, 1e30, 5)
        t0, n0, e0 = ref.time_disc(0.0, 1e30, 5)
        out[rank] = (t1 == t0 and n1 == n0 and e1 == e0 == 0, float(np.abs(sh.get_state() - ref.get_state()).max()))
        sh.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_nccl_exchange_path_one_rank(gpu_lib):
    """The torch.distributed transport under NCCL through the library's callback (one rank on one GPU: the
    dt all-reduce and an empty halo); several GPUs are not available to these tests."""
    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_nccl_rank, args=(1, port, out), nprocs=1, join=True)
        ok, diff = out[0]
    assert ok and diff == 0.0
