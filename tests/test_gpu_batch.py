"""Batched solves (``fluxo_batch_*``): every instance of a mix ends bit-identical to its solo run.

A batch concatenates instances of the same kernel configuration into one launch per kernel and
gives each instance its own CALCTIMESTEP minimum and end time, so an instance's arithmetic is the
same alone and in the mix: the tests require identical bits (same step count, same final time,
same state) against ``DGOperator.time_disc`` of the same instance, and the solo path itself is
pinned to the oracle (relative L2 <= 1e-12, checked here once more through the batch).
"""
import numpy as np
import pytest

import fluxo_b200 as fb
from fluxo_b200.batch import Batch, instance_bytes
from fluxo_b200.workloads import fourier_state
from oracle.oracle import OracleCase

pytestmark = pytest.mark.gpu

BOX = dict(xmin=(0.0, 0.0, 0.0), xmax=(2.0, 2.0, 2.0))


def instance(seed, N, elems, eqn, t_end, riemann=1, volume_flux=10, deform=0.0, max_iter=-1, **cfg):
    mesh = fb.box_mesh(N, elems, BOX["xmin"], BOX["xmax"], NGeo=2 if deform else 1, deform_amp=deform)
    U = fourier_state(mesh["Elem_xGP"], BOX["xmin"], BOX["xmax"], np.random.default_rng(seed))
    kw = dict(N=N, eqn=eqn, riemann=riemann, volume_flux=volume_flux, ini_exact_func=0)
    if eqn == 1:
        kw.update(mu0=0.002, lifting=1, lifting_var=2)
    kw.update(cfg)
    return dict(mesh=mesh, U=U, t_end=t_end, max_iter=max_iter, cfg=fb.make_cfg(**kw))


def solo(inst):
    op = fb.DGOperator(cfg=inst["cfg"])
    op.set_mesh(inst["mesh"])
    op.set_state(inst["U"])
    t, n, err = op.time_disc(0.0, inst["t_end"], inst["max_iter"])
    U = op.get_state()
    op.close()
    return t, n, err, U


MIX = [  # CALCTIMESTEP of the initial states: dt = 0.050, 0.067, 0.048, 0.145, 0.100, 0.029, 0.050
    dict(seed=1, N=3, elems=(4, 4, 4), eqn=0, t_end=0.6),
    dict(seed=2, N=3, elems=(3, 3, 3), eqn=0, t_end=0.9),                        # same group as seed 1
    dict(seed=3, N=4, elems=(2, 3, 2), eqn=1, t_end=0.5, deform=0.05),
    dict(seed=4, N=2, elems=(3, 2, 2), eqn=0, t_end=1.5, riemann=44, volume_flux=5),
    dict(seed=5, N=3, elems=(2, 2, 2), eqn=1, t_end=1.2, lifting=2, lifting_var=3),
    dict(seed=6, N=5, elems=(2, 2, 2), eqn=0, t_end=0.35, time_disc=1),
    dict(seed=7, N=3, elems=(4, 4, 4), eqn=0, t_end=2.0, max_iter=7),              # stops on max_iter
]


def test_mix_matches_solo_runs(gpu_lib):
    insts = [instance(**m) for m in MIX]
    ref = [solo(i) for i in insts]
    b = Batch()
    ids = [b.add(i["mesh"], i["U"], 0.0, i["t_end"], cfg=i["cfg"], max_iter=i["max_iter"]) for i in insts]
    b.run_to_end()
    groups, placed, nbytes = b.info()
    assert groups == 5 and placed == len(MIX)
    assert nbytes == sum(instance_bytes(i["cfg"], i["mesh"]["ElemToSide"].shape[0],
                                        i["mesh"]["SideToElem"].shape[0]) for i in insts)
    for iid, (t, n, err, U) in zip(ids, ref):
        tb, nb, done, errb = b.status(iid)
        assert done and errb == err == 0
        assert nb == n and tb == t
        assert np.array_equal(b.get_state(iid), U)
    b.close()


def test_joining_and_leaving_mid_run(gpu_lib):
    """Instances added while others run (the group arrays are rebuilt and the state moved on the
    device) and removed after finishing: every result still equals its solo run."""
    insts = [instance(**dict(m, t_end=2 * m["t_end"])) for m in MIX[:4]]
    ref = [solo(i) for i in insts]
    assert min(r[1] for r in ref) > 10
    b = Batch()
    ids = [b.add(i["mesh"], i["U"], 0.0, i["t_end"], cfg=i["cfg"]) for i in insts[:2]]
    assert b.run(3) == 2
    ids.append(b.add(insts[2]["mesh"], insts[2]["U"], 0.0, insts[2]["t_end"], cfg=insts[2]["cfg"]))
    b.run(5)
    ids.append(b.add(insts[3]["mesh"], insts[3]["U"], 0.0, insts[3]["t_end"], cfg=insts[3]["cfg"]))
    while b.run(4):
        for k, iid in enumerate(ids[:2]):
            if iid is not None and b.status(iid)[2]:
                assert np.array_equal(b.get_state(iid), ref[k][3])
                b.remove(iid)
                ids[k] = None
    for iid, (t, n, err, U) in zip(ids, ref):
        if iid is None:
            continue
        tb, nb, done, errb = b.status(iid)
        assert done and nb == n and tb == t
        assert np.array_equal(b.get_state(iid), U)
    b.close()


def test_bad_instance_stops_alone(gpu_lib):
    """A state with p <= 0 stops its own instance with errType 2 (as CALCTIMESTEP reports it);
    the other instances of the same group finish unchanged."""
    good = instance(seed=11, N=3, elems=(3, 3, 3), eqn=0, t_end=0.5)
    bad = instance(seed=12, N=3, elems=(3, 3, 3), eqn=0, t_end=0.5)
    bad["U"][4, 1, 1, 1, 4] = -1.0
    t, n, err, U = solo(good)
    b = Batch()
    ig = b.add(good["mesh"], good["U"], 0.0, 0.5, cfg=good["cfg"])
    ib = b.add(bad["mesh"], bad["U"], 0.0, 0.5, cfg=bad["cfg"])
    b.run_to_end()
    assert b.status(ib)[2:] == (True, 2) and b.status(ib)[1] == 0
    assert b.status(ig) == (t, n, True, 0)
    assert np.array_equal(b.get_state(ig), U)
    b.close()


def test_batch_against_oracle(gpu_lib):
    """One instance of a mix against the oracle's TimeDisc loop (relative L2 <= 1e-12)."""
    kw = dict(N=3, nElems=(3, 3, 3), NGeo=2, deform_amp=0.1, ini_exact_func=2, riemann=1, volume_flux=10,
              xmin=(0, 0, 0), xmax=(2, 2, 2))
    c = OracleCase(**kw)
    U0 = c.get_U()
    other = instance(seed=21, N=3, elems=(2, 2, 2), eqn=0, t_end=0.5)
    b = Batch()
    b.add(other["mesh"], other["U"], 0.0, 0.5, cfg=other["cfg"])
    p = c.params
    cfg = fb.make_cfg(N=p.N, eqn=p.eqn, riemann=p.riemann, volume_flux=p.volume_flux, kappa=p.kappa, R=p.R,
                      time_disc=p.time_disc, cfl_scale=p.cfl_scale, dfl_scale=p.dfl_scale, ini_exact_func=2)
    iid = b.add(c.mesh(), U0, 0.0, 0.3, cfg=cfg)
    b.run_to_end()
    t_ref, n_ref = c.run(0.0, 0.3)
    t, n, done, err = b.status(iid)
    assert done and err == 0 and n == n_ref > 5 and abs(t - t_ref) < 1e-15
    Ub, Uo = b.get_state(iid), c.get_U()
    assert np.linalg.norm(Ub - Uo) / np.linalg.norm(Uo) <= 1e-12
    b.close()


def test_rejects_unsupported_instances(gpu_lib):
    b = Batch()
    m = instance(seed=1, N=3, elems=(2, 2, 2), eqn=0, t_end=0.1)
    with pytest.raises(fb.FluxoError):
        b.add(m["mesh"], m["U"], 0.0, 0.1, N=3, eqn=2)
    with pytest.raises(fb.FluxoError):
        b.add(m["mesh"], m["U"], 0.0, 0.1, N=3, ini_exact_func=4)
    b.close()
