"""Parity of the configurations used by the batched / served mixes (EC-KEP volume flux + Riemann 44,
Euler and Navier-Stokes BR1, N = 3..7) with the mixes' random-Fourier data: one RHS at every N, and
whole TimeDisc runs of served requests against the oracle's loop."""
import numpy as np
import pytest

import fluxo_b200 as fb
from fluxo_b200.workloads import BOX_MAX, BOX_MIN, fourier_state, instance_fields, serve_request_specs
from oracle.oracle import OracleCase

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)


def case(N, eqn, elems, seed):
    f = instance_fields(dict(N=N, eqn=eqn))
    c = OracleCase(nElems=(elems,) * 3, xmin=BOX_MIN, xmax=BOX_MAX, NGeo=1, deform_amp=0.0, **f)
    c.set_U(fourier_state(c.mesh()["Elem_xGP"], BOX_MIN, BOX_MAX, np.random.default_rng(seed)))
    op = fb.DGOperator(cfg=fb.make_cfg(**f))
    op.set_mesh(c.mesh())
    op.set_state(c.get_U())
    return c, op


@pytest.mark.parametrize("eqn", [0, 1])
@pytest.mark.parametrize("N", [3, 4, 5, 6, 7])
def test_mix_rhs_parity(gpu_lib, N, eqn):
    c, op = case(N, eqn, 3, seed=100 + N)
    ref = c.dg_time_derivative(0.0)
    op.dg_time_derivative(0.0)
    assert rel_l2(op.get_ut(), ref) <= 1e-12


@pytest.mark.parametrize("rid", [54, 40, 62])
def test_served_request_full_run_parity(gpu_lib, rid):
    """Requests of the served stream (rate 20/s, 3 s) on their own meshes, run to their end times."""
    s = serve_request_specs(20.0, 3.0)[rid]
    c, op = case(s["N"], s["eqn"], s["elems"], s["seed"])
    # 25 steps: same states to roundoff growth
    t_ref, n_ref = c.run(0.0, 1e30, max_iter=25)
    t, n, err = op.time_disc(0.0, 1e30, 25)
    assert err == 0 and n == n_ref == 25 and abs(t - t_ref) <= 1e-13 * t_ref
    assert rel_l2(op.get_state(), c.get_U()) <= 1e-10
    # on to the end time: both finish without a CALCTIMESTEP error; the last step's clipping rule
    # (timedisc.f90:306-317) may fall one step apart when dt agrees only to roundoff
    t_ref, n_ref = c.run(t_ref, s["t_end"])
    t, n, err = op.time_disc(t, s["t_end"])
    assert err == 0 and c.calc_timestep()[1] == 0 and abs(n - n_ref) <= 1
    assert t == s["t_end"] or abs(t - s["t_end"]) <= 1e-12
