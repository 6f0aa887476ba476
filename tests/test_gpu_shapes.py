"""Launch shapes of the volume kernel (vol_shapes.h): every candidate of an N matches the oracle and
the other candidates to roundoff (the shapes are separate instantiations whose multiply-add fusion
may differ), the autotuner picks one of them, and a process keeps using it (same bits on re-use)."""
import numpy as np
import pytest

import fluxo_b200 as fb
from fluxo_b200.solver import set_volume_shape, volume_shape
from oracle.oracle import OracleCase

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("vf", [5, 10])
@pytest.mark.parametrize("eqn", [0, 1])
@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
def test_every_shape_same_bits(gpu_lib, N, eqn, vf):
    kw = dict(N=N, nElems=(3, 2, 2), NGeo=2, deform_amp=0.1, ini_exact_func=2, riemann=44, volume_flux=vf,
              xmin=(-1, -1, -1), xmax=(1, 1, 1), eqn=eqn, mu0=0.01 if eqn else 0.0, lifting=1, lifting_var=3)
    c = OracleCase(**kw)
    U = c.get_U() * (1 + 0.05 * np.random.default_rng(N).standard_normal(c.get_U().shape))
    c.set_U(U)
    ref = c.dg_time_derivative(0.0)
    p = c.params
    op = fb.DGOperator(N=N, eqn=eqn, riemann=44, volume_flux=vf, lifting=1, lifting_var=3, mu0=p.mu0, kappa=p.kappa,
                       R=p.R, Pr=p.Pr, ini_exact_func=2)
    op.set_mesh(c.mesh())
    op.set_state(U)
    count = volume_shape(N, vf, eqn == 1)[0]
    assert count >= 1
    outs = []
    for i in range(count):
        set_volume_shape(N, vf, eqn == 1, i)
        assert volume_shape(N, vf, eqn == 1)[1] == i
        op.dg_time_derivative(0.0)
        outs.append(op.get_ut())
    for o in outs:
        assert np.linalg.norm(o - ref) / np.linalg.norm(ref) <= 1e-12
        assert np.linalg.norm(o - outs[0]) / np.linalg.norm(outs[0]) <= 1e-14
    set_volume_shape(N, vf, eqn == 1, -1)   # the next RHS tunes again
    op.dg_time_derivative(0.0)
    cnt, chosen, epb, lpw = volume_shape(N, vf, eqn == 1)
    assert 0 <= chosen < cnt and epb >= 1
    assert np.array_equal(op.get_ut(), outs[chosen])
    op.dg_time_derivative(0.0)             # the tuned shape stays: same bits
    assert np.array_equal(op.get_ut(), outs[chosen])
    op.close()
