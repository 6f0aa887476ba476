"""Parity of the sm_100a MHD + GLM path against the CPU oracle, through the C ABI.

Ideal and resistive MHD on curved periodic boxes: Ut of one DGTimeDerivative (with the
non-conservative Powell / Brackbill / Janhunen terms and the GLM terms), the BR1/BR2 gradients,
CALCTIMESTEP with the GLM speed, one LSERK step and the device-resident TimeDisc loop.
Tolerance: relative L2 <= 1e-12 (FP64, different summation order and fused multiply-adds)."""
import numpy as np
import pytest

import fluxo_b200 as fb
from oracle.oracle import OracleCase

pytestmark = pytest.mark.gpu
TOL = 1e-12
REF = ((1.2, 0.1, 0.0, 0.1, 0.9, 1.0, 1.0, 1.0), (1.1, 0.2, -0.1, 0.2, 0.6, 1.0, 1.0, 1.0))


def rel_l2(a, b):
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)


def mhd_pair(seed=0, ch=0.7, noise=0.02, **kw):
    """An oracle case (soft blast with node noise and a psi field) and a GPU operator on the same
    mesh, state and GLM speed."""
    base = dict(eqn=2, N=3, nElems=(3, 2, 2), xmin=(-1, -1, -1), xmax=(1, 1, 1), NGeo=2, deform_amp=0.1,
                kappa=5 / 3, mhd_ref_state=REF, ini_exact_func=201, ini_center=(0, 0, 0), ini_halfwidth=0.4,
                ini_amplitude=0.1, glm_ch=ch)
    base.update(kw)
    c = OracleCase(**base)
    rng = np.random.default_rng(seed)
    U = c.get_U()
    U = U * (1 + noise * rng.standard_normal(U.shape))
    U[..., 8] = 0.05 * rng.standard_normal(U[..., 8].shape)
    c.set_U(U)
    p = c.params
    op = fb.DGOperator(N=p.N, eqn=p.eqn, riemann=p.riemann, volume_flux=p.volume_flux, lifting=p.lifting,
                       lifting_var=p.lifting_var, kappa=p.kappa, Pr=p.Pr, mu0=p.mu0, etaBR2=p.etaBR2,
                       time_disc=p.time_disc, cfl_scale=p.cfl_scale, dfl_scale=p.dfl_scale,
                       ini_exact_func=1, mu_0=p.mu_0, eta=p.eta, glm_scale=p.glm_scale, glm_scr=p.glm_scr,
                       noncons=p.noncons, nc_glm=p.nc_glm)
    op.set_mesh(c.mesh())
    op.set_state(U)
    op.glm_ch = ch
    return c, op


IDEAL = [
    dict(N=3, volume_flux=10, riemann=14, noncons=1, nc_glm=0),
    dict(N=4, volume_flux=10, riemann=10, noncons=1, nc_glm=1),
    dict(N=2, volume_flux=12, riemann=15, noncons=1, nc_glm=1),
    dict(N=3, volume_flux=12, riemann=13, noncons=2, nc_glm=0),
    dict(N=3, volume_flux=0, riemann=1, noncons=3, nc_glm=0),
    dict(N=5, volume_flux=1, riemann=4, noncons=1, nc_glm=0),
    dict(N=1, volume_flux=10, riemann=11, noncons=1, nc_glm=1),
    dict(N=3, volume_flux=10, riemann=12, noncons=0, nc_glm=0),
    dict(N=7, volume_flux=10, riemann=14, noncons=1, nc_glm=0, nElems=(1, 2, 1)),
    dict(N=6, volume_flux=12, riemann=0, noncons=1, nc_glm=1, nElems=(2, 1, 1)),
    dict(N=3, volume_flux=10, riemann=2, noncons=1, nc_glm=1),
    dict(N=4, volume_flux=0, riemann=3, noncons=1, nc_glm=0),
    dict(N=3, volume_flux=12, riemann=5, noncons=2, nc_glm=0),
]


@pytest.mark.parametrize("case", IDEAL, ids=lambda c: "N%d_vf%d_rs%d_nc%d%s" % (
    c["N"], c["volume_flux"], c["riemann"], c["noncons"], "g" if c["nc_glm"] else ""))
def test_mhd_ideal_ut_parity(gpu_lib, case):
    c, op = mhd_pair(**case)
    ref = c.dg_time_derivative(0.0)
    op.dg_time_derivative(0.0)
    assert rel_l2(op.get_ut(), ref) <= TOL


PARA = [
    dict(N=3, lifting=1, lifting_var=3, volume_flux=10, riemann=14),
    dict(N=4, lifting=1, lifting_var=1, volume_flux=10, riemann=10),
    dict(N=3, lifting=2, lifting_var=2, volume_flux=12, riemann=1),
    dict(N=2, lifting=2, lifting_var=3, volume_flux=0, riemann=4),
    dict(N=3, lifting=1, lifting_var=3, volume_flux=10, riemann=5),
    dict(N=7, lifting=2, lifting_var=3, volume_flux=10, riemann=14),
]


@pytest.mark.parametrize("case", PARA, ids=lambda c: "N%d_br%d_lv%d_rs%d" % (c["N"], c["lifting"], c["lifting_var"],
                                                                           c["riemann"]))
def test_mhd_resistive_parity(gpu_lib, case):
    c, op = mhd_pair(eqn=3, eta=0.02, mu0=0.01, noncons=1, **case)
    ref = c.dg_time_derivative(0.0)
    op.dg_time_derivative(0.0)
    assert rel_l2(op.get_ut(), ref) <= TOL
    for g, r in zip(op.get_gradients(), c.gradients()):
        assert rel_l2(g, r) <= TOL


def test_mhd_glm_damping_parity(gpu_lib):
    c, op = mhd_pair(glm_scr=0.3, volume_flux=10, riemann=14)
    ref = c.dg_time_derivative(0.0)
    op.dg_time_derivative(0.0)
    assert rel_l2(op.get_ut(), ref) <= TOL


@pytest.mark.parametrize("eqn", [2, 3])
def test_mhd_calc_timestep_and_glm_speed(gpu_lib, eqn):
    c, op = mhd_pair(eqn=eqn, eta=0.02, N=4, volume_flux=10, riemann=14)
    dref, eref = c.calc_timestep()
    d, e = op.calc_timestep()
    assert e == eref == 0
    assert abs(d - dref) <= 1e-13 * dref
    assert op.glm_ch == pytest.approx(c.glm_ch, rel=1e-13)


@pytest.mark.parametrize("eqn", [2, 3])
def test_mhd_timestep_parity(gpu_lib, eqn):
    c, op = mhd_pair(eqn=eqn, eta=0.02, mu0=0.005, N=3, volume_flux=10, riemann=14, nc_glm=1)
    dt, _ = c.calc_timestep()
    op.calc_timestep()
    c.timestep(0.0, dt)
    op.timestep(0.0, dt)
    assert rel_l2(op.get_state(), c.get_U()) <= TOL


def test_mhd_time_disc_parity(gpu_lib):
    c, op = mhd_pair(N=3, volume_flux=10, riemann=14, noise=0.0)
    t_ref, n_ref = c.run(0.0, 1.0, max_iter=12)
    t, n, err = op.time_disc(0.0, 1.0, max_iter=12)
    assert err == 0 and n == n_ref == 12
    assert t == pytest.approx(t_ref, rel=1e-12)
    assert op.glm_ch == pytest.approx(c.glm_ch, rel=1e-12)
    assert rel_l2(op.get_state(), c.get_U()) <= 1e-11
