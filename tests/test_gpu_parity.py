"""Parity of the sm_100a path against the CPU oracle, through the C ABI (the drop-in boundary).

The oracle builds the mesh arrays exactly as the reference's InitMesh would hand them to the
host; they go to the GPU through fluxo_gpu_set_mesh, and Ut, gradients, dt and time-stepped
states are compared.  Tolerance: relative L2 of Ut <= 1e-12 (FP64, different summation order
and fused multiply-adds on the GPU)."""
import numpy as np
import pytest

import fluxo_b200 as fb
from oracle.oracle import OracleCase

pytestmark = pytest.mark.gpu
TOL = 1e-12


def rel_l2(a, b):
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)


def pair(perturb=0.05, seed=0, **kw):
    """An oracle case and a GPU operator on the oracle's mesh and (perturbed) state."""
    c = OracleCase(**kw)
    if perturb:
        U = c.get_U()
        rng = np.random.default_rng(seed)
        c.set_U(U * (1 + perturb * rng.standard_normal(U.shape)))
    p = c.params
    op = fb.DGOperator(N=p.N, eqn=p.eqn, riemann=p.riemann, volume_flux=p.volume_flux, lifting=p.lifting,
                       lifting_var=p.lifting_var, visc=p.visc, kappa=p.kappa, R=p.R, Pr=p.Pr, mu0=p.mu0, Ts=p.Ts,
                       Tref=p.Tref, ExpoSuth=p.ExpoSuth, ExpoPow=p.ExpoPow, etaBR2=p.etaBR2,
                       time_disc=p.time_disc, cfl_scale=p.cfl_scale, dfl_scale=p.dfl_scale,
                       ini_exact_func=p.ini_exact_func, ini_frequency=p.ini_frequency,
                       ini_amplitude=p.ini_amplitude)
    op.set_mesh(c.mesh())
    op.set_state(c.get_U())
    return c, op


CUBE = dict(xmin=(-1, -1, -1), xmax=(1, 1, 1))
EULER_CASES = [
    dict(N=3, nElems=(4, 3, 2), NGeo=1, deform_amp=0.0, riemann=1, volume_flux=10),
    dict(N=3, nElems=(3, 3, 3), NGeo=2, deform_amp=0.1, riemann=1, volume_flux=5),
    dict(N=2, nElems=(3, 2, 2), NGeo=2, deform_amp=0.1, riemann=44, volume_flux=5),
    dict(N=4, nElems=(2, 2, 2), NGeo=3, deform_amp=0.1, riemann=4, volume_flux=10),
    dict(N=5, nElems=(2, 2, 2), NGeo=2, deform_amp=0.1, riemann=33, volume_flux=32),
    dict(N=1, nElems=(3, 3, 3), NGeo=1, deform_amp=0.1, riemann=22, volume_flux=0),
    dict(N=6, nElems=(2, 2, 1), NGeo=2, deform_amp=0.1, riemann=0, volume_flux=1),
    dict(N=7, nElems=(2, 1, 2), NGeo=2, deform_amp=0.1, riemann=5, volume_flux=2),
    dict(N=7, nElems=(1, 2, 1), NGeo=2, deform_amp=0.1, riemann=9, volume_flux=5),
    dict(N=3, nElems=(2, 2, 2), NGeo=2, deform_amp=0.1, riemann=13, volume_flux=10),
    dict(N=3, nElems=(2, 2, 2), NGeo=2, deform_amp=0.1, riemann=14, volume_flux=2),
    dict(N=3, nElems=(2, 2, 2), NGeo=2, deform_amp=0.1, riemann=16, volume_flux=5),
    dict(N=3, nElems=(2, 2, 2), NGeo=2, deform_amp=0.1, riemann=32, volume_flux=32),
    dict(N=3, nElems=(2, 2, 2), NGeo=2, deform_amp=0.1, riemann=6, volume_flux=2),
]


@pytest.mark.parametrize("case", EULER_CASES, ids=lambda c: "N%d_rs%d_vf%d" % (c["N"], c["riemann"], c["volume_flux"]))
def test_euler_ut_parity(gpu_lib, case):
    c, op = pair(ini_exact_func=2, ini_amplitude=0.3, adv_vel=(0.3, -0.2, 0.5), **CUBE, **case)
    ref = c.dg_time_derivative(0.3)
    op.dg_time_derivative(0.3)
    assert rel_l2(op.get_ut(), ref) <= TOL


# every remaining Riemann solver and volume flux of navierstokes/equation.f90:291-466 (Roe with each
# of its baseline fluxes; the point-flux and LLF variants with their own volume flux)
OPTION_CASES = [
    dict(N=3, riemann=2, volume_flux=3), dict(N=4, riemann=23, volume_flux=4), dict(N=2, riemann=24, volume_flux=6),
    dict(N=3, riemann=3, volume_flux=0), dict(N=3, riemann=3, volume_flux=2), dict(N=5, riemann=3, volume_flux=3),
    dict(N=3, riemann=3, volume_flux=4), dict(N=3, riemann=7, volume_flux=3), dict(N=6, riemann=8, volume_flux=4),
    dict(N=3, riemann=10, volume_flux=6), dict(N=4, riemann=11, volume_flux=7), dict(N=3, riemann=12, volume_flux=8),
    dict(N=7, riemann=20, volume_flux=9), dict(N=3, riemann=15, volume_flux=3), dict(N=3, riemann=17, volume_flux=7),
    dict(N=6, riemann=18, volume_flux=8), dict(N=3, riemann=19, volume_flux=4), dict(N=1, riemann=21, volume_flux=9),
]


@pytest.mark.parametrize("case", OPTION_CASES, ids=lambda c: "N%d_rs%d_vf%d" % (c["N"], c["riemann"], c["volume_flux"]))
def test_every_riemann_and_volume_flux(gpu_lib, case):
    c, op = pair(ini_exact_func=2, ini_amplitude=0.3, adv_vel=(0.3, -0.2, 0.5), nElems=(2, 2, 2), NGeo=2,
                 deform_amp=0.1, **CUBE, **case)
    ref = c.dg_time_derivative(0.1)
    op.dg_time_derivative(0.1)
    assert rel_l2(op.get_ut(), ref) <= TOL


NS_CASES = [
    dict(N=3, lifting=1, lifting_var=3, visc=0, riemann=44, volume_flux=5),
    dict(N=4, lifting=1, lifting_var=3, visc=0, riemann=17, volume_flux=7),
    dict(N=3, lifting=2, lifting_var=1, visc=0, riemann=3, volume_flux=3),
    dict(N=4, lifting=1, lifting_var=1, visc=0, riemann=1, volume_flux=10),
    dict(N=2, lifting=1, lifting_var=2, visc=1, riemann=22, volume_flux=2),
    dict(N=5, lifting=2, lifting_var=3, visc=0, riemann=4, volume_flux=32),
    dict(N=3, lifting=2, lifting_var=1, visc=2, riemann=1, volume_flux=5),
    dict(N=7, lifting=1, lifting_var=3, visc=0, riemann=44, volume_flux=5),
    dict(N=7, lifting=2, lifting_var=3, visc=0, riemann=44, volume_flux=5),
    dict(N=6, lifting=2, lifting_var=2, visc=1, riemann=1, volume_flux=5),
]


@pytest.mark.parametrize("case", NS_CASES,
                         ids=lambda c: "N%d_br%d_lv%d_visc%d_rs%d" % (c["N"], c["lifting"], c["lifting_var"], c["visc"],
                                                                     c["riemann"]))
def test_navier_stokes_parity(gpu_lib, case):
    extra = dict(R=1.0, Tref=1.0, Ts=0.4, ExpoPow=0.7) if case["visc"] else {}
    c, op = pair(eqn=1, mu0=0.02, ini_exact_func=7, nElems=(2, 3, 2), NGeo=2, deform_amp=0.05,
                 xmin=(-np.pi,) * 3, xmax=(np.pi,) * 3, **extra, **case)
    ref = c.dg_time_derivative(0.0)
    op.dg_time_derivative(0.0)
    assert rel_l2(op.get_ut(), ref) <= TOL
    gref = c.gradients()
    for g, r in zip(op.get_gradients(), gref):
        assert rel_l2(g, r) <= TOL


def test_source_term_parity(gpu_lib):
    c, op = pair(perturb=0.0, N=3, nElems=(2, 2, 2), ini_exact_func=4, ini_amplitude=0.1, ini_frequency=1.0,
                 riemann=1, volume_flux=10, **CUBE)
    m = c.mesh()
    op.set_mesh(m)
    op.set_state(c.get_U())
    ref = c.dg_time_derivative(0.37)
    op.dg_time_derivative(0.37)
    assert rel_l2(op.get_ut(), ref) <= TOL


@pytest.mark.parametrize("eqn", [0, 1])
def test_calc_timestep_parity(gpu_lib, eqn):
    c, op = pair(eqn=eqn, mu0=0.05, N=4, nElems=(3, 2, 2), NGeo=2, deform_amp=0.1, ini_exact_func=2,
                 riemann=1, volume_flux=5, **CUBE)
    dref, eref = c.calc_timestep()
    d, e = op.calc_timestep()
    assert e == eref == 0
    assert abs(d - dref) <= 1e-13 * dref
    U = c.get_U()
    U[2, 1, 0, 1, 4] = -1.0
    U[5, 0, 0, 0, 0] = np.nan
    c.set_U(U)
    op.set_state(U)
    assert op.calc_timestep()[1] == c.calc_timestep()[1] == 2


@pytest.mark.parametrize("eqn,td", [(0, 0), (1, 0), (0, 1)])
def test_timestep_parity(gpu_lib, eqn, td):
    c, op = pair(eqn=eqn, mu0=0.01, time_disc=td, N=3, nElems=(3, 2, 2), NGeo=2, deform_amp=0.1,
                 ini_exact_func=2, riemann=44, volume_flux=5, **CUBE)
    dt, _ = c.calc_timestep()
    c.timestep(0.1, dt)
    op.timestep(0.1, dt)
    assert rel_l2(op.get_state(), c.get_U()) <= TOL


def test_time_disc_parity(gpu_lib):
    """Device-resident TimeDisc loop vs the oracle's loop: same step count, same final state."""
    c, op = pair(perturb=0.0, N=3, nElems=(4, 4, 4), xmin=(0, 0, 0), xmax=(2, 2, 2), ini_exact_func=2,
                 riemann=1, volume_flux=10)
    t_ref, n_ref = c.run(0.0, 0.05)
    t, n, err = op.time_disc(0.0, 0.05)
    assert err == 0 and n == n_ref and abs(t - t_ref) < 1e-15
    assert rel_l2(op.get_state(), c.get_U()) <= 1e-12


def test_config1_full_run(gpu_lib):
    """Euler density wave on [0,2]^3, 8^3, N=3, EC volume flux + LLF, LSERK4-5 CFL 0.9, 200 steps:
    the final L2 errors of the GPU run match the oracle's to 3 significant digits."""
    kw = dict(N=3, nElems=(8, 8, 8), xmin=(0, 0, 0), xmax=(2, 2, 2), ini_exact_func=2, riemann=1, volume_flux=10)
    c, op = pair(perturb=0.0, **kw)
    t_ref, n_ref = c.run(0.0, 100.0, max_iter=200)
    t, n, err = op.time_disc(0.0, 100.0, 200)
    assert n == n_ref == 200 and err == 0
    c2 = OracleCase(**kw)
    c2.set_U(op.get_state())
    e_gpu = c2.analyze(t)["L2"]
    e_ref = c.analyze(t_ref)["L2"]
    assert np.allclose(e_gpu, e_ref, rtol=1e-3, atol=1e-14)
    assert rel_l2(op.get_state(), c.get_U()) <= 1e-11


def test_product_setup_path(gpu_lib):
    """Fluxo() builds its own mesh and initial state (no oracle data) and matches the oracle."""
    ini = """
    N = 3
    BoxElems = (/3,2,2/)
    BoxMin = (/-1.,-1.,-1./)
    BoxMax = (/1.,1.,1./)
    NGeo = 2
    MeshDeformAmp = 0.1
    Riemann = 44
    VolumeFlux = 5
    Parabolic = T
    mu0 = 0.01
    IniExactFunc = 2
    IniAmplitude = 0.2
    AdvVel = (/0.3,-0.2,0.5/)
    CFLScale = 0.9
    DFLScale = 0.4
    """
    f = fb.Fluxo(ini)
    f.DGTimeDerivative(0.0)
    c = OracleCase(N=3, nElems=(3, 2, 2), NGeo=2, deform_amp=0.1, eqn=1, mu0=0.01, riemann=44, volume_flux=5,
                   ini_exact_func=2, ini_amplitude=0.2, adv_vel=(0.3, -0.2, 0.5), **CUBE)
    ref = c.dg_time_derivative(0.0)
    assert rel_l2(f.Ut, ref) <= 1e-11


def test_deterministic_reruns(gpu_lib):
    """Same input, same launch sequence: bitwise-identical Ut (no races, no atomics in the RHS)."""
    c, op = pair(eqn=1, mu0=0.01, N=4, nElems=(3, 3, 2), NGeo=2, deform_amp=0.1, ini_exact_func=2,
                 riemann=44, volume_flux=5, **CUBE)
    op.dg_time_derivative(0.0)
    a = op.get_ut()
    op.dg_time_derivative(0.0)
    assert np.array_equal(a, op.get_ut())
