"""Parity of the sm_100a Gauss-node (PP_NodeType = 1) path against the CPU oracle through the C ABI:
interpolated / entropy-projected face states, the FluxB-corrected surface integral, the Gauss BR1 / BR2
lifting and viscous terms, the Gauss CFL / DFL scaling, and device-resident time steps.  Ut to relative
L2 <= 1e-12 (FP64, other summation orders), states after steps <= 1e-11."""
import numpy as np
import pytest

import fluxo_b200 as fb
from fluxo_b200._lib import FluxoError
from oracle.oracle import OracleCase

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)


def pair(noise=0.03, seed=2, **kw):
    base = dict(eqn=0, N=3, nElems=(3, 2, 2), xmin=(-1, -1, -1), xmax=(1, 1, 1), NGeo=2, deform_amp=0.1,
                ini_exact_func=2, ini_amplitude=0.3, adv_vel=(0.3, -0.2, 0.5), node_type=1)
    base.update(kw)
    c = OracleCase(**base)
    U = c.get_U()
    if noise:
        U = U * (1 + noise * np.random.default_rng(seed).standard_normal(U.shape))
        c.set_U(U)
    p = c.params
    op = fb.DGOperator(N=p.N, eqn=p.eqn, riemann=p.riemann, volume_flux=p.volume_flux, lifting=p.lifting,
                       lifting_var=p.lifting_var, visc=p.visc, kappa=p.kappa, Pr=p.Pr, mu0=p.mu0, etaBR2=p.etaBR2,
                       R=p.R, Ts=p.Ts, Tref=p.Tref, ExpoSuth=p.ExpoSuth, ExpoPow=p.ExpoPow,
                       time_disc=p.time_disc, cfl_scale=p.cfl_scale, dfl_scale=p.dfl_scale, ini_exact_func=1,
                       node_type=1)
    op.set_mesh(c.mesh())
    op.set_state(U)
    return c, op


EULER = [(N, vf, rs) for N, vf, rs in [
    (1, 5, 44), (2, 10, 4), (3, 5, 44), (3, 0, 1), (3, 1, 22), (3, 2, 2), (3, 32, 33), (4, 10, 5), (4, 5, 9),
    (5, 3, 1), (5, 4, 23), (6, 6, 44), (6, 7, 1), (7, 5, 44), (7, 8, 24), (7, 9, 3), (3, 5, 14)]]


@pytest.mark.parametrize("N,vf,rs", EULER, ids=lambda v: str(v))
def test_gauss_euler_parity(gpu_lib, N, vf, rs):
    kw = dict(nElems=(1, 2, 1)) if N == 7 else {}
    c, op = pair(N=N, volume_flux=vf, riemann=rs, **kw)
    ref = c.dg_time_derivative(0.0)
    op.dg_time_derivative(0.0)
    assert rel_l2(op.get_ut(), ref) <= 1e-12


NS = [dict(N=3, lifting=1, lifting_var=3), dict(N=3, lifting=1, lifting_var=1), dict(N=4, lifting=2, lifting_var=3),
      dict(N=2, lifting=2, lifting_var=2), dict(N=7, lifting=1, lifting_var=3, nElems=(1, 2, 1)),
      dict(N=5, lifting=1, lifting_var=2, visc=1), dict(N=4, lifting=2, lifting_var=1, visc=2, ExpoPow=0.7)]


@pytest.mark.parametrize("case", NS, ids=lambda c: "N%d_br%d_lv%d" % (c["N"], c["lifting"], c["lifting_var"]))
def test_gauss_navier_stokes_parity(gpu_lib, case):
    c, op = pair(eqn=1, volume_flux=5, riemann=44, mu0=0.02, **case)
    ref = c.dg_time_derivative(0.0)
    op.dg_time_derivative(0.0)
    assert rel_l2(op.get_ut(), ref) <= 1e-12
    gx, gy, gz = c.gradients()
    g = op.get_gradients()
    for a, b in zip(g, (gx, gy, gz)):
        assert rel_l2(a, b) <= 1e-12


def test_gauss_freestream_and_entropy_on_gpu(gpu_lib):
    """The reference's regression criteria, evaluated on GPU output: freestream on a warped NGeo=3 mesh
    (L_inf <= 1e-11) and entropy conservation with the EC fluxes and entropy-projected face states
    (|sum dS/dU . Ut| <= 1e-13, device-side analysis)."""
    c, op = pair(noise=0.0, ini_exact_func=1, ref_state=(1.1, 0.3, -0.2, 0.1, 0.8), volume_flux=5, riemann=44,
                 NGeo=3, nElems=(3, 3, 3))
    op.dg_time_derivative(0.0)
    assert np.abs(op.get_ut()).max() <= 1e-11
    c, op = pair(noise=0.05, volume_flux=5, riemann=9, NGeo=3, nElems=(3, 3, 3))
    a = op.analyze(0.0)
    assert abs(a["dSdU_Ut"]) <= 1e-13
    c, op = pair(noise=0.05, volume_flux=5, riemann=44, NGeo=3, nElems=(3, 3, 3))
    assert op.analyze(0.0)["dSdU_Ut"] < 0.


@pytest.mark.parametrize("time_disc,eqn", [(0, 0), (0, 1), (8, 0), (6, 1)])
def test_gauss_time_disc_parity(gpu_lib, time_disc, eqn):
    """Device-resident steps with the Gauss CFL / DFL scaling (timedisc_vars.f90 PP_NodeType = 1 tables)."""
    c, op = pair(eqn=eqn, volume_flux=5, riemann=44, mu0=0.01, time_disc=time_disc, noise=0.0)
    dt, err = c.calc_timestep()
    dtg, errg = op.calc_timestep()
    assert err == errg == 0 and dtg == pytest.approx(dt, rel=1e-12)
    t_ref, n_ref = c.run(0.0, 1.0, max_iter=5)
    t, n, err = op.time_disc(0.0, 1.0, max_iter=5)
    assert err == 0 and n == n_ref == 5 and t == pytest.approx(t_ref, rel=1e-12)
    assert rel_l2(op.get_state(), c.get_U()) <= 1e-11


def test_gauss_configuration_checks(gpu_lib):
    with pytest.raises(FluxoError):
        fb.DGOperator(N=3, eqn=0, riemann=44, volume_flux=5, nfvse=1, node_type=1)
    c, op = pair()
    m = c.mesh()
    del m["SurfMetrics"]
    op2 = fb.DGOperator(N=3, eqn=0, riemann=44, volume_flux=5, node_type=1)
    op2.set_mesh(m)
    op2.set_state(c.get_U())
    with pytest.raises(FluxoError):
        op2.dg_time_derivative(0.0)


def test_gauss_product_setup_path(gpu_lib):
    """Fluxo() from a parameter.ini with NodeType = GAUSS: the product's own Gauss box mesh (metrics at the
    Gauss nodes, SurfMetrics), initial state and operator, against the oracle."""
    ini = """
    N = 4
    NodeType = GAUSS
    BoxElems = (/3,2,2/)
    BoxMin = (/-1.,-1.,-1./)
    BoxMax = (/1.,1.,1./)
    NGeo = 2
    MeshDeformAmp = 0.1
    IniExactFunc = 2
    IniAmplitude = 0.3
    AdvVel = (/0.3,-0.2,0.5/)
    Riemann = 44
    VolumeFlux = 5
    mu0 = 0.01
    CFLScale = 0.5
    """
    f = fb.Fluxo(ini)
    f.DGTimeDerivative(0.0)
    c = OracleCase(eqn=1, N=4, nElems=(3, 2, 2), xmin=(-1, -1, -1), xmax=(1, 1, 1), NGeo=2, deform_amp=0.1,
                   ini_exact_func=2, ini_amplitude=0.3, adv_vel=(0.3, -0.2, 0.5), riemann=44, volume_flux=5,
                   mu0=0.01, cfl_scale=0.5, node_type=1)
    ref = c.dg_time_derivative(0.0)
    assert rel_l2(f.Ut, ref) <= 1e-11


# --- ideal MHD + GLM with Gauss nodes ---------------------------------------------------------------------------
MHD_REF = ((1.2, 0.1, 0.0, 0.1, 0.9, 1.0, 1.0, 1.0), (1.1, 0.2, -0.1, 0.2, 0.6, 1.0, 1.0, 1.0))


def mhd_pair(noise=0.01, seed=0, ch=0.7, **kw):
    base = dict(eqn=2, N=3, nElems=(3, 2, 2), xmin=(-1, -1, -1), xmax=(1, 1, 1), NGeo=2, deform_amp=0.1,
                kappa=5 / 3, mhd_ref_state=MHD_REF, ini_exact_func=201, ini_center=(0.1, 0.05, 0.0),
                ini_halfwidth=0.4, ini_amplitude=0.02, glm_ch=ch, node_type=1, volume_flux=10, riemann=11)
    base.update(kw)
    c = OracleCase(**base)
    U = c.get_U()
    if noise:
        rng = np.random.default_rng(seed)
        U = U * (1 + noise * rng.standard_normal(U.shape))
        U[..., 8] = 0.05 * rng.standard_normal(U[..., 8].shape)
        c.set_U(U)
    p = c.params
    op = fb.DGOperator(N=p.N, eqn=p.eqn, riemann=p.riemann, volume_flux=p.volume_flux, kappa=p.kappa, mu_0=p.mu_0,
                       glm_scale=p.glm_scale, glm_scr=p.glm_scr, noncons=p.noncons, nc_glm=p.nc_glm,
                       mu0=p.mu0, eta=p.eta, Pr=p.Pr, lifting=p.lifting, lifting_var=p.lifting_var, etaBR2=p.etaBR2,
                       time_disc=p.time_disc, cfl_scale=p.cfl_scale, dfl_scale=p.dfl_scale, ini_exact_func=1,
                       node_type=1)
    op.set_mesh(c.mesh())
    op.set_state(U)
    op.glm_ch = ch
    return c, op


MHD_CASES = [
    dict(N=1, volume_flux=10, riemann=11), dict(N=2, volume_flux=12, riemann=12), dict(N=3, volume_flux=10, riemann=11),
    dict(N=3, volume_flux=10, riemann=10, nc_glm=1), dict(N=3, volume_flux=1, riemann=1), dict(N=3, volume_flux=0, riemann=4),
    dict(N=3, volume_flux=12, riemann=15, noncons=2), dict(N=4, volume_flux=10, riemann=14, noncons=3),
    dict(N=4, volume_flux=10, riemann=5), dict(N=5, volume_flux=12, riemann=13), dict(N=6, volume_flux=10, riemann=2),
    dict(N=7, volume_flux=10, riemann=10, nElems=(2, 1, 1)), dict(N=7, volume_flux=1, riemann=3, nElems=(2, 1, 1)),
    dict(N=3, volume_flux=10, riemann=11, noncons=0),
]


@pytest.mark.parametrize("case", MHD_CASES, ids=lambda c: "N%d_vf%d_rs%d_nc%d%s" % (
    c["N"], c["volume_flux"], c["riemann"], c.get("noncons", 1), "_ncglm" if c.get("nc_glm") else ""))
def test_gauss_mhd_parity(gpu_lib, case):
    """Ideal MHD + GLM with Gauss nodes: entropy-projected face states (Derigs, FloGor), the MHD FluxB surface
    correction with the non-conservative fluxes of both directions, the sides' own non-conservative surface
    terms from the face states; Ut against the oracle (1e-10 with the 9-wave solver 14, else 1e-12)."""
    c, op = mhd_pair(**case)
    ref = c.dg_time_derivative(0.0)
    op.dg_time_derivative(0.0)
    assert rel_l2(op.get_ut(), ref) <= (1e-10 if case["riemann"] == 14 else 1e-12)


def test_gauss_mhd_entropy_and_freestream_on_gpu(gpu_lib):
    c, op = mhd_pair(volume_flux=10, riemann=11, nElems=(3, 3, 2))
    op.dg_time_derivative(0.0)
    assert abs(op.analyze(0.0)["dSdU_Ut"]) < 1e-13
    c, op = mhd_pair(volume_flux=10, riemann=14, nElems=(3, 3, 2))
    op.dg_time_derivative(0.0)
    assert op.analyze(0.0)["dSdU_Ut"] < -1e-6
    c, op = mhd_pair(noise=0.0, ini_exact_func=1, volume_flux=12, riemann=15)
    op.dg_time_derivative(0.0)
    assert np.abs(op.get_ut()).max() < 1e-11


@pytest.mark.parametrize("time_disc", [0, 8])
def test_gauss_mhd_time_steps(gpu_lib, time_disc):
    """CALCTIMESTEP with the Gauss CFL table and GLM_ch, and three steps: states within 1e-11 of the oracle's."""
    c, op = mhd_pair(time_disc=time_disc, cfl_scale=0.5)
    t = 0.0
    for _ in range(3):
        dt_o, err_o = c.calc_timestep()
        dt, err = op.calc_timestep()
        assert err == err_o == 0 and abs(dt - dt_o) <= 1e-12 * dt_o
        assert abs(op.glm_ch - c.glm_ch) <= 1e-12 * c.glm_ch
        c.timestep(t, dt_o)
        op.timestep(t, dt_o)
        t += dt_o
    assert rel_l2(op.get_state(), c.get_U()) <= 1e-11


RESISTIVE = [dict(N=3, lifting=1, lifting_var=3), dict(N=3, lifting=1, lifting_var=1), dict(N=4, lifting=2, lifting_var=3),
             dict(N=4, lifting=2, lifting_var=2), dict(N=2, lifting=1, lifting_var=2), dict(N=5, lifting=1, lifting_var=3),
             dict(N=7, lifting=2, lifting_var=3, nElems=(2, 1, 1)), dict(N=7, lifting=1, lifting_var=1, nElems=(2, 1, 1))]


@pytest.mark.parametrize("case", RESISTIVE, ids=lambda c: "N%d_br%d_lv%d" % (c["N"], c["lifting"], c["lifting_var"]))
def test_gauss_resistive_mhd_parity(gpu_lib, case):
    """Resistive / viscous MHD with Gauss nodes: BR1 / BR2 gradients of the lifting variable with the surface terms
    along the lines, face traces converted with the face states, the 7-component viscous face shares and volume
    integral; Ut against the oracle to 1e-12."""
    c, op = mhd_pair(eqn=3, mu0=0.01, eta=0.02, volume_flux=10, riemann=11, **case)
    ref = c.dg_time_derivative(0.0)
    op.dg_time_derivative(0.0)
    assert rel_l2(op.get_ut(), ref) <= 1e-12


def test_gauss_resistive_mhd_time_steps(gpu_lib):
    c, op = mhd_pair(eqn=3, mu0=0.01, eta=0.02, volume_flux=10, riemann=14, N=4, time_disc=0, cfl_scale=0.5,
                     dfl_scale=0.5)
    t = 0.0
    for _ in range(3):
        dt_o, err_o = c.calc_timestep()
        dt, err = op.calc_timestep()
        assert err == err_o == 0 and abs(dt - dt_o) <= 1e-12 * dt_o
        c.timestep(t, dt_o)
        op.timestep(t, dt_o)
        t += dt_o
    assert rel_l2(op.get_state(), c.get_U()) <= 1e-10
