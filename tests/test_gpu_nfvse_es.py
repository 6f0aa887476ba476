"""Parity of the entropy-stable NFVSE subcell schemes and of the NFVSE positivity correction on the
sm_100a path against the CPU oracle, through the C ABI:
  SubFVMethod 3 (TVD-ES, shockcapturing/nfvse.f90:826-1090) and 4 (TVD-Fjordholm, :1101-1386) with every
  boundary reconstruction, Euler / Navier-Stokes (Riemann 4, 44, 33) and MHD (Riemann 14, 15);
  NFVSE_CORR (Apply_NFVSE_Correction, :1688-1883) after the stages of carpenterrk4-5 and ssprk4-5, on
  the host-driven and on the device-resident time loop.
Data carry node noise, so that no minmod limiter of the reconstructions sees two exactly equal slopes
(a tie selects a branch by the last bit).  Tolerances: Ut relative L2 <= 1e-12 (FP64, another
summation order), 1e-10 with the 9-wave MHD solver whose TVD states move by 4e-11 between two legal
roundings; states after corrected steps <= 1e-10."""
import numpy as np
import pytest

import fluxo_b200 as fb
from fluxo_b200._lib import FluxoError
from oracle.oracle import OracleCase

pytestmark = pytest.mark.gpu
REF = ((1.2, 0.1, 0.0, 0.1, 0.9, 1.0, 1.0, 1.0), (1.1, 0.2, -0.1, 0.2, 0.6, 1.0, 1.0, 1.0))
NFVSE_KEYS = ("nfvse", "compute_alpha", "shock_blend_coef", "modal_threshold", "alpha_max", "alpha_min",
              "space_prop_factor", "space_prop_sweeps", "time_rel_factor", "indicator_quantity", "sub_fv_method",
              "recons_boundaries", "nfvse_corr", "posit_corr_factor", "posit_max_iter")


def rel_l2(a, b):
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)


def operator_for(c, U, ch=None):
    p = c.params
    fields = dict(N=p.N, eqn=p.eqn, riemann=p.riemann, volume_flux=p.volume_flux, lifting=p.lifting,
                  lifting_var=p.lifting_var, visc=p.visc, kappa=p.kappa, Pr=p.Pr, mu0=p.mu0, time_disc=p.time_disc,
                  cfl_scale=p.cfl_scale, dfl_scale=p.dfl_scale, ini_exact_func=1, mu_0=p.mu_0, eta=p.eta,
                  glm_scale=p.glm_scale, glm_scr=p.glm_scr, noncons=p.noncons, nc_glm=p.nc_glm)
    fields.update({k: getattr(p, k) for k in NFVSE_KEYS})
    op = fb.DGOperator(**fields)
    op.set_mesh(c.mesh())
    op.set_state(U)
    if ch is not None:
        op.glm_ch = ch
    return op


def euler_pair(noise=0.03, seed=4, **kw):
    base = dict(eqn=0, N=3, nElems=(3, 2, 2), xmin=(-1, -1, -1), xmax=(1, 1, 1), NGeo=2, deform_amp=0.1,
                ini_exact_func=2, ini_amplitude=0.3, adv_vel=(0.3, -0.2, 0.5), nfvse=1, shock_blend_coef=0.4,
                alpha_min=0.001, riemann=44, volume_flux=5)
    base.update(kw)
    c = OracleCase(**base)
    U = c.get_U()
    U = U * (1 + noise * np.random.default_rng(seed).standard_normal(U.shape))
    c.set_U(U)
    return c, operator_for(c, U)


def mhd_pair(noise=0.05, seed=0, ch=0.7, **kw):
    base = dict(eqn=2, N=3, nElems=(3, 3, 2), xmin=(-1, -1, -1), xmax=(1, 1, 1), NGeo=2, deform_amp=0.1,
                kappa=5 / 3, mhd_ref_state=REF, ini_exact_func=201, ini_center=(0.1, 0.05, 0.0),
                ini_halfwidth=0.4, ini_amplitude=0.02, glm_ch=ch, nfvse=1, volume_flux=10, riemann=14)
    base.update(kw)
    c = OracleCase(**base)
    U = c.get_U()
    rng = np.random.default_rng(seed)
    U = U * (1 + noise * rng.standard_normal(U.shape))
    U[..., 8] = 0.05 * rng.standard_normal(U[..., 8].shape)
    c.set_U(U)
    return c, operator_for(c, U, ch)


EULER_ES = [
    dict(N=3, riemann=44, volume_flux=5, sub_fv_method=3, recons_boundaries=1),
    dict(N=3, riemann=44, volume_flux=5, sub_fv_method=3, recons_boundaries=2),
    dict(N=4, riemann=44, volume_flux=5, sub_fv_method=3, recons_boundaries=3),
    dict(N=3, riemann=4, volume_flux=10, sub_fv_method=4, recons_boundaries=1),
    dict(N=4, riemann=44, volume_flux=5, sub_fv_method=4, recons_boundaries=2),
    dict(N=3, riemann=33, volume_flux=32, sub_fv_method=4, recons_boundaries=3),
    dict(N=7, riemann=44, volume_flux=5, sub_fv_method=4, recons_boundaries=3, nElems=(2, 1, 1)),
    dict(N=7, riemann=33, volume_flux=32, sub_fv_method=3, recons_boundaries=3, nElems=(2, 1, 1)),
    dict(N=3, riemann=44, volume_flux=5, sub_fv_method=4, recons_boundaries=3, eqn=1, mu0=0.01),
]


@pytest.mark.parametrize("case", EULER_ES, ids=lambda c: "eqn%d_N%d_rs%d_m%d_rb%d" % (
    c.get("eqn", 0), c["N"], c["riemann"], c["sub_fv_method"], c["recons_boundaries"]))
def test_es_subcell_euler_parity(gpu_lib, case):
    for ca in (3, 1):
        c, op = euler_pair(compute_alpha=ca, **case)
        ref = c.dg_time_derivative(0.0)
        op.dg_time_derivative(0.0)
        assert np.abs(op.alpha() - c.alpha()).max() <= 1e-12
        if ca == 1:
            assert (c.alpha() > 0).any()
        assert rel_l2(op.get_ut(), ref) <= 1e-12


MHD_ES = [
    dict(N=3, riemann=14, volume_flux=10, sub_fv_method=3, recons_boundaries=1),
    dict(N=4, riemann=15, volume_flux=12, sub_fv_method=3, recons_boundaries=3, nc_glm=1),
    dict(N=3, riemann=14, volume_flux=10, sub_fv_method=4, recons_boundaries=2),
    dict(N=4, riemann=15, volume_flux=12, sub_fv_method=4, recons_boundaries=3, noncons=3),
    dict(N=2, riemann=14, volume_flux=10, sub_fv_method=4, recons_boundaries=1, noncons=2),
]


@pytest.mark.parametrize("case", MHD_ES, ids=lambda c: "N%d_rs%d_m%d_rb%d" % (
    c["N"], c["riemann"], c["sub_fv_method"], c["recons_boundaries"]))
def test_es_subcell_mhd_parity(gpu_lib, case):
    for ca in (3, 1):
        c, op = mhd_pair(compute_alpha=ca, shock_blend_coef=0.4, **case)
        ref = c.dg_time_derivative(0.0)
        op.dg_time_derivative(0.0)
        assert np.abs(op.alpha() - c.alpha()).max() <= 1e-12
        assert rel_l2(op.get_ut(), ref) <= 1e-10


CORR_BOX = dict(eqn=0, N=3, nElems=(4, 4, 4), xmin=(-1, -1, -1), xmax=(1, 1, 1), NGeo=1, ini_exact_func=1,
                ref_state=(1.0, 0.0, 0.0, 0.0, 1.0), volume_flux=5, riemann=1, nfvse=1, alpha_max=0.5,
                alpha_min=0.01, cfl_scale=0.2, nfvse_corr=1)


def corr_pair(**kw):
    """Density and pressure jumps by a factor 100 across a sphere (the DG update undershoots there)."""
    c = OracleCase(**dict(CORR_BOX, **kw))
    x = c.mesh()["Elem_xGP"].reshape(c.nElems, c.N + 1, c.N + 1, c.N + 1, 3)
    r = np.sqrt(((x - 0.05) ** 2).sum(-1))
    U = np.zeros(x.shape[:4] + (5,))
    U[..., 0] = np.where(r < 0.35, 1.0, 0.01)
    U[..., 4] = np.where(r < 0.35, 1.0, 0.01) / 0.4
    c.set_U(U)
    return c, operator_for(c, U), U


def test_nfvse_corr_lserk_host_steps_parity(gpu_lib):
    """carpenterrk4-5, host-driven steps: the correction after every stage (fused stage update, then
    the correction kernel) matches the oracle step by step; without it the states differ."""
    c, op, U0 = corr_pair(time_disc=0)
    c0, _, _ = corr_pair(time_disc=0, nfvse_corr=0)
    t = 0.0
    for _ in range(4):
        dt, err = c.calc_timestep()
        dtg, errg = op.calc_timestep()
        assert err == errg == 0 and dtg == pytest.approx(dt, rel=1e-12)
        c.timestep(t, dt)
        op.timestep(t, dt)
        c0.timestep(t, dt)
        t += dt
        assert rel_l2(op.get_state(), c.get_U()) <= 1e-10
    assert c.corr_error == 0
    assert rel_l2(c0.get_U(), c.get_U()) > 1e-8


def test_nfvse_corr_ssprk45_device_loop_parity(gpu_lib):
    """ssprk4-5 at CFLScale 0.5: without the correction the first step fails (NaN density), with it the
    device-resident loop runs six steps (correction after every stage, the r1 register from the
    corrected U and Ut) and matches the oracle."""
    c, op, U0 = corr_pair(time_disc=8, cfl_scale=0.5)
    t_ref, n_ref = c.run(0.0, 10.0, max_iter=6)
    t, n, err = op.time_disc(0.0, 10.0, max_iter=6)
    assert c.corr_error == 0 and err == 0 and n == n_ref == 6
    assert t == pytest.approx(t_ref, rel=1e-10)
    assert rel_l2(op.get_state(), c.get_U()) <= 1e-10
    c0, op0, _ = corr_pair(time_disc=8, cfl_scale=0.5, nfvse_corr=0)
    _, _, err0 = op0.time_disc(0.0, 10.0, max_iter=6)
    assert err0 == 1


def test_nfvse_corr_ssprk33_runs_without_correction(gpu_lib):
    """ssprk3-3 steps without Apply_NFVSE_Correction in the reference: nfvse_corr leaves its states as
    they are without it (the FV flux of every element is blended with alpha = 0 where not flagged)."""
    c, op, _ = corr_pair(time_disc=9)
    c0, op0, _ = corr_pair(time_disc=9, nfvse_corr=0)
    op.time_disc(0.0, 10.0, max_iter=3)
    op0.time_disc(0.0, 10.0, max_iter=3)
    c.run(0.0, 10.0, max_iter=3)
    assert rel_l2(op.get_state(), op0.get_state()) <= 1e-14
    assert rel_l2(op.get_state(), c.get_U()) <= 1e-11


def test_nfvse_corr_mhd_parity(gpu_lib):
    """MHD (9-wave ES solver, Powell terms), ssprk4-5 on a factor-300 density / pressure blast in a
    constant field: the uncorrected run fails in its first step, the corrected one runs four steps on
    the device loop and matches the oracle."""
    def blast(corr):
        c = OracleCase(eqn=2, N=3, nElems=(4, 4, 4), xmin=(-1, -1, -1), xmax=(1, 1, 1), NGeo=1, kappa=5 / 3,
                       mhd_ref_state=REF, ini_exact_func=1, glm_ch=0.5, nfvse=1, volume_flux=10, riemann=14,
                       alpha_max=0.5, alpha_min=0.01, cfl_scale=0.3, nfvse_corr=corr, time_disc=8, noncons=1)
        x = c.mesh()["Elem_xGP"].reshape(c.nElems, 4, 4, 4, 3)
        r = np.sqrt(((x - 0.05) ** 2).sum(-1))
        U = np.zeros(x.shape[:4] + (9,))
        U[..., 0] = np.where(r < 0.35, 1.0, 0.003)
        U[..., 5:8] = (0.1, 0.05, 0.02)
        U[..., 4] = np.where(r < 0.35, 1.0, 0.003) / (2 / 3) + 0.5 * (U[..., 5:8] ** 2).sum(-1)
        c.set_U(U)
        return c, operator_for(c, U, 0.5)
    c, op = blast(1)
    t_ref, n_ref = c.run(0.0, 10.0, max_iter=4)
    t, n, err = op.time_disc(0.0, 10.0, max_iter=4)
    assert c.corr_error == 0 and err == 0 and n == n_ref == 4
    assert rel_l2(op.get_state(), c.get_U()) <= 1e-10
    _, op0 = blast(0)
    assert op0.time_disc(0.0, 10.0, max_iter=4)[2] != 0


def test_nfvse_corr_inadmissible_safe_state_is_an_error(gpu_lib):
    """carpenterrk4-5 at CFLScale 0.5 on the blast: a safe state with negative density appears in the first
    step (the reference stops there); fluxo_gpu_timestep returns FLUXO_ENAN_STATE."""
    c, op, _ = corr_pair(time_disc=0, cfl_scale=0.5)
    dt, _ = c.calc_timestep()
    c.timestep(0.0, dt)
    assert c.corr_error > 0
    with pytest.raises(FluxoError) as ex:
        op.timestep(0.0, dt)
    assert ex.value.code == -4 and "NFVSE correction" in str(ex.value)
