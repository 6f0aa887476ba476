"""The oracle's MHD + GLM equation system (equation/mhd/*) pinned on the reference's own regression
criteria for MHD (tests/job_def.py:495-570): freestream preservation on a heavily warped mesh
(L_inf <= 1e-11), discrete entropy conservation of the EC volume / surface flux pairs with the
non-conservative terms (|dS/dU.Ut| <= 1e-13), entropy stability of the dissipative solvers
(dS/dU.Ut <= 1e-13), and the convergence order of the Alfven wave (IniExactFunc 3)."""
import numpy as np
import pytest

from oracle.oracle import OracleCase

REF = ((1.2, 0.1, 0.0, 0.1, 0.9, 1.0, 1.0, 1.0), (1.1, 0.2, -0.1, 0.2, 0.6, 1.0, 1.0, 1.0))  # softBlast RefStates
WARPED = dict(N=3, nElems=(3, 3, 3), xmin=(-1, -1, -1), xmax=(1, 1, 1), NGeo=3, deform_amp=0.1, kappa=5 / 3,
              mhd_ref_state=REF, glm_ch=0.7)
PARA = dict(eta=0.05, mu0=0.02)


def blast(seed=1, **kw):
    """Soft blast (IniExactFunc 201) with node-wise noise, so that the element interfaces carry jumps,
    and a non-zero psi field."""
    c = OracleCase(ini_exact_func=201, ini_center=(0, 0, 0), ini_halfwidth=0.3, ini_amplitude=0.1, **WARPED, **kw)
    rng = np.random.default_rng(seed)
    U = c.get_U()
    U = U * (1 + 0.02 * rng.standard_normal(U.shape))
    U[..., 8] = 0.05 * rng.standard_normal(U[..., 8].shape)
    c.set_U(U)
    c.dg_time_derivative(0.0)
    return c.analyze(0.0)["dSdU_Ut"]


@pytest.mark.parametrize("eqn", [2, 3])
@pytest.mark.parametrize("vf,rs", [(10, 11), (12, 12), (10, 14), (0, 1), (1, 4), (10, 10), (12, 13), (12, 15), (10, 0)])
def test_mhd_freestream(eqn, vf, rs):
    c = OracleCase(eqn=eqn, ini_exact_func=1, volume_flux=vf, riemann=rs, noncons=1, nc_glm=1, **WARPED,
                   **(PARA if eqn == 3 else {}))
    assert np.abs(c.dg_time_derivative(0.0)).max() <= 1e-11


@pytest.mark.parametrize("vf,rs,ncglm", [(10, 11, 1), (12, 12, 1), (10, 11, 0)])
def test_mhd_entropy_conservation(vf, rs, ncglm):
    assert abs(blast(eqn=2, volume_flux=vf, riemann=rs, noncons=1, nc_glm=ncglm)) <= 1e-13


def test_mhd_noncons_term_is_needed():
    """Without the Powell term the EC pair does not conserve entropy (div B != 0 at the nodes)."""
    assert abs(blast(eqn=2, volume_flux=10, riemann=11, noncons=0)) > 1e-6


@pytest.mark.parametrize("eqn", [2, 3])
@pytest.mark.parametrize("vf,rs", [(10, 14), (10, 10), (12, 13), (12, 15), (0, 1), (1, 4)])
def test_mhd_entropy_stability(eqn, vf, rs):
    assert blast(eqn=eqn, volume_flux=vf, riemann=rs, noncons=1, nc_glm=1, **(PARA if eqn == 3 else {})) <= 1e-13


def test_mhd_alfven_wave_convergence():
    errs = []
    for ne in (2, 4, 8):
        c = OracleCase(eqn=2, N=3, nElems=(ne, ne, ne), xmin=(-1, -1, -1), xmax=(1, 1, 1), NGeo=2, deform_amp=0.05,
                       kappa=5 / 3, ini_exact_func=3, ini_frequency=1.0, volume_flux=10, riemann=14, noncons=1,
                       cfl_scale=0.5)
        t, _ = c.run(0.0, 0.1)
        assert t == pytest.approx(0.1)
        errs.append(c.analyze(t)["L2"][1:4].sum())
    eoc = np.log(np.array(errs[:-1]) / np.array(errs[1:])) / np.log(2)
    assert eoc[-1] > 3.0


def test_mhd_glm_speed_from_timestep():
    """GLM_dtch1 = CFLScale*2/sum(sJ|Ja|) on a Cartesian box (dx/3 * CFLScale) and
    GLM_ch = GLM_scale*GLM_dtch1/dt (mhd/calctimestep.f90:176, :187-223)."""
    c = OracleCase(eqn=2, N=3, nElems=(4, 4, 4), xmin=(0, 0, 0), xmax=(2, 2, 2), NGeo=1, kappa=5 / 3,
                   ini_exact_func=311, glm_scale=0.5, cfl_scale=0.9)
    dt, err = c.calc_timestep()
    assert err == 0
    cfl = 0.9 * 2.8451 / 7.0  # CFLScale * alpha(N=3) / (2N+1)
    dtch1 = cfl * 0.5 / 3.0
    assert c.glm_ch == pytest.approx(0.5 * dtch1 / dt, rel=1e-13)


def _mhd_state(rng, B=True, psi=True):
    rho, p = 1 + 0.3 * rng.random(), 0.8 + 0.4 * rng.random()
    v = 0.4 * rng.standard_normal(3)
    b = 0.6 * rng.standard_normal(3) if B else np.zeros(3)
    s = 0.1 * rng.standard_normal() if psi else 0.0
    E = p / (5 / 3 - 1) + 0.5 * rho * v @ v + 0.5 * (b @ b + s * s)
    return np.array([rho, *(rho * v), E, *b, s])


def _point_case(**kw):
    return OracleCase(eqn=2, N=1, nElems=(1, 1, 1), volume_flux=10, kappa=5 / 3, glm_ch=0.7, ini_exact_func=1,
                      mhd_ref_state=REF, **kw)


@pytest.mark.parametrize("rs", [2, 3, 5])
def test_mhd_hllc_roe_hlld_consistent(rs):
    """F*(U, U) equals the Rusanov flux at U, i.e. the physical flux (GLM terms included)."""
    rng = np.random.default_rng(40 + rs)
    c = _point_case(riemann=rs)
    r = _point_case(riemann=1)
    for _ in range(5):
        U = _mhd_state(rng)
        Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        args = (U, U, Q[:, 0], Q[:, 1], Q[:, 2])
        assert np.allclose(c.riemann(*args), r.riemann(*args), rtol=1e-12, atol=1e-13)


def test_mhd_roe_without_field_is_the_euler_roe_flux():
    """With B = 0 and psi = 0 the Cargo-Gallice Roe matrix reduces to the Euler Roe solver."""
    rng = np.random.default_rng(7)
    m = _point_case(riemann=3)
    e = OracleCase(eqn=0, N=1, nElems=(1, 1, 1), riemann=3, volume_flux=0, kappa=5 / 3)
    for _ in range(5):
        UL, UR = _mhd_state(rng, B=False, psi=False), _mhd_state(rng, B=False, psi=False)
        Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        Fm = m.riemann(UL, UR, Q[:, 0], Q[:, 1], Q[:, 2])
        Fe = e.riemann(UL[:5], UR[:5], Q[:, 0], Q[:, 1], Q[:, 2])
        assert np.allclose(Fm[:5], Fe, rtol=1e-12, atol=1e-13)
        assert np.allclose(Fm[5:], 0, atol=1e-13)


@pytest.mark.parametrize("eqn", [2, 3])
@pytest.mark.parametrize("vf,rs", [(10, 2), (0, 3), (10, 5)])
def test_mhd_freestream_hllc_roe_hlld(eqn, vf, rs):
    c = OracleCase(eqn=eqn, ini_exact_func=1, volume_flux=vf, riemann=rs, noncons=1, nc_glm=1, **WARPED,
                   **(PARA if eqn == 3 else {}))
    assert np.abs(c.dg_time_derivative(0.0)).max() <= 1e-11


def test_hlld_needs_unit_mu0():
    with pytest.raises(Exception):
        _point_case(riemann=5, mu_0=2.0)
