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
