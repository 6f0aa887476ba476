"""The oracle's Gauss-node (PP_NodeType = 1) entropy-stable collocation scheme (dg.f90:458-511 entropy-
projected ProlongToFace, prolongtoface.f90:103-132, surfint.f90:118-175 FluxB correction, br1/br2 Gauss
lifting, mesh/metrics.f90:325-427 metrics through the LGL grid with SurfMetrics) pinned on the reference's
own regression criteria (tests/job_def.py: freestream L_inf <= 1e-11 on a warped mesh, entropy
conservation |dS/dU . Ut| <= 1e-13 with the EC fluxes, entropy stability with the ES solvers) and on the
order of convergence (tests/convergence/runtest.py)."""
import numpy as np
import pytest

from oracle.oracle import OracleCase

WARPED = dict(N=3, nElems=(3, 3, 3), xmin=(-1, -1, -1), xmax=(1, 1, 1), NGeo=3, deform_amp=0.1, node_type=1)


def noisy(seed=5, **kw):
    c = OracleCase(eqn=0, ini_exact_func=2, ini_amplitude=0.3, adv_vel=(0.3, -0.2, 0.5), **kw)
    U = c.get_U()
    c.set_U(U * (1 + 0.05 * np.random.default_rng(seed).standard_normal(U.shape)))
    return c


@pytest.mark.parametrize("vf,rs", [(1, 1), (0, 22), (5, 44), (10, 4), (32, 33), (2, 1), (9, 2)])
def test_gauss_freestream(vf, rs):
    c = OracleCase(eqn=0, ini_exact_func=1, volume_flux=vf, riemann=rs, ref_state=(1.1, 0.3, -0.2, 0.1, 0.8),
                   **WARPED)
    assert np.abs(c.dg_time_derivative(0.0)).max() <= 1e-11


@pytest.mark.parametrize("lifting,lv", [(1, 3), (1, 1), (2, 2), (2, 3)])
def test_gauss_navier_stokes_freestream(lifting, lv):
    c = OracleCase(eqn=1, ini_exact_func=1, volume_flux=5, riemann=44, ref_state=(1.1, 0.3, -0.2, 0.1, 0.8),
                   mu0=0.01, lifting=lifting, lifting_var=lv, **WARPED)
    assert np.abs(c.dg_time_derivative(0.0)).max() <= 1e-11


@pytest.mark.parametrize("vf,rs", [(5, 9), (10, 5), (32, 32)])
def test_gauss_entropy_conservation(vf, rs):
    """EC volume flux, EC surface flux, entropy-projected face states: the Gauss scheme conserves the
    entropy to roundoff on a curved mesh."""
    c = noisy(volume_flux=vf, riemann=rs, **WARPED)
    c.dg_time_derivative(0.0)
    assert abs(c.analyze(0.0)["dSdU_Ut"]) <= 1e-13


@pytest.mark.parametrize("vf,rs", [(5, 44), (10, 4), (32, 33), (5, 1)])
def test_gauss_entropy_stability(vf, rs):
    c = noisy(volume_flux=vf, riemann=rs, **WARPED)
    c.dg_time_derivative(0.0)
    assert c.analyze(0.0)["dSdU_Ut"] <= 1e-13


def test_gauss_converges_at_order_n_plus_1_and_beats_lgl():
    """Advected density wave (IniExactFunc 2), N = 3, 2^3 / 4^3 / 8^3 elements to t = 0.2: the Gauss
    scheme converges at about N+1 and has a smaller error than the LGL scheme on every mesh."""
    err = {}
    for nt in (1, 2):
        e = []
        for ne in (2, 4, 8):
            c = OracleCase(eqn=0, N=3, nElems=(ne, ne, ne), xmin=(0, 0, 0), xmax=(2, 2, 2), NGeo=1, ini_exact_func=2,
                           ini_amplitude=0.1, adv_vel=(1, 1, 1), volume_flux=5, riemann=44, node_type=nt, cfl_scale=0.5)
            t, _ = c.run(0.0, 0.2)
            e.append(c.analyze(t)["L2"][0])
        err[nt] = e
    eoc = np.log2(err[1][1] / err[1][2])
    assert eoc > 3.7
    assert all(g < l for g, l in zip(err[1], err[2]))


def test_gauss_restrictions():
    """Gauss nodes here run without the NFVSE subcells (which need LGL nodes)."""
    with pytest.raises(Exception):
        OracleCase(eqn=0, ini_exact_func=1, volume_flux=5, riemann=44, nfvse=1, **WARPED)


MHD_REF = ((1.2, 0.1, 0.0, 0.1, 0.9, 1.0, 1.0, 1.0), (1.1, 0.2, -0.1, 0.2, 0.6, 1.0, 1.0, 1.0))
MHD = dict(eqn=2, N=3, nElems=(3, 3, 2), xmin=(-1, -1, -1), xmax=(1, 1, 1), NGeo=2, deform_amp=0.1, kappa=5 / 3,
           mhd_ref_state=MHD_REF, ini_exact_func=201, ini_center=(0.1, 0.05, 0.0), ini_halfwidth=0.4,
           ini_amplitude=0.02, glm_ch=0.7, node_type=1)


def noisy_mhd(seed=0, **kw):
    c = OracleCase(**dict(MHD, **kw))
    U = c.get_U()
    rng = np.random.default_rng(seed)
    U = U * (1 + 0.01 * rng.standard_normal(U.shape))
    U[..., 8] = 0.05 * rng.standard_normal(U[..., 8].shape)
    c.set_U(U)
    return c


@pytest.mark.parametrize("vf,rs,nc", [(1, 1, 1), (10, 11, 1), (12, 12, 2), (10, 14, 3), (0, 4, 1)])
def test_gauss_mhd_freestream(vf, rs, nc):
    """MHD + GLM with Gauss nodes on a curved box: a constant state stays constant (|Ut| < 1e-11), with the
    non-conservative terms in the volume, on the faces and in the split-form surface correction."""
    c = OracleCase(**dict(MHD, ini_exact_func=1, volume_flux=vf, riemann=rs, noncons=nc))
    assert np.abs(c.dg_time_derivative()).max() < 1e-11


@pytest.mark.parametrize("vf,rs,ncg", [(10, 11, 0), (10, 11, 1), (12, 12, 0)])
def test_gauss_mhd_entropy_conservation(vf, rs, ncg):
    """Derigs (10) / FloGor (12) volume and surface fluxes with Powell terms, Gauss nodes with the entropy-projected
    face states and the FluxB correction with the non-conservative fluxes (surfint.f90:118-175): dS/dU . Ut
    vanishes to round-off (the criterion of the reference's mhd softBlast/entropyCons runs, 1e-13)."""
    c = noisy_mhd(volume_flux=vf, riemann=rs, noncons=1, nc_glm=ncg)
    c.dg_time_derivative()
    assert abs(c.analyze(0.0)["dSdU_Ut"]) < 1e-13


@pytest.mark.parametrize("vf,rs", [(10, 10), (12, 15), (10, 14)])
def test_gauss_mhd_entropy_stability(vf, rs):
    c = noisy_mhd(volume_flux=vf, riemann=rs, noncons=1)
    c.dg_time_derivative()
    assert c.analyze(0.0)["dSdU_Ut"] < -1e-6


def test_gauss_mhd_needs_the_powell_terms_for_entropy_conservation():
    c = noisy_mhd(volume_flux=10, riemann=11, noncons=0)
    c.dg_time_derivative()
    assert abs(c.analyze(0.0)["dSdU_Ut"]) > 1e-6


@pytest.mark.parametrize("lifting,lv", [(1, 3), (2, 2)])
def test_gauss_resistive_mhd(lifting, lv):
    """Resistive / viscous MHD with Gauss nodes (the lifting's Gauss branches): free-stream preserving and
    dissipative with the entropy-conserving inviscid fluxes."""
    kw = dict(eqn=3, mu0=0.01, eta=0.01, lifting=lifting, lifting_var=lv, volume_flux=10, riemann=11)
    f = OracleCase(**dict(MHD, ini_exact_func=1, **kw))
    assert np.abs(f.dg_time_derivative()).max() < 1e-11
    c = noisy_mhd(**kw)
    c.dg_time_derivative()
    assert c.analyze(0.0)["dSdU_Ut"] < -1e-6
