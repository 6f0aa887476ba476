"""The oracle's NFVSE shock capturing (shockcapturing/nfvse.f90, first-order subcell FV) pinned on the
reference's regression criteria for shock capturing (tests/job_def.py:817-870: freestream with the
first-order subcell scheme, L_inf <= 1e-11; entropy conservation / stability of the blended scheme with
EC / ES fluxes) and on the properties of the blending coefficient (indicators/indicators.f90:108-173,
nfvse.f90:1537-1620, nfvse_mpi.f90:62-131)."""
import numpy as np
import pytest

from oracle.oracle import OracleCase

REF = ((1.2, 0.1, 0.0, 0.1, 0.9, 1.0, 1.0, 1.0), (1.1, 0.2, -0.1, 0.2, 0.6, 1.0, 1.0, 1.0))
WARPED = dict(N=3, nElems=(3, 3, 3), xmin=(-1, -1, -1), xmax=(1, 1, 1), NGeo=3, deform_amp=0.1)
MHD = dict(eqn=2, kappa=5 / 3, mhd_ref_state=REF, glm_ch=0.7, noncons=1, nc_glm=1)
FIXED = dict(nfvse=1, compute_alpha=3, shock_blend_coef=0.4, alpha_max=0.5, alpha_min=0.01)


def noisy_blast(seed=1, **kw):
    c = OracleCase(ini_exact_func=201, ini_center=(0, 0, 0), ini_halfwidth=0.3, ini_amplitude=0.1, **WARPED, **kw)
    rng = np.random.default_rng(seed)
    U = c.get_U()
    U = U * (1 + 0.02 * rng.standard_normal(U.shape))
    U[..., 8] = 0.05 * rng.standard_normal(U[..., 8].shape)
    c.set_U(U)
    return c


@pytest.mark.parametrize("vf,rs", [(10, 11), (10, 14), (12, 13), (0, 1)])
def test_nfvse_mhd_freestream(vf, rs):
    c = OracleCase(ini_exact_func=1, volume_flux=vf, riemann=rs, **WARPED, **MHD, **FIXED)
    assert np.abs(c.dg_time_derivative(0.0)).max() <= 1e-11


@pytest.mark.parametrize("rs", [1, 44, 9])
def test_nfvse_euler_freestream(rs):
    c = OracleCase(eqn=0, ini_exact_func=1, volume_flux=5, riemann=rs, ref_state=(1.1, 0.3, -0.2, 0.1, 0.8),
                   **WARPED, **FIXED)
    assert np.abs(c.dg_time_derivative(0.0)).max() <= 1e-11


@pytest.mark.parametrize("vf,rs", [(10, 11), (12, 12)])
def test_nfvse_mhd_entropy_conservation(vf, rs):
    c = noisy_blast(volume_flux=vf, riemann=rs, **MHD, **FIXED)
    c.dg_time_derivative(0.0)
    assert abs(c.analyze(0.0)["dSdU_Ut"]) <= 1e-13


@pytest.mark.parametrize("vf,rs", [(10, 14), (10, 10), (12, 15)])
def test_nfvse_mhd_entropy_stability(vf, rs):
    c = noisy_blast(volume_flux=vf, riemann=rs, **MHD, **FIXED)
    c.dg_time_derivative(0.0)
    assert c.analyze(0.0)["dSdU_Ut"] <= 1e-13


def test_nfvse_blending_reduces_to_dg_when_alpha_is_zero():
    c0 = noisy_blast(volume_flux=10, riemann=14, **MHD)
    c1 = noisy_blast(volume_flux=10, riemann=14, **MHD, nfvse=1, compute_alpha=3, shock_blend_coef=0.005)
    assert np.array_equal(c0.dg_time_derivative(0.0), c1.dg_time_derivative(0.0))
    assert np.all(c1.alpha() == 0.0)


def test_persson_peraire_indicator_and_propagation():
    """Smooth data stays pure DG; a sharp blast switches elements on (alpha in (0, alpha_max]) and the
    space propagation gives every neighbour of a blended element at least SpacePropFactor * alpha."""
    smooth = OracleCase(ini_exact_func=3, eqn=2, N=4, nElems=(3, 3, 3), xmin=(-1, -1, -1), xmax=(1, 1, 1),
                        kappa=5 / 3, volume_flux=10, riemann=14, nfvse=1)
    smooth.dg_time_derivative(0.0)
    assert np.all(smooth.alpha() == 0.0)
    c = OracleCase(ini_exact_func=201, ini_center=(0.1, 0.05, 0.0), ini_halfwidth=0.4, ini_amplitude=0.01, eqn=2,
                   N=4, nElems=(4, 4, 4), xmin=(-1, -1, -1), xmax=(1, 1, 1), kappa=5 / 3, mhd_ref_state=REF,
                   volume_flux=10, riemann=14, nfvse=1, space_prop_sweeps=0)
    c.dg_time_derivative(0.0)
    a0 = c.alpha()
    assert a0.max() > 0.0 and a0.max() <= 0.5
    assert np.all((a0 == 0.0) | (a0 >= 0.01))
    cp = OracleCase(ini_exact_func=201, ini_center=(0.1, 0.05, 0.0), ini_halfwidth=0.4, ini_amplitude=0.01, eqn=2,
                    N=4, nElems=(4, 4, 4), xmin=(-1, -1, -1), xmax=(1, 1, 1), kappa=5 / 3, mhd_ref_state=REF,
                    volume_flux=10, riemann=14, nfvse=1, space_prop_sweeps=1)
    cp.dg_time_derivative(0.0)
    a1 = cp.alpha()
    assert np.all(a1 >= a0)
    e2s = cp.mesh()["ElemToSide"][:, :, 0] - 1
    s2e = cp.mesh()["SideToElem"][:, :2] - 1
    for e in range(cp.nElems):
        nbs = {int(x) for s in e2s[e] for x in s2e[s] if x != e}
        assert a1[e] >= 0.5 * max(a0[n] for n in nbs) - 1e-15


TVD = dict(FIXED, sub_fv_method=2)


@pytest.mark.parametrize("rb", [1, 2, 3])
def test_nfvse_tvd_freestream(rb):
    """SubFVMethod 2 (minmod reconstruction of the primitive variables) keeps a constant state."""
    c = OracleCase(ini_exact_func=1, volume_flux=10, riemann=14, recons_boundaries=rb, **WARPED, **MHD, **TVD)
    assert np.abs(c.dg_time_derivative(0.0)).max() <= 1e-11
    c = OracleCase(eqn=0, ini_exact_func=1, volume_flux=5, riemann=1, ref_state=(1.1, 0.3, -0.2, 0.1, 0.8),
                   recons_boundaries=rb, **WARPED, **TVD)
    assert np.abs(c.dg_time_derivative(0.0)).max() <= 1e-11


def test_nfvse_tvd_is_conservative_and_differs_from_first_order():
    """The blended scheme with the TVD subcell fluxes conserves mass, momentum and energy on a periodic
    mesh (sum of w J Ut = 0), and each reconstruction at the element boundaries gives another Ut."""
    from oracle.oracle import basis
    out = []
    for kw in (dict(FIXED), dict(TVD, recons_boundaries=1), dict(TVD, recons_boundaries=2),
               dict(TVD, recons_boundaries=3)):
        c = OracleCase(eqn=0, ini_exact_func=2, ini_amplitude=0.3, volume_flux=5, riemann=1,
                       adv_vel=(0.3, -0.2, 0.5), **WARPED, **kw)
        U = c.get_U()
        c.set_U(U * (1 + 0.05 * np.random.default_rng(5).standard_normal(U.shape)))
        Ut = c.dg_time_derivative(0.0)
        w = basis(3)["wGP"]
        W = w[None, None, None, :] * w[None, None, :, None] * w[None, :, None, None]
        sJ = c.mesh()["sJ"].reshape(Ut.shape[:4])
        total = np.einsum("ekji,ekjiv->v", W / sJ, Ut)
        assert np.abs(total).max() <= 1e-12 * np.abs(Ut).max()
        out.append(Ut)
    for a in range(4):
        for b in range(a + 1, 4):
            assert np.abs(out[a] - out[b]).max() > 1e-6
