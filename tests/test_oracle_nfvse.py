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


# ---- SubFVMethod 3 (TVD-ES, nfvse.f90:826-1090) and 4 (TVD-Fjordholm, :1101-1386) --------------------
EULER_ES = dict(eqn=0, volume_flux=5, riemann=44, ref_state=(1.1, 0.3, -0.2, 0.1, 0.8))


def noisy_euler(seed=5, noise=0.05, **kw):
    c = OracleCase(eqn=0, ini_exact_func=2, ini_amplitude=0.3, adv_vel=(0.3, -0.2, 0.5), **WARPED, **kw)
    U = c.get_U()
    c.set_U(U * (1 + noise * np.random.default_rng(seed).standard_normal(U.shape)))
    return c


def integral(c, Ut):
    from oracle.oracle import basis
    w = basis(c.N)["wGP"]
    W = w[None, None, None, :] * w[None, None, :, None] * w[None, :, None, None]
    sJ = c.mesh()["sJ"].reshape(Ut.shape[:4])
    return np.einsum("ekji,ekjiv->v", W / sJ, Ut)


@pytest.mark.parametrize("sfm", [3, 4])
@pytest.mark.parametrize("rb", [1, 2, 3])
def test_nfvse_es_freestream(sfm, rb):
    """A constant state stays constant with both entropy-stable subcell schemes and every boundary
    reconstruction (Euler with the ES matrix-dissipation solver, MHD with the 9-wave solvers)."""
    c = OracleCase(ini_exact_func=1, sub_fv_method=sfm, recons_boundaries=rb, **WARPED, **EULER_ES, **FIXED)
    assert np.abs(c.dg_time_derivative(0.0)).max() <= 1e-11
    for vf, rs in ((10, 14), (12, 15)):
        c = OracleCase(ini_exact_func=1, volume_flux=vf, riemann=rs, sub_fv_method=sfm, recons_boundaries=rb,
                       **WARPED, **MHD, **FIXED)
        assert np.abs(c.dg_time_derivative(0.0)).max() <= 1e-11


@pytest.mark.parametrize("rs,vf", [(44, 5), (4, 10), (33, 32)])
def test_nfvse_es_conservative_entropy_stable_and_distinct(rs, vf):
    """Euler, every solver with dissipation matrices: the blended scheme with the TVD-ES and Fjordholm
    subcell fluxes conserves mass, momentum and energy on the periodic mesh, produces entropy
    (dS/dU . Ut <= 0), and each method and boundary reconstruction gives another Ut."""
    out = []
    for sfm in (2, 3, 4):
        for rb in (1, 2, 3):
            c = noisy_euler(riemann=rs, volume_flux=vf, sub_fv_method=sfm, recons_boundaries=rb, **FIXED)
            Ut = c.dg_time_derivative(0.0)
            assert np.abs(integral(c, Ut)).max() <= 1e-12 * np.abs(Ut).max()
            assert c.analyze(0.0)["dSdU_Ut"] <= 1e-13
            out.append(Ut)
    for a in range(len(out)):
        for b in range(a + 1, len(out)):
            assert np.abs(out[a] - out[b]).max() > 1e-8


@pytest.mark.parametrize("sfm", [3, 4])
@pytest.mark.parametrize("vf,rs", [(10, 14), (12, 15)])
def test_nfvse_es_mhd_entropy_stability(sfm, vf, rs):
    c = noisy_blast(volume_flux=vf, riemann=rs, sub_fv_method=sfm, recons_boundaries=3, **MHD, **FIXED)
    c.dg_time_derivative(0.0)
    assert c.analyze(0.0)["dSdU_Ut"] <= 1e-13


def test_tvd2es_on_zigzag_data_is_the_first_order_es_scheme():
    """Node-to-node zigzag data zeroes every minmod slope; with ReconsBoundaries 1 the reconstructed
    states are the nodal ones, the entropy switch keeps them, and TVD-ES reduces to the first-order
    subcell scheme with the same entropy-stable solver."""
    def zig(**kw):
        c = OracleCase(ini_exact_func=1, **WARPED, **EULER_ES, **FIXED, **kw)
        U = c.get_U()
        n = c.N + 1
        i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
        sgn = ((-1.0) ** (i + j + k)).transpose(2, 1, 0)[None, :, :, :, None]  # U[e, k, j, i, v]
        U = U * (1 + 0.02 * sgn * np.array([1, 1, 1, 1, 1.0]))
        c.set_U(U)
        return c.dg_time_derivative(0.0)
    u1 = zig(sub_fv_method=1)
    u3 = zig(sub_fv_method=3, recons_boundaries=1)
    assert np.abs(u3 - u1).max() <= 1e-12 * np.abs(u1).max()


def test_nfvse_es_needs_dissipation_matrices():
    """SubFVMethod 3/4 with a solver without RiemannVolFluxAndDissipMatrices is refused
    (nfvse.f90:174-187), as is the NFVSE correction with the LSERKK3 schemes (timedisc_vars.f90:111-114)."""
    with pytest.raises(Exception):
        OracleCase(ini_exact_func=1, sub_fv_method=3, riemann=1, volume_flux=5, eqn=0, **WARPED, **FIXED)
    with pytest.raises(Exception):
        OracleCase(ini_exact_func=1, sub_fv_method=4, riemann=10, volume_flux=10, **WARPED, **MHD, **FIXED)
    with pytest.raises(Exception):
        OracleCase(ini_exact_func=1, nfvse_corr=1, time_disc=6, **WARPED, **EULER_ES, **FIXED)


# ---- NFVSE_CORR: Apply_NFVSE_Correction (nfvse.f90:1688-1883) ------------------------------------
CORR_BOX = dict(eqn=0, N=3, nElems=(4, 4, 4), xmin=(-1, -1, -1), xmax=(1, 1, 1), NGeo=1, ini_exact_func=1,
                ref_state=(1.0, 0.0, 0.0, 0.0, 1.0), volume_flux=5, riemann=1, nfvse=1, alpha_max=0.5,
                alpha_min=0.01, cfl_scale=0.2)


def corr_blast(c, rin=1.0, rout=0.01, pin=1.0, pout=0.01):
    """Density and pressure jumps by a factor 100 across a sphere: the DG update undershoots there."""
    x = c.mesh()["Elem_xGP"].reshape(c.nElems, c.N + 1, c.N + 1, c.N + 1, 3)
    r = np.sqrt(((x - 0.05) ** 2).sum(-1))
    U = np.zeros(x.shape[:4] + (5,))
    U[..., 0] = np.where(r < 0.35, rin, rout)
    U[..., 4] = np.where(r < 0.35, pin, pout) / 0.4
    c.set_U(U)
    return U


def run_steps(c, n):
    t = 0.0
    for _ in range(n):
        dt, err = c.calc_timestep()
        assert err == 0
        c.timestep(t, dt)
        t += dt
    return c.get_U()


def pressure(U):
    return 0.4 * (U[..., 4] - 0.5 * (U[..., 1:4] ** 2).sum(-1) / U[..., 0])


def test_nfvse_corr_lserk_raises_alpha_and_conserves():
    """carpenterrk4-5: with the correction, elements whose density or pressure would drop below
    PositCorrFactor of the subcell-FV update get a larger alpha: the run differs from the uncorrected
    one, stays conservative (the correction moves U along F_FV - F_DG, whose integral vanishes on an
    element), and no safe state is inadmissible."""
    res = {}
    for corr in (0, 1):
        c = OracleCase(nfvse_corr=corr, time_disc=0, **CORR_BOX)
        U0 = corr_blast(c)
        U = run_steps(c, 4)
        assert c.corr_error == 0
        drift = integral(c, U - U0)
        assert np.abs(drift).max() <= 1e-12 * np.abs(integral(c, U0)).max()
        res[corr] = (U, c.alpha())
    assert np.abs(res[1][0] - res[0][0]).max() > 1e-6
    assert res[1][1].max() <= 1.0
    assert res[1][0][..., 0].min() > 0 and pressure(res[1][0]).min() > 0


def test_nfvse_corr_ssprk45_keeps_a_failing_run_positive():
    """ssprk4-5 at CFLScale 0.5 on the factor-100 blast: without the correction the first step leaves a
    NaN density (CALCTIMESTEP errType 1); with it six steps run with positive density and pressure,
    conserved totals and admissible safe states."""
    c = OracleCase(nfvse_corr=0, time_disc=8, **dict(CORR_BOX, cfl_scale=0.5))
    corr_blast(c)
    dt, err = c.calc_timestep()
    c.timestep(0.0, dt)
    assert c.calc_timestep()[1] == 1
    c = OracleCase(nfvse_corr=1, time_disc=8, **dict(CORR_BOX, cfl_scale=0.5))
    U0 = corr_blast(c)
    U = run_steps(c, 6)
    assert c.corr_error == 0
    assert U[..., 0].min() > 0 and pressure(U).min() > 0
    assert np.abs(integral(c, U - U0)).max() <= 1e-12 * np.abs(integral(c, U0)).max()


def test_nfvse_corr_is_inactive_on_smooth_data():
    """On smooth data no element needs a correction: the corrected and uncorrected runs are identical
    bit for bit (every element's FV flux is computed, but blended with alpha = 0)."""
    out = []
    for corr in (0, 1):
        c = OracleCase(nfvse_corr=corr, **dict(CORR_BOX, ini_exact_func=2, ini_amplitude=0.1, cfl_scale=0.9))
        out.append(run_steps(c, 3))
    assert np.array_equal(out[0], out[1])
