"""The oracle's two-point volume fluxes (VolumeFlux 0-10, 32) and Riemann solvers (every id of
navierstokes/equation.f90:291-406) checked on the properties the reference's fluxes are built to
have: consistency with the Euler flux, symmetry of the two-point fluxes, freestream preservation
on a warped mesh (the reference's job_def.py:1099-1118 criterion) and the exact resolution of a
stationary contact by the Roe and HLLC solvers."""
import numpy as np
import pytest

from oracle.oracle import OracleCase

KAPPA = 1.4
VOLUME_FLUXES = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 32]
RIEMANN = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 32, 33, 44]
CUBE = dict(xmin=(-1, -1, -1), xmax=(1, 1, 1))


def euler_flux(U, m):
    """Physical Euler flux f*m1 + g*m2 + h*m3 (navierstokes/flux.f90:56-110)."""
    rho, mom, E = U[0], U[1:4], U[4]
    v = mom / rho
    p = (KAPPA - 1) * (E - 0.5 * rho * v @ v)
    q = v @ m
    return np.array([rho * q, *(mom * q + p * m), (E + p) * q])


def cons(rho, v, p):
    v = np.asarray(v, float)
    return np.array([rho, *(rho * v), p / (KAPPA - 1) + 0.5 * rho * v @ v])


@pytest.fixture(scope="module")
def cases():
    return {vf: OracleCase(N=1, nElems=(1, 1, 1), volume_flux=vf, riemann=1, **CUBE) for vf in VOLUME_FLUXES}


@pytest.mark.parametrize("vf", VOLUME_FLUXES)
def test_volume_flux_consistent_and_symmetric(cases, vf):
    c = cases[vf]
    rng = np.random.default_rng(vf)
    for _ in range(5):
        UL = cons(1 + 0.3 * rng.random(), rng.standard_normal(3) * 0.5, 1 + 0.5 * rng.random())
        UR = cons(1 + 0.3 * rng.random(), rng.standard_normal(3) * 0.5, 1 + 0.5 * rng.random())
        mL, mR = rng.standard_normal(3), rng.standard_normal(3)
        F = c.volume_flux(UL, UL, mL, mL)
        assert np.allclose(F, euler_flux(UL, mL), rtol=1e-13, atol=1e-13)
        assert np.allclose(c.volume_flux(UL, UR, mL, mR), c.volume_flux(UR, UL, mR, mL), rtol=1e-13, atol=1e-14)


def _riemann_case(rs, vf=0):
    return OracleCase(N=1, nElems=(1, 1, 1), volume_flux=vf, riemann=rs, **CUBE)


@pytest.mark.parametrize("rs", RIEMANN)
def test_riemann_consistent(rs):
    """F*(U, U) = F(U).n for every solver (rotated frame n, t1, t2 orthonormal)."""
    c = _riemann_case(rs)
    rng = np.random.default_rng(100 + rs)
    for _ in range(4):
        U = cons(1 + 0.3 * rng.random(), rng.standard_normal(3) * 0.4, 1 + 0.5 * rng.random())
        Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        n, t1, t2 = Q[:, 0], Q[:, 1], Q[:, 2]
        assert np.allclose(c.riemann(U, U, n, t1, t2), euler_flux(U, n), rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("vf", [0, 2, 3, 4])
def test_roe_consistent_with_every_baseline_flux(vf):
    c = _riemann_case(3, vf)
    U = cons(1.2, [0.3, -0.2, 0.1], 0.9)
    n = np.array([1.0, 0, 0])
    assert np.allclose(c.riemann(U, U, n, np.array([0, 1.0, 0]), np.array([0, 0, 1.0])), euler_flux(U, n),
                       rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("rs", [3, 2])
def test_stationary_contact_resolved_exactly(rs):
    """Roe and HLLC keep a density jump at rest with equal pressure: F = (0, p n, 0)."""
    c = _riemann_case(rs)
    UL, UR = cons(1.0, [0, 0, 0], 1.0), cons(0.125, [0, 0, 0], 1.0)
    e = np.eye(3)
    F = c.riemann(UL, UR, e[0], e[1], e[2])
    assert np.allclose(F, [0, 1.0, 0, 0, 0], atol=1e-14)


def test_hllem_less_diffusive_than_hlle_on_contact():
    UL, UR = cons(1.0, [0, 0, 0], 1.0), cons(0.125, [0, 0, 0], 1.0)
    e = np.eye(3)
    F23 = _riemann_case(23).riemann(UL, UR, e[0], e[1], e[2])
    F24 = _riemann_case(24).riemann(UL, UR, e[0], e[1], e[2])
    assert abs(F24[0]) < 0.5 * abs(F23[0]) and F23[0] > 0


def test_llf_variants_add_the_side_maximum_dissipation():
    """Riemann 15/17/18/19/21 = the point flux of 7/11/12/8/20 minus lambda_max/2 (U_R - U_L)."""
    UL, UR = cons(1.0, [0.2, 0.1, 0], 1.0), cons(0.8, [0.1, 0, 0.2], 0.7)
    e = np.eye(3)
    for llf, plain in ((15, 7), (17, 11), (18, 12), (19, 8), (21, 20)):
        Fl = _riemann_case(llf).riemann(UL, UR, e[0], e[1], e[2])
        Fp = _riemann_case(plain).riemann(UL, UR, e[0], e[1], e[2])
        lam = max(abs(UL[1] / UL[0]), abs(UR[1] / UR[0])) + np.sqrt(
            max(KAPPA * (KAPPA - 1) * (U[4] / U[0] - 0.5 * (U[1:4] @ U[1:4]) / U[0] ** 2) for U in (UL, UR)))
        assert np.allclose(Fl, Fp - 0.5 * lam * (UR - UL), rtol=1e-13, atol=1e-14)


@pytest.mark.parametrize("vf", VOLUME_FLUXES)
def test_freestream_every_volume_flux(vf):
    """Warped NGeo=3 mesh, constant state: Ut = 0 to 1e-11 (job_def.py:1099-1103)."""
    c = OracleCase(N=3, nElems=(2, 2, 2), NGeo=3, deform_amp=0.1, ini_exact_func=1, riemann=1, volume_flux=vf,
                   **CUBE)
    assert np.abs(c.dg_time_derivative(0.0)).max() < 1e-11


@pytest.mark.parametrize("rs", RIEMANN)
def test_freestream_every_riemann(rs):
    c = OracleCase(N=2, nElems=(2, 2, 2), NGeo=2, deform_amp=0.1, ini_exact_func=1, riemann=rs, volume_flux=1,
                   **CUBE)
    assert np.abs(c.dg_time_derivative(0.0)).max() < 1e-11
