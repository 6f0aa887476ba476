"""The CPU oracle pinned on the reference's own regression criteria (tests/job_def.py of the
reference: freestream L_inf, dSdU*Ut entropy conservation / stability, convergence order) and on
known answers (LGL nodes and weights, SBP properties, Taylor-Green initial integrals)."""
import json
import os

import numpy as np
import pytest

from oracle.oracle import OracleCase, basis, ln_mean

GOLD = os.path.join(os.path.dirname(__file__), "golden", "lgl_kat.json")
CUBE = dict(xmin=(-1, -1, -1), xmax=(1, 1, 1))


@pytest.mark.parametrize("N", range(1, 9))
def test_lgl_known_answers(N):
    kat = json.load(open(GOLD))
    b = basis(N)
    assert np.allclose(b["xGP"], kat[str(N)]["x"], atol=2e-15, rtol=0)
    assert np.allclose(b["wGP"], kat[str(N)]["w"], atol=2e-15, rtol=0)
    if str(N) in kat["closed_form"]:
        assert np.allclose(b["xGP"], kat["closed_form"][str(N)]["x"], atol=1e-15)
        assert np.allclose(b["wGP"], kat["closed_form"][str(N)]["w"], atol=1e-15)


@pytest.mark.parametrize("N", [2, 3, 4, 7])
def test_sbp_operators(N):
    """D differentiates polynomials exactly; M*Dvolsurf is skew (dg/dg.f90:227-240);
    D_hat = -M^-1 D^T M."""
    b = basis(N)
    x, w = b["xGP"], b["wGP"]
    for p in range(N + 1):
        assert np.allclose(b["D"] @ x ** p, p * x ** max(p - 1, 0) if p else 0 * x, atol=1e-12)
    MD = np.diag(w) @ b["Dvolsurf"]
    assert np.allclose(MD, -MD.T, atol=1e-13)
    assert np.allclose(b["Dhat"], -np.diag(1 / w) @ b["D"].T @ np.diag(w), atol=1e-13)


def test_ln_mean_branches():
    for a, b in ((1.0, 1.0), (1.0, 1.0 + 1e-9), (1.0, 1.001), (1.0, 1.5), (0.2, 7.0)):
        ref = (b - a) / (np.log(b) - np.log(a)) if a != b else a
        assert abs(ln_mean(a, b) - ref) <= 1e-12 * ref


@pytest.mark.parametrize("eqn,NGeo", [(0, 1), (0, 3), (1, 2)])
def test_freestream_preservation(eqn, NGeo):
    """Reference criterion: freestream L_inf < 1e-11 on a warped mesh (job_def.py:1099-1103)."""
    c = OracleCase(N=3, nElems=(3, 3, 3), NGeo=NGeo, deform_amp=0.1, eqn=eqn, mu0=0.01, ini_exact_func=1,
                   riemann=1, volume_flux=1, **CUBE)
    Ut = c.dg_time_derivative(0.0)
    assert np.abs(Ut).max() < 1e-11
    t, n = c.run(0.0, 1.0, max_iter=3)
    assert n == 3
    assert c.analyze(t)["Linf"].max() < 1e-11


def _perturbed(rng, **kw):
    c = OracleCase(N=3, nElems=(3, 3, 3), NGeo=2, deform_amp=0.1, ini_exact_func=2, ini_amplitude=0.3,
                   adv_vel=(0.3, -0.2, 0.5), **CUBE, **kw)
    U = c.get_U()
    c.set_U(U * (1 + 0.05 * rng.standard_normal(U.shape)))
    return c


@pytest.mark.parametrize("vf,rs", [(10, 5), (5, 9), (32, 32)])
def test_entropy_conservation(vf, rs):
    """EC volume flux + EC surface flux: dS/dU*Ut = 0 to roundoff (job_def.py:1125-1131)."""
    c = _perturbed(np.random.default_rng(1), riemann=rs, volume_flux=vf)
    Ut = c.dg_time_derivative(0.0)
    a = c.analyze(0.0)
    assert abs(a["dSdU_Ut"]) < 1e-13 * max(1.0, np.abs(Ut).max())


@pytest.mark.parametrize("vf,rs", [(10, 4), (5, 44), (32, 33), (5, 1), (10, 22), (5, 13), (5, 16), (2, 14)])
def test_entropy_stability(vf, rs):
    """Entropy-stable surface fluxes only produce entropy (job_def.py:1133-1139)."""
    c = _perturbed(np.random.default_rng(2), riemann=rs, volume_flux=vf)
    c.dg_time_derivative(0.0)
    assert c.analyze(0.0)["dSdU_Ut"] < 1e-13


def test_convergence_order():
    """Density sine wave (IniExactFunc=2), N=3: L2 error decays at about N+1 (tests/convergence)."""
    errs = []
    for ne in (2, 4, 8):
        c = OracleCase(N=3, nElems=(ne, ne, ne), xmin=(0, 0, 0), xmax=(2, 2, 2), ini_exact_func=2, riemann=1,
                       volume_flux=10)
        t, _ = c.run(0.0, 0.2)
        errs.append(c.analyze(t)["L2"][0])
    eoc = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert eoc.mean() > 3.3 and eoc[-1] > 3.6


def test_taylor_green_initial_integrals():
    """TGV (IniExactFunc=7): mean kinetic energy 1/8 and enstrophy 3/8 at t=0."""
    c = OracleCase(N=5, nElems=(4, 4, 4), xmin=(-np.pi,) * 3, xmax=(np.pi,) * 3, eqn=1, mu0=1 / 1600.,
                   ini_exact_func=7, riemann=44, volume_flux=5)
    c.dg_time_derivative(0.0)
    a = c.analyze(0.0)
    assert abs(a["ekin"] - 0.125) < 1e-4
    assert abs(a["enstrophy"] - 0.375) < 5e-3


def test_br1_br2_differ_only_in_face_gradients():
    rng = np.random.default_rng(3)
    out = []
    for lift in (1, 2):
        c = _perturbed(np.random.default_rng(3), eqn=1, lifting=lift, mu0=0.01, riemann=1, volume_flux=5)
        out.append((c.dg_time_derivative(0.0), c.gradients()))
    assert np.allclose(out[0][1][0], out[1][1][0], atol=1e-12)  # same volume gradients
    assert np.abs(out[0][0] - out[1][0]).max() > 1e-6  # different face fluxes
    del rng


def test_calc_timestep_errors():
    c = OracleCase(N=2, nElems=(2, 2, 2), ini_exact_func=1, **CUBE)
    dt, err = c.calc_timestep()
    assert err == 0 and dt > 0
    U = c.get_U()
    U[1, 0, 0, 0, 4] = 0.0  # negative pressure in element 2
    c.set_U(U)
    assert c.calc_timestep()[1] == 2
    U[0, 1, 0, 0, 0] = np.nan  # NaN density in element 1 comes first
    c.set_U(U)
    assert c.calc_timestep()[1] == 1
