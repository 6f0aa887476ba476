"""Device-side analysis (fluxo_gpu_analyze) against the oracle's restatement of the reference's Analyze.

CalcErrorNorms (src/analyze/analyze.f90:557-632: L2 and L_inf on NAnalyze = 2(N+1) points, L2 at the
collocation points), CalcEntropy and dS/dU.Ut (navierstokes/analyze_equation.f90:549-599,
mhd/analyze_equation.f90:421-470) and the Taylor-Green integrands (kinetic energy and enstrophy,
testcase/taylorgreenvortex/testcase_analyze.f90:127-330), each computed on the GPU after a right-hand side
at the analysis time, as the reference's TimeDisc does (timedisc.f90:387-404).  Tolerance: relative
1e-12 (FP64 sums in another order).

The reference's own entropy criteria (tests/job_def.py:1120-1139, runs/navst/softBlast: soft blast,
N=3, curved mesh) are then checked on GPU output: |dS/dU.Ut| <= 1e-13 for entropy-conservative volume
and surface fluxes (EC-KEP with Riemann 9, Ranocha with Riemann 32, EC-KEP with NFVSE blending, Derigs
MHD with the EC surface flux), and dS/dU.Ut <= 1e-13 for the entropy-stable surface fluxes (LLF,
matrix dissipation)."""
import numpy as np
import pytest

import fluxo_b200 as fb
from oracle.oracle import OracleCase

pytestmark = pytest.mark.gpu
TOL = 1e-12


def rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)


def ns_pair(perturb=0.05, seed=0, **kw):
    c = OracleCase(**kw)
    if perturb:
        U = c.get_U()
        c.set_U(U * (1 + perturb * np.random.default_rng(seed).standard_normal(U.shape)))
    p = c.params
    op = fb.DGOperator(N=p.N, eqn=p.eqn, riemann=p.riemann, volume_flux=p.volume_flux, lifting=p.lifting,
                       lifting_var=p.lifting_var, visc=p.visc, kappa=p.kappa, R=p.R, Pr=p.Pr, mu0=p.mu0,
                       ini_exact_func=p.ini_exact_func, nfvse=p.nfvse, compute_alpha=p.compute_alpha,
                       shock_blend_coef=p.shock_blend_coef, alpha_max=p.alpha_max, alpha_min=p.alpha_min,
                       space_prop_sweeps=p.space_prop_sweeps)
    op.set_mesh(c.mesh())
    op.set_state(c.get_U())
    return c, op


def collocation_l2(op, c, mesh, exact_U):
    """sqrt(sum (U - U_exact)^2 wGPVol/sJ / Vol) at the nodes (the L_2_colloc of CalcErrorNorms)."""
    from oracle.oracle import basis

    w = basis(c.N)["wGP"]
    wv = w[None, :, None, None] * w[None, None, :, None] * w[None, None, None, :]  # [e][k][j][i]
    wgt = wv / mesh["sJ"]
    d = op.get_state() - exact_U
    return np.sqrt((d ** 2 * wgt[..., None]).sum(axis=(0, 1, 2, 3)) / wgt.sum())


def test_error_norms_density_wave(gpu_lib):
    kw = dict(N=3, nElems=(3, 3, 3), NGeo=2, deform_amp=0.1, xmin=(-1, -1, -1), xmax=(1, 1, 1), riemann=1,
              volume_flux=10, ini_exact_func=2, ini_amplitude=0.3, adv_vel=(0.3, -0.2, 0.5),
              ini_wavenumber=(1.0, 1.0, 1.0))
    c, op = ns_pair(perturb=0.01, **kw)
    t = 0.2
    c.dg_time_derivative(t)
    ref = c.analyze(t)
    ex = dict(func=2, adv_vel=(0.3, -0.2, 0.5), ini_wavenumber=(1.0, 1.0, 1.0), ini_amplitude=0.3)
    out = op.analyze(t, exact=ex)
    assert rel(out["L2"], ref["L2"]) <= TOL
    assert rel(out["Linf"], ref["Linf"]) <= TOL
    assert rel(out["entropy"], ref["entropy"]) <= TOL
    assert rel(out["ekin"], ref["ekin"]) <= TOL
    assert abs(out["dSdU_Ut"] - ref["dSdU_Ut"]) <= TOL * abs(ref["dSdU_Ut"]) + 1e-13
    m = c.mesh()
    Uex = c.exact(2, t, m["Elem_xGP"]).reshape(op.shape)
    assert rel(out["L2_colloc"], collocation_l2(op, c, m, Uex)) <= TOL
    assert abs(out["volume"] - 8.0) <= 1e-12 * 8.0


def test_taylor_green_integrands(gpu_lib):
    kw = dict(N=3, nElems=(2, 3, 2), NGeo=2, deform_amp=0.05, xmin=(-np.pi,) * 3, xmax=(np.pi,) * 3, eqn=1,
              mu0=0.02, lifting=1, lifting_var=3, riemann=44, volume_flux=5, ini_exact_func=7)
    c, op = ns_pair(perturb=0.02, **kw)
    c.dg_time_derivative(0.0)
    ref = c.analyze(0.0)
    out = op.analyze(0.0, exact=dict(func=7))
    for k in ("ekin", "enstrophy", "entropy"):
        assert rel(out[k], ref[k]) <= TOL, k
    assert rel(out["L2"], ref["L2"]) <= TOL
    assert abs(out["dSdU_Ut"] - ref["dSdU_Ut"]) <= TOL * abs(ref["dSdU_Ut"]) + 1e-13
    # the unperturbed initial state: kinetic energy 1/8 and enstrophy 3/8 of the Taylor-Green vortex,
    # to the discretisation error of this coarse mesh (2 x 3 x 2 elements at N=3: a few percent)
    c0, op0 = ns_pair(perturb=0.0, **kw)
    a0 = op0.analyze(0.0)
    assert abs(a0["ekin"] - 0.125) < 0.01 and abs(a0["enstrophy"] - 0.375) < 0.1


def test_mhd_entropy_and_energy(gpu_lib):
    from test_gpu_mhd import mhd_pair

    c, op = mhd_pair(N=3, volume_flux=10, riemann=14, noncons=1, nc_glm=0)
    c.glm_ch = op.glm_ch
    c.dg_time_derivative(0.0)
    ref = c.analyze(0.0)
    out = op.analyze(0.0)
    for k in ("ekin", "entropy"):
        assert rel(out[k], ref[k]) <= TOL, k
    assert abs(out["dSdU_Ut"] - ref["dSdU_Ut"]) <= TOL * abs(ref["dSdU_Ut"]) + 1e-13
    assert out["enstrophy"] == 0.0


BLAST = dict(N=3, nElems=(3, 3, 3), NGeo=3, deform_amp=0.1, xmin=(-1, -1, -1), xmax=(1, 1, 1), ini_exact_func=14)
EC_CASES = [
    dict(riemann=9, volume_flux=5),
    dict(riemann=32, volume_flux=32),
    dict(riemann=9, volume_flux=5, nfvse=1, compute_alpha=3, shock_blend_coef=0.5, space_prop_sweeps=0),
]


@pytest.mark.parametrize("case", EC_CASES, ids=["ec_kep_rs9", "ranocha_rs32", "ec_kep_rs9_nfvse"])
def test_entropy_conservation_on_gpu(gpu_lib, case):
    """|dS/dU.Ut| at roundoff (tests/job_def.py:1125-1131: 1e-13 absolute) for a perturbed soft blast, whose
    node noise makes every face carry a jump."""
    c, op = ns_pair(perturb=0.05, seed=3, **BLAST, **case)
    out = op.analyze(0.0)
    c.dg_time_derivative(0.0)
    ref = c.analyze(0.0)
    assert abs(out["dSdU_Ut"]) <= 1e-13, out["dSdU_Ut"]
    assert abs(ref["dSdU_Ut"]) <= 1e-13
    assert np.abs(op.get_ut()).max() > 10.0  # a right-hand side far from zero


@pytest.mark.parametrize("riemann", [1, 44, 22])
def test_entropy_stability_on_gpu(gpu_lib, riemann):
    """dS/dU.Ut <= 1e-13 (tests/job_def.py:1133-1139) with the EC-KEP volume flux and a dissipative
    surface flux, and the same value as the oracle."""
    c, op = ns_pair(perturb=0.05, seed=3, riemann=riemann, volume_flux=5, **BLAST)
    out = op.analyze(0.0)
    c.dg_time_derivative(0.0)
    ref = c.analyze(0.0)
    assert out["dSdU_Ut"] <= 1e-13 and out["dSdU_Ut"] < -1e-3
    assert rel(out["dSdU_Ut"], ref["dSdU_Ut"]) <= TOL


def test_mhd_entropy_conservation_on_gpu(gpu_lib):
    """Derigs EC volume flux with the EC surface flux (Riemann 11) and the Powell and GLM non-conservative
    terms: the mathematical entropy is conserved to roundoff on GPU output."""
    from test_gpu_mhd import mhd_pair

    c, op = mhd_pair(N=3, volume_flux=10, riemann=11, noncons=1, nc_glm=1)
    out = op.analyze(0.0)
    assert abs(out["dSdU_Ut"]) <= 1e-13, out["dSdU_Ut"]
