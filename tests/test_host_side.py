"""Host side of the product without a GPU: the C ABI library loads and exports every entry point
of include/fluxo_gpu.h, rejects bad configurations with FLUXO_EINVAL_CFG, and its host setup
(periodic box mesh, curl metrics, exact functions) agrees with the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

import fluxo_b200 as fb
from fluxo_b200 import _lib
from fluxo_b200.params import parse_ini, resolve, to_cfg_fields
from oracle.oracle import OracleCase

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_exports_match_header():
    hdr = open(os.path.join(ROOT, "include", "fluxo_gpu.h")).read()
    names = set(re.findall(r"^int (fluxo_\w+)\(", hdr, re.M))
    assert len(names) >= 20
    lib = fb.load()
    for n in names:
        assert hasattr(lib, n), n
    assert names == set(_lib.EXPORTS)


def test_invalid_config_fails_loudly():
    lib = fb.load()
    for bad in (dict(N=0), dict(N=8), dict(riemann=77), dict(volume_flux=11), dict(riemann=25), dict(time_disc=10), dict(time_disc=-1),
                dict(eqn=1, lifting=3), dict(kappa=1.0), dict(eqn=2, riemann=5, volume_flux=10, mu_0=2.0),
                dict(eqn=2, riemann=6, volume_flux=10)):
        cfg = fb.make_cfg(**bad)
        h = ctypes.c_void_p()
        r = lib.fluxo_gpu_create(ctypes.byref(cfg), ctypes.byref(h))
        assert r == -1, bad
        assert _lib.last_error(None)
    cfg = fb.make_cfg()
    cfg.struct_size = 8
    assert lib.fluxo_gpu_create(ctypes.byref(cfg), ctypes.byref(ctypes.c_void_p())) == -1


@pytest.mark.parametrize("N,NGeo,ne,amp", [(3, 2, (3, 3, 3), 0.1), (7, 2, (2, 2, 3), 0.05), (4, 3, (2, 3, 2), 0.05),
                                           (3, 4, (2, 2, 2), 0.05), (2, 1, (4, 2, 3), 0.0)])
def test_box_mesh_matches_oracle(N, NGeo, ne, amp):
    lo, hi = (-np.pi,) * 3, (np.pi,) * 3
    m = fb.box_mesh(N, ne, lo, hi, NGeo=NGeo, deform_amp=amp)
    mo = OracleCase(N=N, nElems=ne, xmin=lo, xmax=hi, NGeo=NGeo, deform_amp=amp).mesh()
    for k, ref in mo.items():
        if ref.dtype.kind == "i":
            assert np.array_equal(m[k], ref), k
        else:
            assert np.abs(m[k] - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max()), k


@pytest.mark.parametrize("N,NGeo,ne,amp", [(3, 2, (3, 3, 3), 0.1), (7, 2, (2, 2, 3), 0.05), (4, 3, (2, 3, 2), 0.05),
                                           (1, 2, (2, 2, 2), 0.05), (2, 1, (4, 2, 3), 0.0)])
def test_gauss_box_mesh_matches_oracle(N, NGeo, ne, amp):
    """Gauss nodes: metric terms, Jacobian and side vectors at the Gauss points, and SurfMetrics, against the
    oracle's restatement of CalcMetrics / CalcSurfMetrics with NodeType 'GAUSS'."""
    lo, hi = (-np.pi,) * 3, (np.pi,) * 3
    m = fb.box_mesh(N, ne, lo, hi, NGeo=NGeo, deform_amp=amp, node_type=1)
    mo = OracleCase(N=N, nElems=ne, xmin=lo, xmax=hi, NGeo=NGeo, deform_amp=amp, node_type=1).mesh()
    assert "SurfMetrics" in mo
    for k, ref in mo.items():
        if ref.dtype.kind == "i":
            assert np.array_equal(m[k], ref), k
        else:
            assert np.abs(m[k] - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), k


@pytest.mark.parametrize("func", [1, 2, 4, 7])
def test_exact_func_matches_oracle(func):
    c = OracleCase(N=2, nElems=(2, 2, 2), xmin=(-1, -1, -1), xmax=(1, 1, 1), ini_exact_func=func,
                   ref_state=(1.1, 0.2, -0.3, 0.1, 0.8), adv_vel=(0.5, 0.2, -0.1), ini_amplitude=0.2)
    x = np.random.default_rng(0).uniform(-1, 1, (50, 3))
    u = fb.exact_func(func, 0.3, x, adv_vel=(0.5, 0.2, -0.1), amplitude=0.2, ref_state=(1.1, 0.2, -0.3, 0.1, 0.8))
    assert np.allclose(u, c.exact(func, 0.3, x), rtol=1e-14, atol=1e-14)


def test_parameter_ini():
    txt = """
    ! Taylor-Green vortex
    N            = 7
    BoxElems     = (/32,32,32/)   # elements
    Riemann      = 44
    VolumeFlux   = 5
    mu0          = 6.25d-4
    IniExactFunc = 7
    CFLScale     = 0.9
    DFLScale     = 0.4
    TimeDiscMethod = CarpenterRK4-5
    Lifting      = br2
    tEnd         = 1.0
    """
    r = resolve(parse_ini(txt))
    assert r["boxelems"] == (32, 32, 32) and r["n"] == 7 and abs(r["mu0"] - 6.25e-4) < 1e-18
    f = to_cfg_fields(r)
    assert f["riemann"] == 44 and f["volume_flux"] == 5 and f["lifting"] == 2 and f["time_disc"] == 0
    assert f["eqn"] == 1 and f["lifting_var"] == 3
    with pytest.raises(KeyError):
        resolve(parse_ini("Riemann = 1"))


def test_parameter_ini_mhd_and_shock_capturing():
    txt = """
    N = 4
    Equation = mhd
    RefState = (/1., 0., 0., 0., 1., 1., 0., 0./)
    RefState = (/1.2, 0.1, 0., 0., 0.9, 1., 0., 0./)
    IniRefState = 2
    Riemann = 14
    VolumeFlux = 10
    eta = 1.0d-3
    GLM_scale = 0.4
    nfvse = T
    ComputeAlpha = 1
    SubFVMethod = 2
    ReconsBoundaries = 3
    ShockIndicatorQuantity = Pressure
    alpha_max = 0.6
    CFLScale = 0.5
    """
    r = resolve(parse_ini(txt))
    assert abs(r["kappa"] - 5 / 3) < 1e-15 and len(r["refstates"]) == 2
    f = to_cfg_fields(r)
    assert f["eqn"] == 3 and f["riemann"] == 14 and f["volume_flux"] == 10 and f["eta"] == 1e-3
    assert f["nfvse"] == 1 and f["sub_fv_method"] == 2 and f["recons_boundaries"] == 3
    assert f["indicator_quantity"] == 2 and f["alpha_max"] == 0.6 and f["glm_scale"] == 0.4
    assert to_cfg_fields(resolve(parse_ini("N = 3\nCFLScale = 0.9")))["kappa"] == 1.4
    with pytest.raises(ValueError):
        to_cfg_fields(resolve(parse_ini(txt.replace("Pressure", "Entropy"))))


@pytest.mark.parametrize("func", [1, 3, 201, 311, 312])
def test_mhd_exact_func_matches_oracle(func):
    from fluxo_b200.workloads import mhd_exact_func
    ref = ((1.2, 0.1, 0.0, 0.1, 0.9, 1.0, 1.0, 1.0), (1.1, 0.2, -0.1, 0.2, 0.6, 1.0, 1.0, 1.0))
    c = OracleCase(eqn=2, N=3, nElems=(2, 2, 2), xmin=(-1, -1, -1), xmax=(1, 1, 1), NGeo=2, deform_amp=0.05,
                   kappa=5 / 3, mhd_ref_state=ref, ini_exact_func=func, ini_center=(0.1, 0.0, 0.0),
                   ini_halfwidth=0.3, ini_amplitude=0.1)
    U = mhd_exact_func(func, 0.0, c.mesh()["Elem_xGP"], kappa=5 / 3, ref_states=ref, ini_ref_state=1,
                       center=(0.1, 0.0, 0.0), halfwidth=0.3, amplitude=0.1)
    assert np.allclose(U, c.get_U(), rtol=1e-13, atol=1e-14)
