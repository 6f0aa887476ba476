"""HOPR mesh ingest and FLUXO State files on the CPU: the HDF5 subset reader and writer, the product's
connectivity and metrics from the reference's own periodic conforming test meshes against the oracle's
restatement of ReadMesh / setLocalSideIDs / fillMeshInfo / CalcMetrics, a geometric check of the side
flips that depends on neither (the face points of both elements of every side coincide), and the
reference's freestream and entropy-conservation criteria evaluated by the oracle on those meshes.

The meshes are tests/golden/hopr_*.h5 (made by tests/golden/make_hopr_fixtures.py from the
reference's tests/meshes); the reference's own files are read directly when the reference tree is
present.
"""
import os

import numpy as np
import pytest

import fluxo_b200 as fb
from fluxo_b200 import hopr
from fluxo_b200.h5lite import H5File, H5FormatError, write_h5
from fluxo_b200.params import parse_ini, resolve
from oracle.oracle import OracleCase

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
WARPED = os.path.join(GOLDEN, "hopr_ConformBoxHeavilyWarped_Ngeo3_03_03_03.h5")
UNSTRUCT = os.path.join(GOLDEN, "hopr_ConformBoxUnstructPeriodicHeavilyWarped_Ngeo2.h5")
REF = "/root/reference"
REF_MESHES = os.path.join(REF, "tests", "meshes")
REF_STATE = os.path.join(REF, "tests", "runs", "navst", "freestream", "conforming",
                         "NAVIERSTOKES_FREESTREAM_State_0000000.000000000.h5")
needs_ref = pytest.mark.skipif(not os.path.isdir(REF_MESHES), reason="reference tree not present")


def _flip_pq(N, p, q, flip):
    # the slave's point of master point (p,q), mappings.f90:262-300
    return [(p, q), (q, p), (N - p, q), (N - q, N - p), (p, N - q)][flip]


def _side_node(N, p, q, flip, side):
    # volume node (i,j,k) at layer 0 of local side `side` (CGNS orientation), mappings.f90:400-464
    a, b = _flip_pq(N, p, q, flip)
    return {1: (b, a, 0), 2: (a, 0, b), 3: (N, a, b), 4: (N - a, N, b), 5: (0, b, a), 6: (a, b, N)}[side]


@pytest.fixture(scope="module")
def warped():
    return hopr.read_mesh(WARPED)


@pytest.fixture(scope="module")
def unstruct():
    return hopr.read_mesh(UNSTRUCT)


# --- HDF5 subset -------------------------------------------------------------------------------
def test_h5_roundtrip(tmp_path):
    rng = np.random.default_rng(1)
    data = {"A": rng.standard_normal((4, 3, 2)), "I": np.arange(12, dtype=np.int32).reshape(3, 4),
            "S": np.array([b"alpha", b"be"], dtype="S8")}
    attrs = {"N": np.int32(7), "Time": 1.25, "Name": "BOX", "Vec": np.array([1.0, 2.0]), "L": ["x", "yz"]}
    p = tmp_path / "t.h5"
    write_h5(p, data, attrs)
    f = H5File(p)
    assert np.array_equal(f.read("A"), data["A"]) and np.array_equal(f.read("I"), data["I"])
    assert [x.rstrip(b"\0") for x in f.read("S")] == [b"alpha", b"be"]
    assert f.attr("N") == 7 and f.attr("Time") == 1.25 and f.attr("Name") == "BOX" and f.attr("L") == ["x", "yz"]
    assert np.array_equal(f.attr("Vec"), [1.0, 2.0])
    with pytest.raises(KeyError):
        f.read("missing")


def test_h5_rejects_non_hdf5(tmp_path):
    p = tmp_path / "x.h5"
    p.write_bytes(b"not an hdf5 file at all" * 4)
    with pytest.raises(H5FormatError):
        H5File(p)


@needs_ref
@pytest.mark.parametrize("name", sorted(n for n in os.listdir(REF_MESHES) if n.endswith(".h5"))
                         if os.path.isdir(REF_MESHES) else [])
def test_reference_meshes_read(name):
    """Every HOPR file the reference ships reads, with the sizes its attributes state."""
    f = H5File(os.path.join(REF_MESHES, name))
    ei, si, nc = f.read("ElemInfo"), f.read("SideInfo"), f.read("NodeCoords")
    assert ei.shape == (f.attr("nElems"), 6) and si.shape == (f.attr("nSides"), 5)
    assert nc.shape == (f.attr("nNodes"), 3) and f.attr("nNodes") == f.attr("nElems") * (f.attr("Ngeo") + 1) ** 3
    assert ei[-1, 3] == si.shape[0] and ei[-1, 5] == nc.shape[0]


@needs_ref
def test_fixtures_equal_reference_meshes():
    for fix, ref in ((WARPED, "ConformBoxHeavilyWarped_Ngeo3__03_03_03_mesh.h5"),
                     (UNSTRUCT, "ConformBoxUnstructPeriodicHeavilyWarped_Ngeo2_mesh.h5")):
        a, b = hopr.read_mesh(fix), hopr.read_mesh(os.path.join(REF_MESHES, ref))
        for k in ("ElemInfo", "SideInfo", "BCType", "NodeCoords"):
            assert np.array_equal(a[k], b[k]), k
        assert (a["BCNames"], a["NGeo"], a["nodes_gl"], a["nUniqueSides"]) == \
               (b["BCNames"], b["NGeo"], b["nodes_gl"], b["nUniqueSides"])


# --- connectivity and metrics --------------------------------------------------------------------
@pytest.mark.parametrize("N,node_type", [(1, 2), (3, 2), (4, 2), (7, 2), (3, 1), (4, 1)])
@pytest.mark.parametrize("mesh", ["warped", "unstruct"])
def test_hopr_mesh_matches_oracle(mesh, N, node_type, request):
    raw = request.getfixturevalue(mesh)
    m = hopr.mesh_arrays(N, raw, node_type=node_type)
    o = OracleCase(hopr=raw, N=N, eqn=1, node_type=node_type)
    assert o.nSides == raw["nUniqueSides"] == m["SideToElem"].shape[0]
    mo = o.mesh()
    for k, ref in mo.items():
        if ref.dtype.kind == "i":
            assert np.array_equal(m[k], ref), k
        else:
            assert np.abs(m[k] - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), k


@pytest.mark.parametrize("mesh", ["warped", "unstruct"])
def test_side_flips_join_the_same_points(mesh, request):
    """The face points of the master (flip 0) and the slave (its flip) of every side are the same points of
    the periodic box [-1,1]^3, up to a period: the side ids, flips and the side/volume maps agree with the
    geometry HOPR wrote."""
    raw = request.getfixturevalue(mesh)
    N = 3
    m = hopr.mesh_arrays(N, raw)
    x = m["Elem_xGP"]
    worst = 0.0
    for s, (e, nb, ls, nls, fl) in enumerate(m["SideToElem"]):
        for q in range(N + 1):
            for p in range(N + 1):
                i, j, k = _side_node(N, p, q, 0, ls)
                a = x[e - 1, k, j, i]
                i, j, k = _side_node(N, p, q, fl, nls)
                b = x[nb - 1, k, j, i]
                d = a - b
                d -= 2.0 * np.round(d / 2.0)
                worst = max(worst, np.abs(d).max())
    assert worst < 1e-12
    # ElemToSide is the inverse of SideToElem
    for s, (e, nb, ls, nls, fl) in enumerate(m["SideToElem"]):
        assert tuple(m["ElemToSide"][e - 1, ls - 1]) == (s + 1, 0)
        assert tuple(m["ElemToSide"][nb - 1, nls - 1]) == (s + 1, fl)


def test_outward_normals(warped):
    """NormVec of every side points out of its master element (towards the slave's centre, across the period)."""
    N = 3
    m = hopr.mesh_arrays(N, warped)
    c = m["Elem_xGP"].reshape(m["Elem_xGP"].shape[0], -1, 3).mean(axis=1)
    for s, (e, nb, ls, nls, fl) in enumerate(m["SideToElem"]):
        d = c[nb - 1] - c[e - 1]
        d -= 2.0 * np.round(d / 2.0)
        assert np.dot(m["NormVec"][s].reshape(-1, 3).mean(axis=0), d) > 0


def test_use_curveds_and_mesh_scale(warped):
    m1 = hopr.mesh_arrays(3, warped, use_curveds=False, mesh_scale=2.0)
    o = OracleCase(hopr=dict(warped, use_curveds=0, mesh_scale=2.0), N=3, eqn=1).mesh()
    for k in ("sJ", "Metrics_fTilde", "NormVec", "Elem_xGP"):
        assert np.abs(m1[k] - o[k]).max() <= 1e-12 * max(1.0, np.abs(o[k]).max()), k
    # trilinear elements of twice the size: |J| grows by 8
    m0 = hopr.mesh_arrays(3, warped, use_curveds=False)
    assert np.allclose(m1["sJ"] * 8.0, m0["sJ"], rtol=1e-12)


def test_refusals(warped, tmp_path):
    # readBCs: a remap to a non-periodic type turns the periodic sides into boundary sides
    with pytest.raises(fb.FluxoError, match="non-periodic"):
        hopr.mesh_arrays(3, hopr.read_mesh(WARPED, {"BC_": (2, 0)}))
    with pytest.raises(ValueError, match="not found"):
        hopr.read_mesh(WARPED, {"BC_nothing": (2, 0)})
    # a mortar side (negative neighbour id)
    bad = dict(warped)
    bad["SideInfo"] = warped["SideInfo"].copy()
    bad["SideInfo"][0, 2] = -1
    with pytest.raises(fb.FluxoError, match="mortar"):
        hopr.mesh_arrays(3, bad)
    # two oriented records of one side
    bad["SideInfo"] = warped["SideInfo"].copy()
    slave = np.nonzero(bad["SideInfo"][:, 1] < 0)[0][0]
    bad["SideInfo"][slave, 1] *= -1
    with pytest.raises(fb.FluxoError, match="oriented"):
        hopr.mesh_arrays(3, bad)


@needs_ref
def test_reference_mortar_and_wall_meshes_refused():
    with pytest.raises(fb.FluxoError, match="mortar"):
        hopr.load_mesh(os.path.join(REF_MESHES, "DeformedBoxMortarPeriodic__Ngeo_2_Level_01_mesh.h5"), 3)
    with pytest.raises(fb.FluxoError, match="non-periodic"):
        hopr.load_mesh(os.path.join(REF_MESHES, "ConformBoxUnstruct2_Ngeo2_mesh.h5"), 3)


# --- the reference's regression criteria on its mesh, evaluated by the oracle --------------------
def test_oracle_freestream_on_warped_mesh(warped):
    """navst/freestream/conforming: N=3, Riemann 1, VolumeFlux 1, RefState (1,.1,.2,-.3,20): Ut vanishes
    to round-off on the curved mesh (free-stream preservation of the curl-form metrics)."""
    o = OracleCase(hopr=warped, N=3, eqn=1, riemann=1, volume_flux=1, ini_exact_func=1,
                   ref_state=(1.0, 0.1, 0.2, -0.3, 20.0), mu0=1e-6)
    assert np.abs(o.dg_time_derivative()).max() < 1e-10


def test_oracle_freestream_run_to_t20(warped):
    """The same case marched with carpenterrk4-5 at CFLscale 0.9 / DFLscale 0.5 to tEnd = 20: L_inf < 1e-11, the
    reference's pass criterion for this run (tests/job_def.py)."""
    o = OracleCase(hopr=warped, N=3, eqn=1, riemann=1, volume_flux=1, ini_exact_func=1,
                   ref_state=(1.0, 0.1, 0.2, -0.3, 20.0), mu0=1e-6, cfl_scale=0.9, dfl_scale=0.5)
    t, n = o.run(0.0, 20.0)
    assert t == 20.0 and n > 1000
    assert o.analyze(t)["Linf"].max() < 1e-11


@pytest.mark.parametrize("riemann,vf,conserving", [(9, 5, True), (32, 32, True), (1, 5, False)])
def test_oracle_entropy_with_random_blending(warped, riemann, vf, conserving):
    """navst/softBlast/entropyCons, entropyCons_Ranocha and entropyStab: NFVSE with ComputeAlpha 20 (random
    blending, alpha_max 1) on the warped mesh; |dS/dU . Ut| < 1e-13 for the EC fluxes, < 1e-13 (signed) for LF."""
    o = OracleCase(hopr=warped, N=3, eqn=0, riemann=riemann, volume_flux=vf, ini_exact_func=14, nfvse=1,
                   compute_alpha=20, space_prop_sweeps=0, alpha_max=1.0, time_disc=8)
    o.dg_time_derivative()
    a = o.alpha()
    assert 0.1 < a.mean() < 0.9 and len(np.unique(a)) > 10  # a real mix of DG and subcell FV
    s = o.analyze(0.0)["dSdU_Ut"]
    if conserving:
        assert abs(s) < 1e-13
    else:
        assert s < 1e-13


# --- State files --------------------------------------------------------------------------------------
def test_state_roundtrip(tmp_path):
    U = np.random.default_rng(3).standard_normal((4, 3, 3, 3, 5))
    p = tmp_path / hopr.state_file_name("PROJ", 0.5)
    assert p.name == "PROJ_State_0000000.500000000.h5"
    hopr.write_state(p, U, 0.5, "mesh.h5", "PROJ", next_time=1.0)
    st = hopr.read_state(p)
    assert np.array_equal(st["U"], U) and st["Time"] == 0.5 and st["N"] == 2
    assert st["NodeType"] == "GAUSS-LOBATTO" and st["MeshFile"] == "mesh.h5" and st["Project_Name"] == "PROJ"
    assert st["VarNames"][0] == "Density" and H5File(p).attr("NextFile") == "PROJ_State_0000001.000000000.h5"


@needs_ref
def test_reference_state_file(warped):
    """The reference's restart file of navst/freestream/conforming holds IniExactFunc 1 of its RefState on the
    Gauss-Lobatto nodes of ConformBoxHeavilyWarped (N=3)."""
    st = hopr.read_state(REF_STATE)
    assert st["N"] == 3 and st["NodeType"] == "GAUSS-LOBATTO" and st["Time"] == 0.0
    assert st["MeshFile"].endswith("ConformBoxHeavilyWarped_Ngeo3__03_03_03_mesh.h5")
    m = hopr.mesh_arrays(3, warped)
    U0 = fb.exact_func(1, 0.0, m["Elem_xGP"], ref_state=(1.0, 0.1, 0.2, -0.3, 20.0))
    assert st["U"].shape == U0.shape and np.abs(st["U"] - U0).max() < 1e-13


def test_parameter_ini_mesh_keys():
    txt = """
    N = 3
    MeshFile = ../../../../meshes/ConformBoxHeavilyWarped_Ngeo3__03_03_03_mesh.h5
    useCurveds = F
    meshScale = 0.5
    BoundaryName = BC_zminus
    BoundaryType = (/1,0/)
    BoundaryName=BC_zplus
    BoundaryType=(/1,0/)
    CFLScale = 0.9
    ProjectName = NAVIERSTOKES_FREESTREAM
    """
    r = resolve(parse_ini(txt))
    assert r["meshfile"].endswith("03_03_03_mesh.h5") and r["usecurveds"] == "F" and r["meshscale"] == 0.5
    assert r["boundarytypes"] == {"BC_zminus": (1, 0), "BC_zplus": (1, 0)}
    assert r["projectname"] == "NAVIERSTOKES_FREESTREAM"


def test_nodes_match_the_golden_lgl_and_gauss():
    import json

    kat = json.load(open(os.path.join(GOLDEN, "lgl_kat.json")))
    for N in range(1, 9):
        assert np.allclose(hopr.nodes(N, 2), kat[str(N)]["x"], rtol=0, atol=1e-15)
        xg, _ = np.polynomial.legendre.leggauss(N + 1)
        assert np.allclose(hopr.nodes(N, 1), xg, rtol=0, atol=1e-15)


@pytest.mark.parametrize("n_in,t_in,n_out,t_out", [(3, 2, 3, 2), (3, 2, 5, 2), (2, 2, 4, 1), (4, 1, 4, 2), (3, 1, 6, 1)])
def test_restart_interpolation_is_exact_for_polynomials(n_in, t_in, n_out, t_out):
    """Restart with N_Restart <= N or the other node set (restart.f90:150-217): the Lagrange Vandermonde
    reproduces a polynomial of degree N_Restart at the new nodes."""
    f = lambda x, y, z: 1.0 + x ** n_in - 2.0 * y * z ** (n_in - 1) + 0.5 * x * y * z  # noqa: E731
    xi = hopr.nodes(n_in, t_in)
    U = np.zeros((3, n_in + 1, n_in + 1, n_in + 1, 5))
    for k in range(n_in + 1):
        for j in range(n_in + 1):
            for i in range(n_in + 1):
                U[:, k, j, i, :] = f(xi[i], xi[j], xi[k]) * np.arange(1, 6)
    st = dict(U=U, N=n_in, NodeType="GAUSS" if t_in == 1 else "GAUSS-LOBATTO")
    out = hopr.restart_state(st, n_out, t_out)
    xo = hopr.nodes(n_out, t_out)
    ref = np.array([[[f(xo[i], xo[j], xo[k]) for i in range(n_out + 1)] for j in range(n_out + 1)]
                    for k in range(n_out + 1)])
    assert out.shape == (3, n_out + 1, n_out + 1, n_out + 1, 5)
    assert np.abs(out[..., 2] - 3 * ref).max() < 1e-13
    if (n_in, t_in) == (n_out, t_out):
        assert out is st["U"] or np.array_equal(out, U)


def test_restart_from_higher_degree_is_refused():
    st = dict(U=np.zeros((1, 5, 5, 5, 5)), N=4, NodeType="GAUSS-LOBATTO")
    with pytest.raises(ValueError, match="not implemented"):
        hopr.restart_state(st, 3, 2)
