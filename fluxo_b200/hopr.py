"""HOPR mesh files and FLUXO State files: the reference's ``MeshFile`` and restart input/output.

* ``read_mesh(path)`` reads the datasets ReadMesh needs (src/mesh/mesh_readin.f90:168-511:
  ElemInfo, SideInfo, NodeCoords, BCNames, BCType and the attributes Ngeo, nUniqueSides,
  OutputNodeType);
* ``mesh_arrays(N, raw, ...)`` turns them into the reference-layout mesh arrays (connectivity,
  metrics, face geometry) through the C ABI ``fluxo_host_hopr_mesh``;
* ``read_state`` / ``write_state`` read and write State files with the attributes and the
  ``DG_Solution`` dataset of WriteState / GenerateFileSkeleton (src/io_hdf5/hdf5_output.f90:74-160)
  for restarts (src/restart/restart.f90:60-200); ``restart_state`` interpolates a state of lower
  degree or of the other node set onto the run's nodes.

HDF5 access goes through ``h5lite`` (the format subset these files use).
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from .h5lite import H5File, write_h5

__all__ = ["read_mesh", "mesh_arrays", "load_mesh", "read_state", "write_state", "state_file_name", "nodes",
           "restart_state"]

def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def read_mesh(path, boundary_types=None):
    """Arrays of a HOPR mesh file.

    ``boundary_types`` maps a ``BoundaryName`` to a ``BoundaryType`` (type, state) that replaces
    the entries of every file BC whose name contains it, as readBCs does (mesh_readin.f90:62-157):
    the last matching name wins, a name that matches nothing and a remap of a non-periodic BC to
    periodic (type 1) are errors.
    Returns ElemInfo (nElems, 6), SideInfo (nSideInfo, 5), BCType (nBCs, 4), BCNames, NodeCoords
    ((NGeo+1)^3 * nElems, 3), NGeo, nUniqueSides and nodes_gl (OutputNodeType GAUSS-LOBATTO)."""
    f = H5File(path)
    ei = f.read("ElemInfo")
    if ei.ndim != 2 or ei.shape[1] != 6:
        raise ValueError("%s: ElemInfo must have 6 entries per element" % path)
    names = [str(x) for x in _names(f.read("BCNames"))] if "BCNames" in f else []
    bct = _i32(f.read("BCType")) if "BCType" in f else np.zeros((0, 4), np.int32)
    if boundary_types:
        user = [(str(k).strip(), tuple(int(x) for x in v)) for k, v in boundary_types.items()]
        found = [False] * len(user)
        bct = bct.copy()
        for i, name in enumerate(names):
            hit = None
            for j, (un, _) in enumerate(user):
                if un in name.strip():
                    hit = j
                    found[j] = True
            if hit is None:
                continue
            typ, state = user[hit][1][0], (user[hit][1][1] if len(user[hit][1]) > 1 else 0)
            if typ == 1 and bct[i, 0] != 1:
                raise ValueError("%s: remapping non-periodic to periodic BCs is not possible (%s)" % (path, name))
            bct[i, 0], bct[i, 2] = typ, state
        for (un, _), ok in zip(user, found):
            if not ok:
                raise ValueError("%s: boundary condition %r of the parameter file not found" % (path, un))
    node_type = f.attr("OutputNodeType", "EQUIDISTANT")
    if node_type not in ("EQUIDISTANT", "GAUSS-LOBATTO"):
        raise ValueError("%s: OutputNodeType must be EQUIDISTANT or GAUSS-LOBATTO, not %r" % (path, node_type))
    return dict(
        ElemInfo=_i32(ei), SideInfo=_i32(f.read("SideInfo")), BCType=bct, BCNames=names,
        NodeCoords=np.ascontiguousarray(f.read("NodeCoords"), dtype=np.float64), NGeo=int(f.attr("Ngeo")),
        nUniqueSides=int(f.attr("nUniqueSides")), nodes_gl=int(node_type == "GAUSS-LOBATTO"),
        path=os.path.abspath(str(path)),
    )


def _names(a):
    out = []
    for x in np.atleast_1d(a):
        s = x.decode("ascii") if isinstance(x, (bytes, np.bytes_)) else str(x)
        out.append(s.split("\0", 1)[0].rstrip())
    return out


def mesh_arrays(N, raw, node_type=2, mesh_scale=1.0, use_curveds=True):
    """Reference-layout mesh arrays (the keys of ``solver.box_mesh``) of a HOPR mesh read by
    ``read_mesh``; node_type 1 (Gauss nodes) adds ``SurfMetrics``."""
    lib = _lib.load()
    ei, si, bct = _i32(raw["ElemInfo"]), _i32(raw["SideInfo"]), _i32(raw["BCType"])
    X = np.ascontiguousarray(raw["NodeCoords"], dtype=np.float64)
    nE = ei.shape[0]
    nS = 3 * nE
    n = N + 1
    m = dict(
        SideToElem=np.zeros((nS, 5), np.int32), ElemToSide=np.zeros((nE, 6, 2), np.int32),
        Metrics_fTilde=np.zeros((nE, n, n, n, 3)), Metrics_gTilde=np.zeros((nE, n, n, n, 3)),
        Metrics_hTilde=np.zeros((nE, n, n, n, 3)), sJ=np.zeros((nE, n, n, n)),
        NormVec=np.zeros((nS, n, n, 3)), TangVec1=np.zeros((nS, n, n, 3)), TangVec2=np.zeros((nS, n, n, 3)),
        SurfElem=np.zeros((nS, n, n)), Elem_xGP=np.zeros((nE, n, n, n, 3)),
    )
    ng = int(raw["NGeo"]) + 1
    if X.shape != (ng ** 3 * nE, 3):
        raise ValueError("NodeCoords must hold (NGeo+1)^3 points per element")
    sm = np.zeros((nE, 6, n, n, 3)) if node_type == 1 else None
    if sm is not None:
        m["SurfMetrics"] = sm
    vp = ctypes.c_void_p
    ptr = lambda a: a.ctypes.data_as(vp) if a is not None else None  # noqa: E731
    r = lib.fluxo_host_hopr_mesh(
        int(N), int(node_type), nE, ptr(ei), si.shape[0], ptr(si), bct.shape[0], ptr(bct), int(raw["NGeo"]),
        int(raw.get("nodes_gl", 0)), ptr(X), float(mesh_scale), int(bool(use_curveds)),
        *[ptr(m[k]) for k in ("SideToElem", "ElemToSide", "Metrics_fTilde", "Metrics_gTilde", "Metrics_hTilde", "sJ",
                               "NormVec", "TangVec1", "TangVec2", "SurfElem", "Elem_xGP")], ptr(sm))
    _lib.check(r)
    return m


def load_mesh(path, N, node_type=2, mesh_scale=1.0, use_curveds=True, boundary_types=None):
    """``read_mesh`` + ``mesh_arrays``."""
    return mesh_arrays(N, read_mesh(path, boundary_types), node_type, mesh_scale, use_curveds)


def state_file_name(project, t, file_type="State"):
    """TIMESTAMP(ProjectName_FileType, t).h5 of the reference (src/globals/globals.f90)."""
    return "%s_%s_%017.9f.h5" % (project, file_type, t)


def read_state(path):
    """A State file: U (nElems, N+1, N+1, N+1, nVar: the C view of DG_Solution(nVar,0:N,0:N,0:N,nElems)),
    Time, N, NodeType, MeshFile, Project_Name and VarNames."""
    f = H5File(path)
    U = f.read("DG_Solution")
    if U.ndim != 5:
        raise ValueError("%s: DG_Solution must have rank 5" % path)
    return dict(U=np.ascontiguousarray(U, dtype=np.float64), Time=float(f.attr("Time")), N=int(f.attr("N")),
                NodeType=str(f.attr("NodeType", "GAUSS-LOBATTO")), MeshFile=f.attr("MeshFile", ""),
                Project_Name=f.attr("Project_Name", ""), VarNames=f.attr("VarNames", []),
                File_Type=f.attr("File_Type", ""))


def nodes(N, node_type):
    """1D nodes of degree N: node_type 1 Gauss, 2 Gauss-Lobatto (C ABI ``fluxo_host_nodes``)."""
    x = np.zeros(N + 1)
    _lib.check(_lib.load().fluxo_host_nodes(int(N), int(node_type), x.ctypes.data_as(ctypes.c_void_p), None))
    return x


def _interp_matrix(x_in, x_out):
    """Lagrange interpolation from x_in to x_out (InitializeVandermonde with barycentric weights,
    interpolation/basis.f90); a point on a node takes that node's value."""
    w = np.array([1.0 / np.prod([xi - xj for j, xj in enumerate(x_in) if j != i]) for i, xi in enumerate(x_in)])
    V = np.zeros((len(x_out), len(x_in)))
    for o, y in enumerate(x_out):
        hit = np.nonzero(np.abs(y - x_in) <= 2.220446049250313e-16 * np.maximum(np.abs(y), np.abs(x_in)))[0]
        if hit.size:
            V[o, hit[0]] = 1.0
            continue
        t = w / (y - x_in)
        V[o] = t / t.sum()
    return V


def restart_state(st, N, node_type):
    """The restart state on (N, node_type) from a State file's (read_state) solution: unchanged when N and
    the node set match, else interpolated with the Lagrange Vandermonde (Restart, restart.f90:150-217, the
    case N_Restart <= N).  N_Restart > N projects J*U modally with the Jacobian at 3*NGeo points, which
    this host setup does not keep: refused."""
    U = np.asarray(st["U"])
    n_in = int(st["N"])
    t_in = 1 if str(st.get("NodeType", "GAUSS-LOBATTO")).strip().upper() == "GAUSS" else 2
    if n_in == N and t_in == node_type:
        return U
    if n_in > N:
        raise ValueError("restart from N=%d onto N=%d (projection with the Jacobian) is not implemented" % (n_in, N))
    V = _interp_matrix(nodes(n_in, t_in), nodes(N, node_type))
    # ChangeBasis3D on the C view [elem][k][j][i][var]: i, then j, then k
    out = np.einsum("ai,ekjiv->ekjav", V, U)
    out = np.einsum("bj,ekjav->ekbav", V, out)
    return np.ascontiguousarray(np.einsum("ck,ekbav->ecbav", V, out))


_VARNAMES = {5: ["Density", "MomentumX", "MomentumY", "MomentumZ", "EnergyStagnationDensity"],
             9: ["Density", "MomentumX", "MomentumY", "MomentumZ", "TotalEnergy", "MagneticFieldX",
                 "MagneticFieldY", "MagneticFieldZ", "Psi"]}


def write_state(path, U, t, mesh_file, project, node_type="GAUSS-LOBATTO", next_time=None, var_names=None,
                file_type="State"):
    """Writes a State file with WriteState's header attributes and DG_Solution (U in the C view)."""
    U = np.ascontiguousarray(U, dtype=np.float64)
    if U.ndim != 5 or not (U.shape[1] == U.shape[2] == U.shape[3]):
        raise ValueError("U must have shape (nElems, N+1, N+1, N+1, nVar)")
    N = U.shape[1] - 1
    names = var_names or _VARNAMES.get(U.shape[4], ["Var%d" % i for i in range(U.shape[4])])
    attrs = {"Program": "Fluxo", "File_Type": file_type, "Project_Name": project, "File_Version": 0.1,
             "N": np.int32(N), "Time": float(t), "MeshFile": str(mesh_file),
             "NextFile": state_file_name(project, next_time if next_time is not None else t, file_type),
             "NodeType": node_type, "VarNames": list(names)}
    write_h5(path, {"DG_Solution": U}, attrs)
