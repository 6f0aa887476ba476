"""Generates tests/golden/hopr_*.h5: the reference's periodic conforming HOPR test meshes
(tests/meshes/ConformBoxHeavilyWarped_Ngeo3__03_03_03_mesh.h5, 27 curved hexahedra of degree 3
with periodic boundaries, the mesh of most of the reference's regression runs, and
tests/meshes/ConformBoxUnstructPeriodicHeavilyWarped_Ngeo2_mesh.h5, 20 unstructured hexahedra
of degree 2) rewritten with the datasets and attributes that ReadMesh reads
(src/mesh/mesh_readin.f90:168-511), so that tests can use them where the reference tree is
absent.  The datasets are copied unchanged; the files are written by fluxo_b200.h5lite.

Run from the repository root, with the reference tree available:
    python tests/golden/make_hopr_fixtures.py /path/to/reference
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from fluxo_b200.h5lite import H5File, write_h5  # noqa: E402

MESHES = {
    "hopr_ConformBoxHeavilyWarped_Ngeo3_03_03_03.h5": "tests/meshes/ConformBoxHeavilyWarped_Ngeo3__03_03_03_mesh.h5",
    "hopr_ConformBoxUnstructPeriodicHeavilyWarped_Ngeo2.h5":
        "tests/meshes/ConformBoxUnstructPeriodicHeavilyWarped_Ngeo2_mesh.h5",
}
DATASETS = ("ElemInfo", "SideInfo", "NodeCoords", "BCNames", "BCType")
ATTRS = ("Version", "Ngeo", "nElems", "nSides", "nNodes", "nUniqueSides", "nUniqueNodes", "nBCs", "OutputNodeType")


def convert(src, dst):
    f = H5File(src)
    data = {k: f.read(k) for k in DATASETS}
    data["BCNames"] = np.array([x.split(b"\0", 1)[0].rstrip() for x in data["BCNames"]], dtype="S255")
    attrs = {k: f.attrs[k] for k in ATTRS if k in f.attrs}
    write_h5(dst, data, attrs)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    for out, rel in MESHES.items():
        convert(os.path.join(ref, rel), os.path.join(HERE, out))
        print("wrote", out)
