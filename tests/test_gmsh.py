"""gmsh v4.1 ingestion (csrc/host/gmsh.cpp, dopamine_b200/meshio.py) against the reference
reader's rules (src/mesh/mod_gmsh_reader.f90:gmsh_read): a hand-written file exercising the
section layout, and round trips of the generated meshes through the writer.  Host code only."""
import numpy as np
import pytest

from dopamine_b200 import abi, cases, meshio
from dopamine_b200.solver import DopamineError

# Two tets sharing the face (2, 3, 4) and a 10-node tet on the far side of (2, 3, 5) whose mid-
# edge nodes are listed but unused; node tags are sparse and split over two entity blocks;
# physical groups out of tag order, one with a quoted name with spaces, one (tag 7) without faces.
TWO_TETS = """$MeshFormat
4.1 0 8
$EndMeshFormat
$PhysicalNames
4
2 7 "unused"
2 12 "outer wall"
2 3 "cap"
3 1 "fluid"
$EndPhysicalNames
$Entities
1 1 2 1
1 0 0 0 0
1 0 0 0 1 0 0 0 2 1 -1
5 0 0 0 1 1 1 1 3 1 2 3
6 0 0 0 1 1 1 1 12 0
9 0 0 0 1 1 1 1 1 0
$EndEntities
$Nodes
2 11 10 110
0 1 0 1
10
0 0 0
3 9 0 10
20
30
40
50
60
70
80
90
100
110
1 0 0
0 1 0
0 0 1
1 1 1
0.5 0 0
0.5 0.5 0
0 0.5 0
0 0 0.5
0.5 0 0.5
0 0.5 0.5
$EndNodes
$Elements
6 9 1 10
0 1 15 1
1 10
1 1 1 1
2 10 20
2 6 2 3
3 10 20 30
4 20 30 40
6 20 40 50
2 5 2 1
7 10 30 40
3 9 4 2
8 10 20 30 40
9 20 30 40 50
3 9 11 1
10 20 30 50 60 70 80 90 100 110 60
$EndElements
"""


def test_hand_written_file(tmp_path):
    p = tmp_path / "two_tets.msh"
    p.write_text(TWO_TETS)
    m = meshio.read_gmsh(p)
    # node tags 10..110 in file order -> 0..10
    assert m.xyz.shape == (11, 3) and np.array_equal(m.xyz[1], [1, 0, 0])
    # volume elements in file order; the 10-node tet by its four corners
    assert m.cell_type.tolist() == [4, 4, 4]
    assert m.cell_off.tolist() == [0, 4, 8, 12]
    assert m.cell_nodes.tolist() == [0, 1, 2, 3, 1, 2, 3, 4, 1, 2, 4, 5]
    # triangles in file order: patches are the 2-D groups holding faces, in $PhysicalNames order
    # ("unused" holds none): "outer wall" (tag 12, entity 6) -> 0, "cap" (tag 3, entity 5) -> 1
    assert m.patch_names == ["outer wall", "cap"]
    assert m.bface_off.tolist() == [0, 3, 6, 9, 12]
    assert m.bface_nodes.tolist() == [0, 1, 2, 1, 2, 3, 1, 3, 4, 0, 2, 3]
    assert m.bface_patch.tolist() == [0, 0, 0, 1]


@pytest.mark.parametrize("make", [lambda: cases.hybrid_config(n=4, kind="mixed").mesh,
                                  lambda: cases.hybrid_config(n=3, kind="tet").mesh,
                                  lambda: cases.urban_config(nx=24, ny=24, nz=12, n_blocks=4, lx=2.4, ly=2.4,
                                                             lz=0.72, scale=0.01).mesh],
                         ids=["mixed", "tet", "urban"])
def test_round_trip(tmp_path, make):
    m = make()
    p = tmp_path / "m.msh"
    meshio.write_gmsh(p, m)
    r = meshio.read_gmsh(p)
    for k in ("xyz", "cell_type", "cell_off", "cell_nodes"):
        assert np.array_equal(getattr(m, k), getattr(r, k)), k
    assert r.patch_names == m.patch_names

    def per_patch(mm):  # the writer groups faces by patch; within a patch the order is kept
        return [[tuple(mm.bface_nodes[mm.bface_off[i]:mm.bface_off[i + 1]]) for i in np.nonzero(mm.bface_patch == q)[0]]
                for q in range(len(mm.patch_names))]

    assert per_patch(r) == per_patch(m)


def _refused(tmp_path, text, status, words):
    p = tmp_path / "bad.msh"
    p.write_text(text)
    with pytest.raises(DopamineError) as e:
        meshio.read_gmsh(p)
    assert e.value.status == status
    assert words in str(e.value), str(e.value)


def test_refusals(tmp_path):
    with pytest.raises(DopamineError) as e:
        meshio.read_gmsh(tmp_path / "missing.msh")
    assert e.value.status == abi.ERR_ARG
    _refused(tmp_path, TWO_TETS.replace("4.1 0 8", "4.1 1 8"), abi.ERR_MESH, "binary")
    _refused(tmp_path, TWO_TETS.replace("4.1 0 8", "2.2 0 8"), abi.ERR_MESH, "format 4")
    # a second-order triangle (type 9) is not read
    _refused(tmp_path, TWO_TETS.replace("2 6 2 3\n", "2 6 9 3\n"), abi.ERR_MESH, "unsupported gmsh element type 9")
    # a triangle on an entity without a physical group, while groups exist
    _refused(tmp_path, TWO_TETS.replace("2 5 2 1\n", "2 4 2 1\n"), abi.ERR_MESH, "belongs to no 2-D physical group")
    _refused(tmp_path, TWO_TETS.replace("$Nodes", "$NodesX"), abi.ERR_MESH, "missing $Nodes")
    _refused(tmp_path, TWO_TETS.replace("7 10 30 40", "7 10 30 41"), abi.ERR_MESH, "unknown node")


def test_no_physical_names_gives_one_patch(tmp_path):
    text = TWO_TETS.split("$PhysicalNames")[0] + "$Entities" + TWO_TETS.split("$Entities")[1]
    p = tmp_path / "nophys.msh"
    p.write_text(text)
    m = meshio.read_gmsh(p)
    assert m.patch_names == ["boundary"] and m.bface_patch.tolist() == [0, 0, 0, 0]
