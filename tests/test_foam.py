"""OpenFOAM polyMesh ingestion (csrc/host/foam.cpp, dopamine_b200/meshio.py) and the polyhedral
set-up (csrc/host/mesh.cpp:build_mesh_poly) on the host, against the reference's foam_read rules
(src/mesh/mod_foam_reader.f90) and its polyhedral geometry (src/mesh/mod_mesh.f90:1336-1461).

* A hand-written polyMesh (two hexes, comments, a FoamFile header, a patch with nested entries)
  is read to the expected arrays; missing files, truncated binary data and compact offsets that
  do not start at 0 are refused.
* Element meshes converted to their face-based form, written and read back, give the same arrays
  in every format foam_read takes: ASCII or binary (32- or 64-bit labels, either byte order),
  faces as a faceList or a faceCompactList.
* Cell centroids and volumes from the faces (polyhedron moments about a vertex of each cell)
  agree with the element path's independent numpy restatement where both are exact: tetrahedra
  and planar-faced hexahedra.
* The set-up refuses what foam_read refuses: owner >= neighbour, patches that leave boundary faces
  uncovered, an odd number of periodic patches.
"""
import numpy as np
import pytest

from dopamine_b200 import abi, cases, meshio
from dopamine_b200.solver import DopamineError
from tests.test_geometry_kats import numpy_cell_geometry

HEADER = """/*--------------------------------*- C++ -*----------------------------------*\\
  a comment block as OpenFOAM writes one
\\*---------------------------------------------------------------------------*/
FoamFile
{{
    version     2.0;
    format      {fmt};
    class       {cls};
    note        "nPoints:12 nCells:2 nFaces:11 nInternalFaces:1";
    location    "constant/polyMesh";
    object      {obj};
}}
// * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * * //

"""

# two unit hexes side by side in x: points 0-5 at z=0, 6-11 at z=1
POINTS = [(0, 0, 0), (1, 0, 0), (2, 0, 0), (0, 1, 0), (1, 1, 0), (2, 1, 0),
          (0, 0, 1), (1, 0, 1), (2, 0, 1), (0, 1, 1), (1, 1, 1), (2, 1, 1)]
FACES = [(1, 4, 10, 7),                                   # internal, normal +x (cell 0 -> 1)
         (0, 6, 9, 3), (0, 3, 4, 1), (1, 4, 5, 2),        # walls: x=0 (cell 0), z=0 (cells 0, 1)
         (6, 7, 10, 9), (7, 8, 11, 10), (2, 5, 11, 8),    # z=1 (cells 0, 1), x=2 (cell 1)
         (0, 1, 7, 6), (1, 2, 8, 7), (3, 9, 10, 4), (4, 10, 11, 5)]  # y=0, y=1
OWNER = [0, 0, 0, 1, 0, 1, 1, 0, 1, 0, 1]


def _write(d, fmt="ascii", faces_cls="faceList"):
    d.mkdir(parents=True, exist_ok=True)
    (d / "points").write_text(HEADER.format(fmt=fmt, cls="vectorField", obj="points") + "12\n(\n" +
                              "\n".join(f"({x} {y} {z})" for x, y, z in POINTS) + "\n)\n")
    (d / "faces").write_text(HEADER.format(fmt="ascii", cls=faces_cls, obj="faces") + "11\n(\n" +
                             "\n".join(f"{len(f)}({' '.join(map(str, f))})" for f in FACES) + "\n)\n")
    (d / "owner").write_text(HEADER.format(fmt="ascii", cls="labelList", obj="owner") + "11\n(\n" +
                             "\n".join(map(str, OWNER)) + "\n)\n")
    (d / "neighbour").write_text(HEADER.format(fmt="ascii", cls="labelList", obj="neighbour") + "1\n(\n1\n)\n")
    (d / "boundary").write_text(HEADER.format(fmt="ascii", cls="polyBoundaryMesh", obj="boundary") + """2
(
    walls
    {
        type            wall;
        inGroups        List<word> 1(wall);
        nFaces          6;
        startFace       1;
    }
    sides
    {
        type            patch;
        nFaces          4;
        startFace       7;
    }
)
""")


def test_hand_written_polymesh(tmp_path):
    _write(tmp_path / "polyMesh")
    m = meshio.read_foam(tmp_path / "polyMesh")
    assert np.array_equal(m.xyz, np.array(POINTS, dtype=float))
    assert m.face_off.tolist() == list(range(0, 45, 4))
    assert m.face_nodes.tolist() == [v for f in FACES for v in f]
    assert m.owner.tolist() == OWNER and m.neighbour.tolist() == [1]
    assert m.patch_names == ["walls", "sides"] and m.patch_types == ["wall", "patch"]
    assert m.patch_start.tolist() == [1, 7] and m.patch_nfaces.tolist() == [6, 4]
    cen, vol = meshio.poly_cell_geometry(m, [abi.BC_WALL_NOSLIP, abi.BC_SLIP])
    assert np.allclose(vol, [1.0, 1.0], atol=1e-15)
    assert np.allclose(cen, [[0.5, 0.5, 0.5], [1.5, 0.5, 0.5]], atol=1e-15)


def test_refusals(tmp_path):
    with pytest.raises(DopamineError) as e:
        meshio.read_foam(tmp_path / "nowhere")
    assert e.value.status == abi.ERR_ARG
    # a binary points file cut short
    _write(tmp_path / "bin")
    pm = meshio.read_foam(tmp_path / "bin")
    meshio.write_foam(tmp_path / "bin", pm, binary=True)
    data = (tmp_path / "bin" / "points").read_bytes()
    (tmp_path / "bin" / "points").write_bytes(data[:-40])
    with pytest.raises(DopamineError) as e:
        meshio.read_foam(tmp_path / "bin")
    assert e.value.status == abi.ERR_MESH and "points" in str(e.value)
    # compact offsets that do not start at 0
    meshio.write_foam(tmp_path / "cmp", pm, compact=True)
    text = (tmp_path / "cmp" / "faces").read_text()
    head, rest = text.split("(\n0\n", 1)
    (tmp_path / "cmp" / "faces").write_text(head + "(\n1\n" + rest)
    with pytest.raises(DopamineError) as e:
        meshio.read_foam(tmp_path / "cmp")
    assert e.value.status == abi.ERR_MESH and "start at 0" in str(e.value)


def _bcs(case):
    return [p.bc_id for p in abi.patch_cfgs(case.patches)]


FORMATS = {"ascii": {}, "ascii-compact": dict(compact=True), "binary": dict(binary=True),
           "binary-compact": dict(binary=True, compact=True), "binary-label64": dict(binary=True, label_bytes=8),
           "binary-msb-compact": dict(binary=True, big_endian=True, compact=True)}


@pytest.mark.parametrize("fmt", sorted(FORMATS))
@pytest.mark.parametrize("make", [lambda: cases.hybrid_config(n=4, kind="tet"), lambda: cases.regression_case("channel"),
                                  lambda: cases.hybrid_config(n=4, kind="mixed")], ids=["tet", "channel", "mixed"])
def test_round_trip(tmp_path, make, fmt):
    pm = meshio.to_poly(make().mesh)
    meshio.write_foam(tmp_path / "polyMesh", pm, **FORMATS[fmt])
    r = meshio.read_foam(tmp_path / "polyMesh")
    for k in ("xyz", "face_off", "face_nodes", "owner", "neighbour", "patch_start", "patch_nfaces"):
        assert np.array_equal(getattr(pm, k), getattr(r, k)), k
    assert r.patch_names == pm.patch_names


@pytest.mark.parametrize("make", [lambda: cases.hybrid_config(n=6, kind="tet"), lambda: cases.regression_case("channel")],
                         ids=["jittered tets", "stretched hexes"])
def test_polyhedral_geometry_matches_the_element_geometry(make):
    case = make()
    cen_p, vol_p = meshio.poly_cell_geometry(meshio.to_poly(case.mesh), _bcs(case))
    cen_e, vol_e = numpy_cell_geometry(case.mesh)
    ev = np.abs(vol_p - vol_e).max() / np.abs(vol_e).max()
    ec = np.abs(cen_p - cen_e).max() / np.abs(cen_e).max()
    print(f"{case.name}: volume {ev:.1e}, centroid {ec:.1e}")
    assert ev <= 1e-12 and ec <= 1e-12


def test_polyhedral_setup_refusals():
    case = cases.hybrid_config(n=3, kind="tet")
    bcs = _bcs(case)
    pm = meshio.to_poly(case.mesh)
    bad = meshio.to_poly(case.mesh)
    bad.owner = bad.owner.copy()
    bad.owner[0] = bad.neighbour[0]  # owner == neighbour on an internal face
    with pytest.raises(DopamineError, match="upper-triangular"):
        meshio.poly_cell_geometry(bad, bcs)
    bad = meshio.to_poly(case.mesh)
    bad.patch_nfaces = bad.patch_nfaces.copy()
    bad.patch_nfaces[-1] -= 1  # the last boundary face in no patch
    with pytest.raises(DopamineError, match="not mapped"):
        meshio.poly_cell_geometry(bad, bcs)
    odd = [abi.BC_PERIODIC] + [abi.BC_WALL_NOSLIP] * (len(bcs) - 1)
    with pytest.raises(DopamineError, match="odd number of periodic"):
        meshio.poly_cell_geometry(pm, odd)
