"""Solver handles on OpenFOAM-style face-based meshes (dpm_create_poly: faces in OpenFOAM's
order, the reference's polyhedral geometry) against handles on the same meshes given as
elements (dpm_create).

* Hexahedral meshes: both describe the same cells, faces and LS stencils (26 vertex neighbours,
  under the 32-entry cap). Only the face numbering and the summation orders differ, so the steps
  agree to round-off: velocity within 1e-10 relative after 5 steps on the stretched channel, and
  after 2 steps on the urban-obstacle mesh read back from polyMesh files.
* Tetrahedral meshes: a tetrahedron shares vertices with up to 70 cells here, and the LS stencil
  keeps the first 32 in cell-vertex order. The face-based path orders a cell's vertices by its
  faces (build_cell_topology_metadata), the element path by the element's nodes, so the two
  stencils hold different neighbours. The reference's gmsh and OpenFOAM paths differ the same
  way. The two runs are different discretisations, so only the physics is compared: kinetic
  energy within 5 % after 5 steps, both divergence-free.
"""
import numpy as np
import pytest

from dopamine_b200 import cases, meshio
from dopamine_b200.solver import Solver

pytestmark = pytest.mark.gpu


def _steps(case, n):
    s = Solver(case)
    s.initialise()
    for _ in range(n):
        s.advance()
    out = s.sync_host()["U"], s.stats(), s.setup_times()
    s.close()
    return out


@pytest.mark.parametrize("name", ["channel", "tet8", "urban24"])
def test_face_based_mesh_steps_like_the_element_mesh(tmp_path, name):
    make = {"channel": lambda: cases.regression_case("channel"),
            "tet8": lambda: cases.hybrid_config(n=8, kind="tet", n_steps=5),
            "urban24": lambda: cases.urban_config(nx=24, ny=24, nz=12, n_blocks=4, lx=2.4, ly=2.4, lz=0.72,
                                                  n_steps=2, scale=0.01)}[name]
    n = 2 if name == "urban24" else 5
    ref_case = make()
    poly_case = make()
    if name == "urban24":  # through the files
        meshio.write_foam(tmp_path / "polyMesh", ref_case.mesh)
        poly_case.mesh = meshio.read_foam(tmp_path / "polyMesh")
    else:
        poly_case.mesh = meshio.to_poly(ref_case.mesh)
    Ue, ste, _ = _steps(ref_case, n)
    Up, stp, tp = _steps(poly_case, n)
    e = float(np.linalg.norm(Up - Ue) / np.linalg.norm(Ue))
    eE = abs(stp["E"] - ste["E"]) / ste["E"]
    print(f"{name}: {n} steps, face-based vs element mesh: U rel {e:.1e}, E rel {eE:.1e}, "
          f"divU {stp['max_abs_divU']:.1e}")
    if name == "tet8":
        assert eE <= 0.05
    else:
        assert e <= 1e-10
    assert stp["max_abs_divU"] <= 1e-9 and ste["max_abs_divU"] <= 1e-9
    assert tp["mesh_ms"] > 0.0 and tp["match_ms"] > 0.0  # the device polyhedral set-up ran


@pytest.mark.parametrize("name", ["channel", "tet8", "mixed8", "urban24"])
def test_device_polyhedral_setup_matches_host(name):
    """The device builder on a face-based mesh against the host builder (build_mesh_poly), entry
    by entry, as tests/test_gpu_setup.py does for element meshes."""
    from dopamine_b200.solver import compare_setups
    case = {"channel": lambda: cases.regression_case("channel"),
            "tet8": lambda: cases.hybrid_config(n=8, kind="tet"),
            "mixed8": lambda: cases.hybrid_config(n=8, kind="mixed"),
            "urban24": lambda: cases.urban_config(nx=24, ny=24, nz=12, n_blocks=4, lx=2.4, ly=2.4, lz=0.72,
                                                  scale=0.01)}[name]()
    case.mesh = meshio.to_poly(case.mesh)
    mism, g, t = compare_setups(case)
    bad = {k: v for k, v in mism.items() if v}
    print(f"{name} (face-based): {len(mism)} arrays compared, G max rel {g:.1e}")
    assert not bad, bad
    assert g <= 1e-14


def _merged_mesh(block):
    """A 4x4x4 box of unit hexes whose cells inside `block` (a box of cell-centre bounds) are merged
    into one polyhedral cell, its faces the block's outer faces (each split where the neighbours'
    faces meet).  Faces in OpenFOAM order (internal faces by owner, then neighbour)."""
    from dopamine_b200.cases import PolyMesh, uniform_box
    box = uniform_box(4, 4, 4, 4.0, 4.0, 4.0)
    pm = meshio.to_poly(box)
    cen = np.array([box.xyz[box.cell_nodes[box.cell_off[c]:box.cell_off[c + 1]]].mean(axis=0) for c in range(box.n_cells)])
    lo, hi = np.array(block[0]), np.array(block[1])
    inner = np.all((cen > lo) & (cen < hi), axis=1)
    first = int(np.nonzero(inner)[0][0])
    merged = int((~inner[:first]).sum())  # the merged cell takes the first inner cell's place
    new_id = np.cumsum(~inner) - 1
    new_id = np.where(new_id >= merged, new_id + 1, new_id)
    new_id[inner] = merged
    nfi = pm.neighbour.shape[0]
    faces, owner, nbr = [], [], []
    for f in range(nfi):
        o, n = int(new_id[pm.owner[f]]), int(new_id[pm.neighbour[f]])
        if o == n:
            continue  # inside the merged block
        nodes = pm.face_nodes[pm.face_off[f]:pm.face_off[f + 1]]
        if o > n:
            o, n, nodes = n, o, nodes[::-1]
        faces.append(nodes); owner.append(o); nbr.append(n)
    order = sorted(range(len(owner)), key=lambda k: (owner[k], nbr[k]))
    faces = [faces[k] for k in order]; owner = [owner[k] for k in order]; nbr = [nbr[k] for k in order]
    n_int = len(owner)
    for f in range(nfi, pm.owner.shape[0]):
        faces.append(pm.face_nodes[pm.face_off[f]:pm.face_off[f + 1]]); owner.append(int(new_id[pm.owner[f]]))
    return PolyMesh(xyz=pm.xyz, face_off=np.concatenate([[0], np.cumsum([len(f) for f in faces])]).astype(np.int64),
                    face_nodes=np.concatenate(faces).astype(np.int32), owner=np.array(owner, np.int32),
                    neighbour=np.array(nbr, np.int32), patch_start=pm.patch_start - nfi + n_int,
                    patch_nfaces=pm.patch_nfaces, patch_names=pm.patch_names, patch_types=pm.patch_types), int(inner.sum())


def test_merged_polyhedral_cell():
    """Two unit hexes merged into one 10-face polyhedral cell (volume 2) inside a periodic box: the
    device builder takes it and the handle steps exactly as with the host builder."""
    pm, k = _merged_mesh(((1.0, 1.0, 1.0), (3.0, 2.0, 2.0)))
    assert k == 2
    out = []
    for host in (0, 1):
        case = cases.hybrid_config(n=4, kind="mixed", n_steps=3)  # the periodic box's parameters
        case.mesh = pm
        p = case.make_params()
        p.host_setup = host
        s = Solver(case, params=p)
        assert s.nc == 63
        assert abs(s.volume.max() - 2.0) < 1e-12 and abs(s.volume.sum() - 64.0) < 1e-10
        s.initialise()
        for _ in range(3):
            s.advance()
        out.append(s.sync_host()["U"])
        assert s.stats()["max_abs_divU"] <= 1e-9
        s.close()
    assert np.array_equal(out[0], out[1])


def test_cell_with_more_than_fifteen_neighbours_is_refused():
    """A 2x2x2 block merged into one cell has 24 face neighbours: its pressure-operator row is wider
    than the kernels' 16 entries. The device builder stops before reading the cell's lists and hands
    the mesh to the host builder, which refuses the row: DPM_ERR_UNSUPPORTED either way, and the
    handle's context stays usable."""
    from dopamine_b200 import abi
    from dopamine_b200.solver import DopamineError
    pm, k = _merged_mesh(((1.0, 1.0, 1.0), (3.0, 3.0, 3.0)))
    assert k == 8
    for host in (0, 1):
        case = cases.hybrid_config(n=4, kind="mixed", n_steps=3)
        case.mesh = pm
        p = case.make_params()
        p.host_setup = host
        with pytest.raises(DopamineError) as e:
            Solver(case, params=p)
        assert e.value.status == abi.ERR_UNSUPPORTED
    s = Solver(cases.regression_case("channel"))  # the context still works
    s.initialise()
    s.advance()
    assert s.stats()["max_abs_divU"] <= 1e-9
    s.close()
