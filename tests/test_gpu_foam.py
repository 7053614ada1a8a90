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
