"""Device set-up of the mesh and static operators (csrc/cuda/setup_gpu.cu) against the host
builder (csrc/host/mesh.cpp, ops.cpp), whose geometry, pressure coefficients and stencils the
oracle's regression CSVs and the independent known-answer tests pin.

* Every array of the Mesh and StaticOps, entry by entry, bit for bit, on tetrahedral, mixed
  hex/prism/pyramid, skewed periodic, wall-bounded, inlet/outlet, ABL-inlet and urban-obstacle
  meshes, and on the 2.44M-cell urban canopy; the SGS filter tensor, whose scale is a cube root by
  pow(), within 1e-14 of each cell's tensor scale.
* Handles created with either builder take the same steps.
* Malformed meshes (an unsupported element, an open cell, a boundary face that no cell has) are
  refused by the device builder with the host builder's status.
"""
import numpy as np
import pytest

from dopamine_b200 import abi, cases
from dopamine_b200.solver import DopamineError, Solver, compare_setups

pytestmark = pytest.mark.gpu

SMALL = {
    "tet8": lambda: cases.hybrid_config(n=8, kind="tet"),
    "mixed8": lambda: cases.hybrid_config(n=8, kind="mixed"),
    "tgv_skew": lambda: cases.regression_case("tgv_skew"),
    "channel": lambda: cases.regression_case("channel"),
    "duct": lambda: cases.regression_case("duct"),
    "inflow": lambda: cases.regression_case("inflow"),
    "rb": lambda: cases.regression_case("rb"),
    "urban24": lambda: cases.urban_config(nx=24, ny=24, nz=12, n_blocks=4, lx=2.4, ly=2.4, lz=0.72, n_steps=3,
                                          scale=0.01),
}


def _check_same(name, case):
    mism, g, t = compare_setups(case)
    bad = {k: v for k, v in mism.items() if v}
    print(f"{name}: {len(mism)} arrays compared, G max rel {g:.1e}, host {t['host_mesh_ms']:.0f}+"
          f"{t['host_ops_ms']:.0f} ms, device {t['device_mesh_ms']:.0f}+{t['device_ops_ms']:.0f} ms")
    assert not bad, bad
    assert g <= 1e-14  # a last-bit difference of pow() carried through the two smoothing passes
    return t


@pytest.mark.parametrize("name", sorted(SMALL))
def test_device_setup_matches_host(name):
    _check_same(name, SMALL[name]())


def test_device_setup_matches_host_urban_2m():
    case = cases.urban_config(200, 200, 63)
    # The stage times are printed, not compared: in this comparison mode the device builder also
    # copies every array back to the host, and the host builder runs on all host threads.
    _check_same("urban 200x200x63", case)


def test_both_builders_take_the_same_steps():
    case = SMALL["urban24"]()
    out = []
    for host in (0, 1):
        p = case.make_params()
        p.host_setup = host
        s = Solver(case, params=p)
        s.initialise()
        for _ in range(3):
            s.advance()
        out.append(s.sync_host()["U"])
        st = s.setup_times()
        assert st["total_ms"] > 0.0 and st["mesh_ms"] > 0.0
        assert (st["match_ms"] > 0.0) == (host == 0)
        s.close()
    e = float(np.linalg.norm(out[0] - out[1]) / np.linalg.norm(out[1]))
    print(f"urban24, 3 steps, device vs host set-up: U rel {e:.1e}")
    assert e <= 1e-12


def _mutated(kind):
    case = SMALL["mixed8"]()
    m = case.mesh
    if kind == "element":
        m.cell_type = m.cell_type.copy()
        m.cell_type[5] = 2  # a surface triangle code among the volume elements
    elif kind == "open":
        nb = m.bface_patch.shape[0]
        m.bface_nodes = m.bface_nodes[: m.bface_off[nb - 1]].copy()
        m.bface_off = m.bface_off[:nb].copy()
        m.bface_patch = m.bface_patch[: nb - 1].copy()
    else:  # a boundary face whose nodes no element face has
        n = m.xyz.shape[0]
        m.bface_nodes = m.bface_nodes.copy()
        lo, hi = m.bface_off[0], m.bface_off[1]
        m.bface_nodes[lo:hi] = np.array([0, n - 1, n - 2, n - 3][: hi - lo], dtype=np.int32)
    return case


@pytest.mark.parametrize("kind", ["element", "open", "orphan"])
def test_malformed_meshes_are_refused(kind):
    for host in (0, 1):
        case = _mutated(kind)
        p = case.make_params()
        p.host_setup = host
        with pytest.raises(DopamineError) as e:
            Solver(case, params=p)
        assert e.value.status == abi.ERR_MESH, (kind, host, e.value.status)


def test_mesh_read_from_a_gmsh_file_takes_the_same_steps(tmp_path):
    from dopamine_b200 import meshio
    case = SMALL["urban24"]()
    path = tmp_path / "urban24.msh"
    meshio.write_gmsh(path, case.mesh)
    read = SMALL["urban24"]()
    read.mesh = meshio.read_gmsh(path)
    out = []
    for c in (case, read):
        s = Solver(c)
        s.initialise()
        for _ in range(2):
            s.advance()
        out.append(s.sync_host()["U"])
        s.close()
    assert np.array_equal(out[0], out[1])
