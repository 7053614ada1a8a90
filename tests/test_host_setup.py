"""The host builder (csrc/host/mesh.cpp build_mesh / build_mesh_poly, csrc/host/ops.cpp
build_static_ops) on the CPU, through dpm_setup_host_digest: a 64-bit FNV-1a digest of every
array it produces, in dpm_setup_array_name order.

* The host threads build each cell's sums by a gather in a fixed order and sort by strict total
  orders, so every array is the same bit for bit on 1, 3 or all host threads.
* The arrays equal the committed digests (tests/golden/host_setup_digests.json, written by
  tests/golden/make_host_setup_digests.py from this builder).  The GPU tests check the same
  arrays, entry by entry, against the device builder; these digests pin them on the CPU.
* Malformed meshes are refused with the host builder's status and reason: an unsupported element,
  an open cell, a boundary face that no cell has, an assembled row wider than 16 entries.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from dopamine_b200 import abi, cases, meshio
from dopamine_b200.solver import DopamineError, host_setup_digests

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "host_setup_digests.json")


def _poly(make):
    def f():
        case = make()
        case.mesh = meshio.to_poly(case.mesh)
        return case
    return f


def _merged(block):
    def f():
        from tests.test_gpu_foam import _merged_mesh
        case = cases.hybrid_config(n=4, kind="mixed", n_steps=3)
        case.mesh = _merged_mesh(block)[0]
        return case
    return f


_URBAN24 = dict(nx=24, ny=24, nz=12, n_blocks=4, lx=2.4, ly=2.4, lz=0.72, n_steps=3, scale=0.01)
CASES = {
    "tet8": lambda: cases.hybrid_config(n=8, kind="tet"),
    "mixed8": lambda: cases.hybrid_config(n=8, kind="mixed"),
    "tgv_skew": lambda: cases.regression_case("tgv_skew"),
    "channel": lambda: cases.regression_case("channel"),
    "duct": lambda: cases.regression_case("duct"),
    "inflow": lambda: cases.regression_case("inflow"),
    "rb": lambda: cases.regression_case("rb"),
    "urban24": lambda: cases.urban_config(**_URBAN24),
    "channel (face-based)": _poly(lambda: cases.regression_case("channel")),
    "tet8 (face-based)": _poly(lambda: cases.hybrid_config(n=8, kind="tet")),
    "mixed8 (face-based)": _poly(lambda: cases.hybrid_config(n=8, kind="mixed")),
    "urban24 (face-based)": _poly(lambda: cases.urban_config(**_URBAN24)),
    "merged 10-face cell (face-based)": _merged(((1.0, 1.0, 1.0), (3.0, 2.0, 2.0))),
}


def digests_as_hex(case):
    arrays, g = host_setup_digests(case)
    out = {k: f"{v:016x}" for k, v in arrays.items()}
    out["G"] = f"{g:016x}"
    return out


class _Threads:
    """Sets the OpenMP thread count of the host builder's parallel loops (one libgomp per process)."""

    def __init__(self):
        self.gomp = ctypes.CDLL("libgomp.so.1")
        self.default = self.gomp.omp_get_max_threads()

    def __call__(self, n):
        self.gomp.omp_set_num_threads(int(n))


@pytest.fixture(scope="module")
def threads():
    t = _Threads()
    yield t
    t(t.default)


@pytest.mark.parametrize("name", list(CASES))
def test_same_arrays_on_any_thread_count(name, threads):
    out = {}
    for n in (1, 3, threads.default):
        threads(n)
        out[n] = digests_as_hex(CASES[name]())
    threads(threads.default)
    base = out[1]
    assert len(base) == 53
    for n, d in out.items():
        diff = [k for k in base if d[k] != base[k]]
        assert not diff, (n, diff)


@pytest.mark.parametrize("name", list(CASES))
def test_arrays_equal_the_committed_digests(name):
    with open(GOLDEN) as fh:
        golden = json.load(fh)[name]
    d = digests_as_hex(CASES[name]())
    diff = [k for k in golden if d.get(k) != golden[k]]
    assert not diff, diff
    assert set(d) == set(golden)


@pytest.mark.parametrize("kind,reason", [("element", "unsupported element type"),
                                         ("open", "unlabelled boundary faces (open cells)"),
                                         ("orphan", "boundary face has no owner cell")])
def test_malformed_meshes_are_refused(kind, reason):
    from tests.test_gpu_setup import _mutated
    with pytest.raises(DopamineError) as e:
        host_setup_digests(_mutated(kind))
    assert e.value.status == abi.ERR_MESH and reason in str(e.value)


def test_row_wider_than_sixteen_entries_is_refused():
    """A 2x2x2 block merged into one cell has 24 face neighbours."""
    with pytest.raises(DopamineError) as e:
        host_setup_digests(_merged(((1.0, 1.0, 1.0), (3.0, 3.0, 3.0)))())
    assert e.value.status == abi.ERR_UNSUPPORTED


def test_digests_see_small_changes():
    """One ulp of one vertex coordinate changes the digest of the copied vertices (in the mesh
    scalars); a move of 1e-9 changes the cell geometry's digests, and no connectivity digest."""
    case = CASES["channel"]()
    a = digests_as_hex(case)
    xyz = case.mesh.xyz
    case.mesh.xyz = xyz.copy()
    case.mesh.xyz[7, 1] = np.nextafter(xyz[7, 1], np.inf)
    b = digests_as_hex(case)
    assert a["mesh_scalars"] != b["mesh_scalars"]
    case.mesh.xyz[7, 1] = xyz[7, 1] + 1e-9
    c = digests_as_hex(case)
    assert a["volume"] != c["volume"] and a["centroid"] != c["centroid"]
    assert a["cell_faces"] == c["cell_faces"] and a["patch_start"] == c["patch_start"]
