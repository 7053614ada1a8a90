"""Independent pins of the static set-up (mesh geometry and pressure-operator coefficients) and
ports of the reference's non-orthogonal k-vector unit test.

The product's geometry code (dopamine_b200/csrc/host/mesh.cpp) is also what the oracle links, so a
comparison of the two alone would check the code against itself.  Here the geometry is restated a
second time, in vectorised numpy written from the reference routines directly:

* cell centroids and volumes by the tetrahedral decompositions of
  src/mesh/mod_gmsh_reader.f90:737-841 (tet exact; hex 5 tets; prism 3; pyramid 2), each tet's
  centroid the vertex mean and its volume |det|/6, the cell centroid the volume-weighted mean;
* face area vectors by the fan from the vertex mean (mod_gmsh_reader.f90:843-869), faces matched
  between cells by their sorted node lists;
* the pressure operator's interior-face coefficient |S_f| / (d . n_f) with d the centroid-to-
  centroid vector (src/solver/mod_pressure_solver.f90:100-452, no cos(theta) floor).

Those are compared with the set-up's arrays on jittered tet, hex/prism/pyramid and skewed-hex
meshes.  Two analytic checks need no restatement at all: an affine map of a box multiplies every
volume by |det| and moves centroids affinely, and every closed cell's outward area vectors sum to
zero (the least-squares test in test_oracle_kats covers the latter through exactness).

The k-vector checks port tests/unit/test_nonortho_limiter.f90 case for case.
"""
import ctypes as C

import numpy as np
import pytest

from dopamine_b200 import abi, cases
from oracle import oracle as O

# gmsh local node orders: the perimeter of each cell face (orientation does not matter here)
FACES = {
    abi.EL_TET4: [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)],
    abi.EL_HEX8: [(0, 1, 2, 3), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7)],
    abi.EL_PRISM6: [(0, 1, 2), (3, 4, 5), (0, 1, 4, 3), (1, 2, 5, 4), (2, 0, 3, 5)],
    abi.EL_PYR5: [(0, 1, 2, 3), (0, 1, 4), (1, 2, 4), (2, 3, 4), (3, 0, 4)],
}
# tetrahedral decompositions, 0-based (mod_gmsh_reader.f90:784-841)
TETS = {
    abi.EL_TET4: [(0, 1, 2, 3)],
    abi.EL_HEX8: [(0, 1, 3, 4), (1, 2, 3, 6), (3, 4, 6, 7), (1, 4, 5, 6), (1, 3, 4, 6)],
    abi.EL_PRISM6: [(0, 1, 2, 3), (1, 3, 4, 2), (2, 3, 4, 5)],
    abi.EL_PYR5: [(0, 1, 3, 4), (1, 2, 3, 4)],
}
NNODES = {abi.EL_TET4: 4, abi.EL_HEX8: 8, abi.EL_PRISM6: 6, abi.EL_PYR5: 5}


def _cells_by_type(mesh):
    out = {}
    for t in np.unique(mesh.cell_type):
        ids = np.nonzero(mesh.cell_type == t)[0]
        nn = NNODES[int(t)]
        nodes = np.stack([mesh.cell_nodes[mesh.cell_off[ids] + k] for k in range(nn)], axis=1)
        out[int(t)] = (ids, nodes)
    return out


def numpy_cell_geometry(mesh):
    nc = mesh.n_cells
    cen = np.zeros((nc, 3))
    vol = np.zeros(nc)
    for t, (ids, nodes) in _cells_by_type(mesh).items():
        P = mesh.xyz[nodes]                      # (m, nn, 3)
        v_acc = np.zeros(len(ids))
        c_acc = np.zeros((len(ids), 3))
        for tet in TETS[t]:
            p1, p2, p3, p4 = (P[:, a, :] for a in tet)
            tv = np.abs(np.einsum("ij,ij->i", p2 - p1, np.cross(p3 - p1, p4 - p1))) / 6.0
            tc = (p1 + p2 + p3 + p4) / 4.0
            v_acc += tv
            c_acc += tv[:, None] * tc
        if len(TETS[t]) > 1:
            c_acc /= v_acc[:, None]
        else:
            c_acc = tc  # a tet's centroid directly (no weighting round trip)
        cen[ids] = c_acc
        vol[ids] = v_acc
    return cen, vol


def numpy_interior_faces(mesh):
    """(cell a, cell b, area vector) for every face shared by two cells."""
    keys, cells, svec = [], [], []
    for t, (ids, nodes) in _cells_by_type(mesh).items():
        for fl in FACES[t]:
            fn = nodes[:, fl]                    # (m, k) perimeter
            P = mesh.xyz[fn]
            c = P.mean(axis=1)
            acc = np.zeros((len(ids), 3))
            k = len(fl)
            for i in range(k):
                acc += 0.5 * np.cross(P[:, i] - c, P[:, (i + 1) % k] - c)
            key = np.full((len(ids), 4), -1, dtype=np.int64)
            key[:, :k] = np.sort(fn, axis=1)
            keys.append(key)
            cells.append(ids)
            svec.append(acc)
    keys = np.concatenate(keys)
    cells = np.concatenate(cells)
    svec = np.concatenate(svec)
    _, inv, cnt = np.unique(keys, axis=0, return_inverse=True, return_counts=True)
    inv = inv.ravel()
    assert cnt.max() <= 2, "a face shared by more than two cells"
    order = np.argsort(inv, kind="stable")
    grp = inv[order]
    first = np.nonzero(np.r_[True, grp[1:] != grp[:-1]])[0]
    pairs = first[cnt[grp[first]] == 2]
    a, b = order[pairs], order[pairs + 1]
    return cells[a], cells[b], svec[a]


MESHES = {
    "tet5": lambda: cases.hybrid_config(n=5, kind="tet"),
    "mixed6": lambda: cases.hybrid_config(n=6, kind="mixed"),
    "skewed_hex": lambda: cases.regression_case("hydrowall"),
}


@pytest.mark.parametrize("name", sorted(MESHES))
def test_cell_geometry_matches_an_independent_restatement(name):
    case = MESHES[name]()
    o = O.Oracle(case)
    cen, vol = numpy_cell_geometry(case.mesh)
    np.testing.assert_allclose(o.volume, vol, rtol=1e-13, atol=0)
    scale = np.abs(case.mesh.xyz).max()
    np.testing.assert_allclose(o.centroid, cen, rtol=0, atol=1e-14 * scale)
    if name == "tet5":  # planar faces: the tets tile the box exactly (warped quads do not)
        assert abs(vol.sum() - 1.0) <= 1e-12


@pytest.mark.parametrize("name", sorted(MESHES))
def test_pressure_coefficients_match_an_independent_restatement(name):
    case = MESHES[name]()
    pr = case.make_params()
    assert pr.pressure_min_cos_theta == 0.0
    o = O.Oracle(case)
    off, col, val = o.poisson_csr()
    a, b, S = numpy_interior_faces(case.mesh)
    cen, _ = numpy_cell_geometry(case.mesh)
    area = np.linalg.norm(S, axis=1)
    d = cen[b] - cen[a]
    dn = np.abs(np.einsum("ij,ij->i", d, S)) / area
    want = area / dn
    got = np.empty_like(want)
    for i, (r, c) in enumerate(zip(a, b)):
        row = slice(off[r], off[r + 1])
        hit = np.nonzero(col[row] == c)[0]
        assert hit.size == 1, (r, c)
        got[i] = -val[row][hit[0]]
    assert a.size > 100
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)


def test_affine_box_volumes_and_centroids_are_exact():
    """A uniform hex box under x -> M x + t: volumes are |det M| h^3 and centroids M c + t."""
    n = 4
    M = np.array([[1.0, 0.3, -0.2], [0.1, 0.9, 0.25], [-0.15, 0.2, 1.1]])
    t = np.array([0.5, -1.0, 2.0])
    m = cases.mixed_box(n, jitter=0.0, prism_cols=0.0, pyramid_hex=0.0)  # uniform hexes only
    assert np.all(m.cell_type == abi.EL_HEX8)
    m.xyz = m.xyz @ M.T + t
    cen, vol = numpy_cell_geometry(m)
    np.testing.assert_allclose(vol, abs(np.linalg.det(M)) / n ** 3, rtol=1e-13)
    # the set-up on the same mapped mesh, walled on all six sides
    case = cases.hybrid_config(n=n, kind="mixed")
    case.mesh = m
    case.patches = [{"bc": "noSlip"} for _ in range(6)]
    o = O.Oracle(case)
    np.testing.assert_allclose(o.volume, abs(np.linalg.det(M)) / n ** 3, rtol=1e-13)
    ref_c = np.zeros((m.n_cells, 3))
    for c in range(m.n_cells):
        nodes = m.cell_nodes[m.cell_off[c]:m.cell_off[c + 1]]
        ref_c[c] = m.xyz[nodes].mean(axis=0)      # a parallelepiped's centroid is its vertex mean
    np.testing.assert_allclose(o.centroid, ref_c, rtol=0, atol=1e-14 * np.abs(m.xyz).max())


def _k(sf, d, min_cos):
    sf = np.asarray(sf, dtype=np.float64)
    d = np.asarray(d, dtype=np.float64)
    k = np.zeros(3)
    dp = C.POINTER(C.c_double)
    O.lib().orc_kfactor_limited(sf.ctypes.data_as(dp), d.ctypes.data_as(dp), min_cos, k.ctypes.data_as(dp))
    return k


def test_nonortho_limiter_known_answers():
    """tests/unit/test_nonortho_limiter.f90, each case at its 1e-12 tolerance."""
    tol = lambda want: 1e-12 * max(1.0, abs(want))
    # orthogonal face: the floor is inactive and k = 0
    assert np.abs(_k([2.0, 0.0, 0.0], [0.5, 0.0, 0.0], 0.3)).max() <= tol(0.0)
    # 89.4 degrees: floor 0 is the over-relaxed vector itself, a floor below cos(theta) changes nothing
    sf, d = [1.0, 0.0, 0.0], [0.01, 1.0, 0.0]
    k0 = _k(sf, d, 0.0)
    assert np.abs(_k(sf, d, 0.005) - k0).max() <= tol(0.0)
    # active floor: the implicit coefficient (S - k).d / d.d is bounded by |S| / (|d| cmin)
    a0 = (sf[0] - k0[0]) / d[0]
    assert a0 > 50.0
    k1 = _k(sf, d, 0.2)
    a = (sf[0] - k1[0]) / d[0]
    want = 1.0 / (np.linalg.norm(d) * 0.2)
    assert abs(a - want) <= tol(want)
    # consistency: a (d.g) + k.g = S.g for any gradient, so linear fields stay exact
    g = np.array([0.7, -1.3, 2.1])
    lhs = a * np.dot(d, g) + np.dot(k1, g)
    assert abs(lhs - np.dot(sf, g)) <= tol(np.dot(sf, g))
