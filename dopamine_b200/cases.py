"""Meshes, initial conditions and run configurations for the RK3W hot path.

The reference reads gmsh / OpenFOAM files and sets initial fields in Fortran
(src/mesh/mod_gmsh_reader.f90, src/init/mod_initconditions.f90).  This module produces the same
inputs directly as arrays: a gmsh-like raw mesh (nodes, volume elements, tagged boundary
elements) and cell-centred initial fields.  It is host set-up code, outside the timed step.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import abi


@dataclass
class RawMesh:
    xyz: np.ndarray            # (n_nodes, 3) float64
    cell_type: np.ndarray      # (n_cells,) int32 gmsh codes
    cell_off: np.ndarray       # (n_cells+1,) int64
    cell_nodes: np.ndarray     # int32, 0-based
    bface_off: np.ndarray      # (n_bfaces+1,) int64
    bface_nodes: np.ndarray    # int32
    bface_patch: np.ndarray    # (n_bfaces,) int32
    patch_names: list = field(default_factory=list)

    @property
    def n_cells(self):
        return int(self.cell_type.shape[0])

    def vertex_bounds(self):
        return self.xyz.min(axis=0), self.xyz.max(axis=0)


def structured_box(X, Y, Z, names=("x0", "xL", "y0", "yL", "z0", "zL")):
    """Hex box from node coordinate arrays X, Y, Z of shape (nx+1, ny+1, nz+1).

    Node, element and boundary-quad numbering follow tests/regression/mk_box_mesh.py:
    node id i + (nx+1)(j + (ny+1) k), hexes in k, j, i order, boundary quads per surface in the
    order x0, xL, y0, yL, z0, zL.
    """
    nx, ny, nz = (s - 1 for s in X.shape)
    xyz = np.stack([X.transpose(2, 1, 0).ravel(), Y.transpose(2, 1, 0).ravel(), Z.transpose(2, 1, 0).ravel()], axis=1)

    def nid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    hexes = np.stack([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
                      nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)], axis=1)
    quads = []
    patch = []

    def surf(s, a_n, b_n, fn):
        b, a = np.meshgrid(np.arange(b_n), np.arange(a_n), indexing="ij")
        # mk_box_mesh loops "for a in range(N): for b in range(N)" -> a slowest
        a, b = a.T.ravel(), b.T.ravel()
        quads.append(fn(a, b))
        patch.append(np.full(a.shape[0], s, dtype=np.int32))

    surf(0, ny, nz, lambda a, b: np.stack([nid(0, a, b), nid(0, a + 1, b), nid(0, a + 1, b + 1), nid(0, a, b + 1)], 1))
    surf(1, ny, nz, lambda a, b: np.stack([nid(nx, a, b), nid(nx, a + 1, b), nid(nx, a + 1, b + 1), nid(nx, a, b + 1)], 1))
    surf(2, nx, nz, lambda a, b: np.stack([nid(a, 0, b), nid(a + 1, 0, b), nid(a + 1, 0, b + 1), nid(a, 0, b + 1)], 1))
    surf(3, nx, nz, lambda a, b: np.stack([nid(a, ny, b), nid(a + 1, ny, b), nid(a + 1, ny, b + 1), nid(a, ny, b + 1)], 1))
    surf(4, nx, ny, lambda a, b: np.stack([nid(a, b, 0), nid(a + 1, b, 0), nid(a + 1, b + 1, 0), nid(a, b + 1, 0)], 1))
    surf(5, nx, ny, lambda a, b: np.stack([nid(a, b, nz), nid(a + 1, b, nz), nid(a + 1, b + 1, nz), nid(a, b + 1, nz)], 1))
    q = np.concatenate(quads).astype(np.int32)
    nh = hexes.shape[0]
    return RawMesh(
        xyz=np.ascontiguousarray(xyz, dtype=np.float64),
        cell_type=np.full(nh, abi.EL_HEX8, dtype=np.int32),
        cell_off=np.arange(0, 8 * nh + 1, 8, dtype=np.int64),
        cell_nodes=hexes.astype(np.int32).ravel(),
        bface_off=np.arange(0, 4 * q.shape[0] + 1, 4, dtype=np.int64),
        bface_nodes=q.ravel(),
        bface_patch=np.concatenate(patch),
        patch_names=list(names),
    )


def uniform_box(nx, ny, nz, lx, ly, lz, names=("x0", "xL", "y0", "yL", "z0", "zL")):
    x = np.arange(nx + 1) * (lx / nx)
    y = np.arange(ny + 1) * (ly / ny)
    z = np.arange(nz + 1) * (lz / nz)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    return structured_box(X, Y, Z, names)


def skewed_unit_box(n, amp):
    """Curvilinear unit box of tests/regression/mk_box_mesh.py (N, AMP): nodes displaced by
    AMP sin(pi X) sin(2 pi Y) sin(pi Z) cyclically; coordinates rounded to 16 significant digits
    as the %.16g gmsh file carries them."""
    X = np.empty((n + 1, n + 1, n + 1))
    Y = np.empty_like(X)
    Z = np.empty_like(X)
    s, pi = math.sin, math.pi
    for k in range(n + 1):
        for j in range(n + 1):
            for i in range(n + 1):
                a, b, c = i / n, j / n, k / n
                X[i, j, k] = float(f"{a + amp * s(pi * a) * s(2 * pi * b) * s(pi * c):.16g}")
                Y[i, j, k] = float(f"{b + amp * s(pi * b) * s(2 * pi * c) * s(pi * a):.16g}")
                Z[i, j, k] = float(f"{c + amp * s(pi * c) * s(2 * pi * a) * s(pi * b):.16g}")
    return structured_box(X, Y, Z)


def channel_box(nx, ny, nz, lx, ly, lz, stretch):
    """Channel with walls at y = -ly/2, +ly/2 and tanh wall-normal clustering:
    y_j = (ly/2) tanh(stretch (2 j/ny - 1)) / tanh(stretch)."""
    x = np.arange(nx + 1) * (lx / nx)
    eta = 2.0 * np.arange(ny + 1) / ny - 1.0
    y = 0.5 * ly * np.tanh(stretch * eta) / math.tanh(stretch)
    z = np.arange(nz + 1) * (lz / nz)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    return structured_box(X, Y, Z, names=("x0", "xL", "bottom_wall", "top_wall", "z0", "zL"))


def bump_nodes(n, coef):
    """Node positions in [0, 1] of a transfinite line of n cells "Using Bump coef" (gmsh): the
    local cell size varies quadratically along the line, the end cells being `coef` times the
    middle one.  Positions are the closed-form inverse of the cumulative point density
    1 / (1 + 4 (coef - 1) x^2), x in [-1/2, 1/2], sampled at equal increments."""
    u = 2.0 * np.arange(n + 1) / n - 1.0
    if abs(coef - 1.0) < 1e-14:
        x = 0.5 * u
    elif coef < 1.0:
        q = math.sqrt(1.0 - coef)
        x = np.tanh(u * math.atanh(q)) / (2.0 * q)
    else:
        q = math.sqrt(coef - 1.0)
        x = np.tan(u * math.atan(q)) / (2.0 * q)
    x = 0.5 + x
    x[0], x[-1] = 0.0, 1.0
    return x


def wall_box(nx, ny, nz, lx, ly, lz, bump_z):
    """Box of examples/RayleighBernard/RB.geo: x, y periodic, walls at z = 0 and z = lz, uniform
    in x and y, "Bump" grading bump_z in z.  Patches in the reference's order."""
    x = np.arange(nx + 1) * (lx / nx)
    y = np.arange(ny + 1) * (ly / ny)
    z = lz * bump_nodes(nz, bump_z)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    m = structured_box(X, Y, Z, names=("periodic_x0", "periodic_xL", "periodic_y0", "periodic_yL",
                                       "bottom_wall", "top_wall"))
    return m


def urban_box(nx, ny, nz, lx=1000.0, ly=1000.0, lz=300.0, n_blocks=200, seed=20261208, side=(10.0, 60.0),
              height=(10.0, 80.0), margin=40.0):
    """Urban canopy: uniform hex box with seeded cuboid obstacles standing on the ground carved
    out (fifth configuration).  Block i has sides side[0] + (side[1] - side[0]) u and height
    height[0] + (height[1] - height[0]) u (u: SplitMix64 draws), its centre placed uniformly so
    that it keeps `margin` from the lateral boundaries (which stay periodic); a cell is removed
    when its centre lies inside a block.  Patches: x0, xL, y0, yL (lateral), ground, top,
    obstacles (every face between a fluid cell and a removed one)."""
    dx, dy, dz = lx / nx, ly / ny, lz / nz
    r = _fast_uniform(5 * n_blocks, seed).reshape(n_blocks, 5)
    sx = side[0] + (side[1] - side[0]) * r[:, 0]
    sy = side[0] + (side[1] - side[0]) * r[:, 1]
    hz = height[0] + (height[1] - height[0]) * r[:, 2]
    cx = margin + 0.5 * sx + (lx - 2.0 * margin - sx) * r[:, 3]
    cy = margin + 0.5 * sy + (ly - 2.0 * margin - sy) * r[:, 4]
    solid = np.zeros((nz, ny, nx), dtype=bool)
    for b in range(n_blocks):
        # cells whose centre (i + 1/2) h lies in [c - s/2, c + s/2]
        i0 = max(0, int(math.ceil((cx[b] - 0.5 * sx[b]) / dx - 0.5)))
        i1 = min(nx - 1, int(math.floor((cx[b] + 0.5 * sx[b]) / dx - 0.5)))
        j0 = max(0, int(math.ceil((cy[b] - 0.5 * sy[b]) / dy - 0.5)))
        j1 = min(ny - 1, int(math.floor((cy[b] + 0.5 * sy[b]) / dy - 0.5)))
        k1 = min(nz - 1, int(math.floor(hz[b] / dz - 0.5)))
        if i1 >= i0 and j1 >= j0 and k1 >= 0:
            solid[: k1 + 1, j0 : j1 + 1, i0 : i1 + 1] = True
    fluid = ~solid
    x = np.arange(nx + 1) * dx
    y = np.arange(ny + 1) * dy
    z = np.arange(nz + 1) * dz
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    xyz = np.stack([X.transpose(2, 1, 0).ravel(), Y.transpose(2, 1, 0).ravel(), Z.transpose(2, 1, 0).ravel()], axis=1)

    def nid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    k, j, i = np.nonzero(fluid)  # k, j, i order, as the structured box numbers its hexes
    hexes = np.stack([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
                      nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)], axis=1)
    quads, patch = [], []

    def add(pid, q):
        quads.append(q)
        patch.append(np.full(q.shape[0], pid, dtype=np.int32))

    def xface(ip, j, k):
        return np.stack([nid(ip, j, k), nid(ip, j + 1, k), nid(ip, j + 1, k + 1), nid(ip, j, k + 1)], 1)

    def yface(i, jp, k):
        return np.stack([nid(i, jp, k), nid(i + 1, jp, k), nid(i + 1, jp, k + 1), nid(i, jp, k + 1)], 1)

    def zface(i, j, kp):
        return np.stack([nid(i, j, kp), nid(i + 1, j, kp), nid(i + 1, j + 1, kp), nid(i, j + 1, kp)], 1)

    k, j = np.nonzero(fluid[:, :, 0])
    add(0, xface(0, j, k))
    k, j = np.nonzero(fluid[:, :, nx - 1])
    add(1, xface(nx, j, k))
    k, i = np.nonzero(fluid[:, 0, :])
    add(2, yface(i, 0, k))
    k, i = np.nonzero(fluid[:, ny - 1, :])
    add(3, yface(i, ny, k))
    j, i = np.nonzero(fluid[0])
    add(4, zface(i, j, 0))
    j, i = np.nonzero(fluid[nz - 1])
    add(5, zface(i, j, nz))
    obs = []
    m = fluid[:, :, :-1] != fluid[:, :, 1:]        # x-neighbours, one fluid one solid
    k, j, i = np.nonzero(m)
    obs.append(xface(i + 1, j, k))
    m = fluid[:, :-1, :] != fluid[:, 1:, :]
    k, j, i = np.nonzero(m)
    obs.append(yface(i, j + 1, k))
    m = fluid[:-1] != fluid[1:]
    k, j, i = np.nonzero(m)
    obs.append(zface(i, j, k + 1))
    add(6, np.concatenate(obs))
    q = np.concatenate(quads).astype(np.int32)
    nh = hexes.shape[0]
    return RawMesh(
        xyz=np.ascontiguousarray(xyz, dtype=np.float64),
        cell_type=np.full(nh, abi.EL_HEX8, dtype=np.int32),
        cell_off=np.arange(0, 8 * nh + 1, 8, dtype=np.int64),
        cell_nodes=hexes.astype(np.int32).ravel(),
        bface_off=np.arange(0, 4 * q.shape[0] + 1, 4, dtype=np.int64),
        bface_nodes=q.ravel(),
        bface_patch=np.concatenate(patch),
        patch_names=["x0", "xL", "y0", "yL", "ground", "top", "obstacles"],
    )


def _jittered_grid(n, jitter, seed):
    """Nodes of the unit cube's n^3 grid, interior nodes moved by a seeded uniform draw in
    [-jitter, jitter] * h per coordinate (boundary nodes stay, so the box stays a periodic box)."""
    h = 1.0 / n
    g = np.arange(n + 1) * h
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    xyz = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], 1)  # id = i + (n+1)(j + (n+1)k)
    r = _fast_uniform(xyz.size, seed).reshape(xyz.shape)
    i = np.arange(n + 1)
    I, J, K = np.meshgrid(i, i, i, indexing="ij")
    interior = ((I > 0) & (I < n) & (J > 0) & (J < n) & (K > 0) & (K < n)).ravel(order="F")
    xyz[interior] += jitter * h * (2.0 * r[interior] - 1.0)
    return xyz


def _hex_nodes(n, i, j, k):
    nid = lambda a, b, c: a + (n + 1) * (b + (n + 1) * c)
    return [nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
            nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)]


_PATCHES6 = ("x0", "xL", "y0", "yL", "z0", "zL")


@dataclass
class PolyMesh:
    """Face-based mesh as an OpenFOAM polyMesh holds it (dpm_create_poly): faces in the file's
    order (internal faces first, owner < neighbour), then each patch's faces."""
    xyz: np.ndarray            # (n_points, 3) float64
    face_off: np.ndarray       # (n_faces+1,) int64
    face_nodes: np.ndarray     # int32
    owner: np.ndarray          # (n_faces,) int32
    neighbour: np.ndarray      # (n_int_faces,) int32
    patch_start: np.ndarray    # (n_patches,) int64, startFace
    patch_nfaces: np.ndarray   # (n_patches,) int64
    patch_names: list = field(default_factory=list)
    patch_types: list = field(default_factory=list)

    @property
    def n_cells(self):
        return int(max(self.owner.max(initial=-1), self.neighbour.max(initial=-1))) + 1

    def vertex_bounds(self):
        return self.xyz.min(axis=0), self.xyz.max(axis=0)


def _assemble(xyz, cells, bfaces):
    """cells: [(type, [nodes])], bfaces: [(patch, [nodes])] -> RawMesh."""
    ct = np.array([c[0] for c in cells], dtype=np.int32)
    cn = np.concatenate([np.asarray(c[1], dtype=np.int32) for c in cells])
    co = np.concatenate([[0], np.cumsum([len(c[1]) for c in cells])]).astype(np.int64)
    bp = np.array([b[0] for b in bfaces], dtype=np.int32)
    bn = np.concatenate([np.asarray(b[1], dtype=np.int32) for b in bfaces])
    bo = np.concatenate([[0], np.cumsum([len(b[1]) for b in bfaces])]).astype(np.int64)
    return RawMesh(xyz=np.ascontiguousarray(xyz), cell_type=ct, cell_off=co, cell_nodes=cn, bface_off=bo,
                   bface_nodes=bn, bface_patch=bp, patch_names=list(_PATCHES6))


# hex faces on the box boundary: (patch, local quad) and the two triangles of the split along
# the main diagonal v0-v6 (consistent across neighbours and across periodic pairs)
_HEX_BFACES = {0: (0, 3, 7, 4), 1: (1, 2, 6, 5), 2: (0, 1, 5, 4), 3: (3, 2, 6, 7), 4: (0, 1, 2, 3), 5: (4, 5, 6, 7)}
_KUHN_TRI = {0: ((0, 3, 7), (0, 7, 4)), 1: ((1, 2, 6), (1, 6, 5)), 2: ((0, 1, 5), (0, 5, 4)),
             3: ((2, 3, 6), (3, 7, 6)), 4: ((0, 1, 2), (0, 2, 3)), 5: ((4, 5, 6), (4, 6, 7))}
_KUHN_TETS = ((0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6))


def _boundary_sides(n, i, j, k):
    out = []
    if i == 0: out.append(0)
    if i == n - 1: out.append(1)
    if j == 0: out.append(2)
    if j == n - 1: out.append(3)
    if k == 0: out.append(4)
    if k == n - 1: out.append(5)
    return out


def tet_box(n, jitter=0.2, seed=20261204):
    """Unit cube of n^3 jittered hexes, each split into 6 tetrahedra around its main diagonal
    (a conforming all-tet mesh; periodic pairs match)."""
    xyz = _jittered_grid(n, jitter, seed)
    cells, bf = [], []
    for k in range(n):
        for j in range(n):
            for i in range(n):
                v = _hex_nodes(n, i, j, k)
                cells += [(abi.EL_TET4, [v[a] for a in t]) for t in _KUHN_TETS]
                for sd in _boundary_sides(n, i, j, k):
                    bf += [(sd, [v[a] for a in tri]) for tri in _KUHN_TRI[sd]]
    return _assemble(xyz, cells, bf)


def mixed_box(n, jitter=0.2, seed=20261205, prism_cols=0.3, pyramid_hex=0.3):
    """Unit cube of n^3 jittered hexes in a conforming seeded mix: whole columns (fixed i, j)
    split into two prisms each along the v0-v2 diagonal (triangles only on the column's z
    faces), and, in the other columns, hexes split into 6 pyramids around an added centre node
    (their faces stay quads); the rest stay hexes."""
    xyz = _jittered_grid(n, jitter, seed)
    rc = _fast_uniform(n * n, seed + 1)
    rh = _fast_uniform(n ** 3, seed + 2)
    extra = []
    cells, bf = [], []
    for k in range(n):
        for j in range(n):
            for i in range(n):
                v = _hex_nodes(n, i, j, k)
                col = rc[i + n * j] < prism_cols
                sides = _boundary_sides(n, i, j, k)
                if col:
                    cells.append((abi.EL_PRISM6, [v[0], v[1], v[2], v[4], v[5], v[6]]))
                    cells.append((abi.EL_PRISM6, [v[0], v[2], v[3], v[4], v[6], v[7]]))
                    for sd in sides:
                        if sd == 4:
                            bf += [(4, [v[0], v[1], v[2]]), (4, [v[0], v[2], v[3]])]
                        elif sd == 5:
                            bf += [(5, [v[4], v[5], v[6]]), (5, [v[4], v[6], v[7]])]
                        else:
                            bf.append((sd, [v[a] for a in _HEX_BFACES[sd]]))
                    continue
                if rh[i + n * (j + n * k)] < pyramid_hex:
                    c = len(xyz) + len(extra)
                    extra.append(xyz[v].mean(axis=0))
                    for quad in ((0, 1, 2, 3), (4, 5, 6, 7), (0, 1, 5, 4), (3, 2, 6, 7), (0, 3, 7, 4), (1, 2, 6, 5)):
                        cells.append((abi.EL_PYR5, [v[a] for a in quad] + [c]))
                else:
                    cells.append((abi.EL_HEX8, v))
                for sd in sides:
                    bf.append((sd, [v[a] for a in _HEX_BFACES[sd]]))
    if extra:
        xyz = np.concatenate([xyz, np.array(extra)], axis=0)
    return _assemble(xyz, cells, bf)


def curl_noise_velocity(centroid, seed=20261206, k0=4.0, kmax=6):
    """Divergence-free random field: U = curl A with A a sum of Fourier modes of the unit box
    (integer wavevectors, 2 <= |k| <= kmax) whose amplitudes are seeded normal draws times a
    Gaussian spectrum exp(-(|k| - k0)^2 / 2); scaled to unit RMS."""
    r = np.arange(-kmax, kmax + 1)
    K = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3).astype(float)
    kk = np.linalg.norm(K, axis=1)
    K = K[(kk >= 2.0) & (kk <= kmax)]
    kk = np.linalg.norm(K, axis=1)
    u = _fast_uniform(4 * len(K), seed).reshape(len(K), 4)
    amp = np.sqrt(-2.0 * np.log(np.maximum(u[:, :3], 1e-300))) * np.cos(2.0 * np.pi * u[:, 3:4])  # normal draws
    amp *= np.exp(-0.5 * (kk - k0) ** 2)[:, None]
    ph = 2.0 * np.pi * u[:, 3]
    arg = 2.0 * np.pi * centroid @ K.T + ph[None, :]          # [n, modes]
    c = np.cos(arg)
    U = np.zeros_like(centroid)
    tk = 2.0 * np.pi * K
    # (curl A)_x = dAz/dy - dAy/dz, A_m = amp_m sin(arg)
    U[:, 0] = c @ (tk[:, 1] * amp[:, 2] - tk[:, 2] * amp[:, 1])
    U[:, 1] = c @ (tk[:, 2] * amp[:, 0] - tk[:, 0] * amp[:, 2])
    U[:, 2] = c @ (tk[:, 0] * amp[:, 1] - tk[:, 1] * amp[:, 0])
    return U / np.sqrt(np.mean(np.sum(U * U, axis=1)))


# ------------------------------------------------------------------------------------------
# Initial conditions (src/init/mod_initconditions.f90)
# ------------------------------------------------------------------------------------------
def taylor_green(centroid, lo, hi, u0=1.0):
    """initialize_taylor_green_ic (mod_initconditions.f90:276-334)."""
    L = hi - lo
    L = np.where(L <= 0.0, 1.0, L)
    k = 2.0 * math.pi / L
    xl = np.mod(centroid - lo, L)
    U = np.zeros_like(centroid)
    U[:, 0] = u0 * np.sin(k[0] * xl[:, 0]) * np.cos(k[1] * xl[:, 1]) * np.cos(k[2] * xl[:, 2])
    U[:, 1] = -u0 * np.cos(k[0] * xl[:, 0]) * np.sin(k[1] * xl[:, 1]) * np.cos(k[2] * xl[:, 2])
    return U


def channel_parabolic(centroid, lo, hi, uref, wall_dir=1, stream_dir=0):
    """initialize_channel_profile_ic 'parabolic' (mod_initconditions.f90:114-196)."""
    H = max(hi[wall_dir] - lo[wall_dir], 1e-30)
    zeta = np.clip((centroid[:, wall_dir] - lo[wall_dir]) / H, 0.0, 1.0)
    U = np.zeros_like(centroid)
    U[:, stream_dir] = 4.0 * uref * zeta * (1.0 - zeta)
    return U


def splitmix64_uniform(n, seed):
    """Seeded uniform draws in [0,1) from SplitMix64 (reproducible on any platform; the
    reference's gfortran random_number stream is not)."""
    out = np.empty(n, dtype=np.float64)
    mask = (1 << 64) - 1
    x = seed & mask
    for i in range(n):
        x = (x + 0x9E3779B97F4A7C15) & mask
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        z ^= z >> 31
        out[i] = (z >> 11) * (1.0 / (1 << 53))
    return out


def multiplicative_noise(U, frac, seed):
    """add_random_velocity_noise (mod_initconditions.f90:200-250): U_k *= 1 + frac (2 r - 1),
    r drawn per cell and component in the reference's loop order (cell outer, component inner)."""
    r = _fast_uniform(U.size, seed).reshape(U.shape)
    return U * (1.0 + frac * (2.0 * r - 1.0))


def _fast_uniform(n, seed):
    # vectorised SplitMix64 (identical stream to splitmix64_uniform)
    idx = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / (1 << 53))


# ------------------------------------------------------------------------------------------
# Run configurations
# ------------------------------------------------------------------------------------------
@dataclass
class Case:
    name: str
    mesh: RawMesh
    patches: list            # dicts for abi.patch_cfgs, in mesh patch order
    params: dict             # keyword arguments of abi.default_params
    ic: str                  # 'taylor_green' | 'uniform' | 'channel'
    ic_uref: float = 1.0
    noise: float = 0.0
    noise_seed: int = 12345
    n_steps: int = 20
    stats_every: int = 1
    description: str = ""

    def make_params(self):
        return abi.default_params(**self.params)

    def initial_velocity(self, centroid):
        lo, hi = self.mesh.vertex_bounds()
        if self.ic == "taylor_green":
            U = taylor_green(centroid, lo, hi, self.ic_uref)
        elif self.ic == "uniform":
            U = np.zeros_like(centroid)
            U[:, 0] = self.ic_uref
        elif self.ic == "channel":
            U = channel_parabolic(centroid, lo, hi, self.ic_uref)
        elif self.ic == "curl_noise":
            U = self.ic_uref * curl_noise_velocity(centroid)
        else:
            raise ValueError(self.ic)
        if self.noise > 0.0:
            U = multiplicative_noise(U, self.noise, self.noise_seed)
        return U


def _periodic6():
    return [{"bc": "periodic"} for _ in range(6)]


def regression_case(name):
    """The reference's regression cases whose meshes need no gmsh
    (tests/regression/cases/<name>/case.input)."""
    if name == "tgv":
        L = 6.283185307179586
        return Case(name, uniform_box(32, 32, 32, L, L, L), _periodic6(),
                    dict(scheme=abi.SCHEME_QUICK, nu=6.25e-4, dt=1.0e-2, cfl_max=0.6, p_tol=1e-10, rhie_chow_dual=0),
                    "taylor_green", 1.0, n_steps=20)
    if name == "tgv_skew":
        return Case(name, skewed_unit_box(16, 0.08), _periodic6(),
                    dict(scheme=abi.SCHEME_KEP, nu=6.25e-4, dt=2.0e-2, cfl_max=0.6, p_tol=1e-10,
                         n_nonortho_corr=3, rhie_chow_dual=1),
                    "taylor_green", 1.0, n_steps=30)
    if name == "tgv_skew_chk":
        return Case(name, skewed_unit_box(16, 0.08), _periodic6(),
                    dict(scheme=abi.SCHEME_KEP, nu=6.25e-4, dt=2.0e-2, cfl_max=0.6, p_tol=1e-10,
                         n_nonortho_corr=5, nonortho_check=1, rhie_chow_dual=1),
                    "taylor_green", 1.0, n_steps=30)
    if name in ("tgv_skew_exact", "default_skew"):
        # the exact cell projection on the 45-degree box; default_skew states no numerics at all,
        # and the reference's defaults are these (mod_input_parser.f90:197-201)
        return Case(name, skewed_unit_box(16, 0.08), _periodic6(),
                    dict(scheme=abi.SCHEME_KEP, nu=6.25e-4, dt=2.0e-2, cfl_max=0.6, p_tol=1e-10,
                         n_nonortho_corr=3, rhie_chow_dual=1, cell_projection=abi.CELL_PROJECTION_EXACT),
                    "taylor_green", 1.0, n_steps=30)
    if name in ("pdrop", "hydro", "hydro_exact"):
        fz = 0.0 if name == "pdrop" else -1.0
        patches = [{"bc": "periodic"}] * 4 + [{"bc": "outlet", "p": 1.0}, {"bc": "outlet", "p": 0.0}]
        prm = dict(scheme=abi.SCHEME_CDS, nu=1.0e-2, dt=2.0e-3, cfl_max=0.5, p_tol=1e-12,
                   n_nonortho_corr=4, rhie_chow_dual=0, f_const=(0.0, 0.0, fz))
        if name == "hydro_exact":
            prm["cell_projection"] = abi.CELL_PROJECTION_EXACT
        return Case(name, skewed_unit_box(12, 0.04), patches, prm, "uniform", 0.0, n_steps=20, stats_every=10)
    if name in ("inflow", "inflow_jarrin"):
        # synthetic-eddy inflow on the 12^3 skewed box: ABL inlet at x0 (log law u_ref 1 at z_ref 0.5,
        # z0 0.01, 300 eddies of scale 0.2), outlet p = 0 at xL, periodic y, slip z
        patches = [{"bc": "ablInlet"}, {"bc": "outlet", "p": 0.0}, {"bc": "periodic"}, {"bc": "periodic"},
                   {"bc": "slip"}, {"bc": "slip"}]
        prm = dict(scheme=abi.SCHEME_CDS, nu=1.0e-3, dt=5.0e-3, cfl_max=0.5, p_tol=1e-12, p_max_iter=1000,
                   n_nonortho_corr=3, rhie_chow_dual=0, sgs_model=abi.SGS_NONE, wall_model=abi.WM_NONE,
                   abl_u_ref=1.0, abl_z_ref=0.5, abl_z0_m=0.01, abl_wind_dir_deg=270.0, use_sem=1,
                   sem_type=abi.SEM_JARRIN if name == "inflow_jarrin" else abi.SEM_DFSEM, sem_n_eddies=300,
                   sem_sigma=0.2)
        return Case(name, skewed_unit_box(12, 0.04), patches, prm, "uniform", 1.0, n_steps=20, stats_every=5)
    if name in ("duct", "duct_exact"):
        # 32x16x16 duct 4 x 1 x 1 on the RB.geo wall box: velocity inlet at x0, outlet p = 0 at xL,
        # periodic in y, no-slip bottom and top
        patches = [{"bc": "inlet", "U": (1.0, 0.0, 0.0)}, {"bc": "outlet", "p": 0.0}, {"bc": "periodic"},
                   {"bc": "periodic"}, {"bc": "noSlip"}, {"bc": "noSlip"}]
        prm = dict(scheme=abi.SCHEME_CDS, nu=1.0e-2, dt=1.0e-2, cfl_max=0.5, p_tol=1e-10, p_max_iter=1000,
                   rhie_chow_dual=0, sgs_model=abi.SGS_NONE)
        if name == "duct_exact":
            prm["cell_projection"] = abi.CELL_PROJECTION_EXACT
        return Case(name, wall_box(32, 16, 16, 4.0, 1.0, 1.0, 0.25), patches, prm, "uniform", 1.0, n_steps=20)
    if name == "hydrowall":
        patches = [{"bc": "noSlip"}] * 6
        return Case(name, skewed_unit_box(12, 0.04), patches,
                    dict(scheme=abi.SCHEME_CDS, nu=1.0e-2, dt=2.0e-3, cfl_max=0.5, p_tol=1e-12,
                         n_nonortho_corr=4, rhie_chow_dual=0, f_const=(0.0, 0.0, -1.0)),
                    "uniform", 0.0, n_steps=20, stats_every=10)
    if name == "rb":
        # 24x24x16 Rayleigh-Benard: fixed-temperature walls T=1 (bottom) / 0 (top), Boussinesq
        patches = [{"bc": "periodic"}] * 4 + [{"bc": "fixedTemp", "T": 1.0}, {"bc": "fixedTemp", "T": 0.0}]
        return Case(name, wall_box(24, 24, 16, 2.0, 2.0, 1.0, 0.25), patches,
                    dict(scheme=abi.SCHEME_KEP, temperature_scheme=abi.SCHEME_VANLEER_TVD, nu=6.3246e-4,
                         alpha_T=6.3246e-4, beta=1.0, T_ref=0.5, g=(0.0, 0.0, -1.0), boussinesq=1, dt=5.0e-2,
                         cfl_max=0.5, p_tol=1e-10, p_max_iter=500, rhie_chow_dual=0, sgs_model=abi.SGS_NONE,
                         wall_model=abi.WM_NONE),
                    "uniform", 1.0e-2, n_steps=20)
    if name == "channel_most":
        # as 'channel' with the MOST wall model (z0_m 1e-3, z0_h 1e-4, T_surface 298) and Boussinesq
        L = 6.283185307179586
        wall = {"bc": "wallModel"}
        patches = [{"bc": "periodic"}] * 4 + [dict(wall, scalar_mode=(1, 0, 0, 0), scalar_value=(1.0, 0, 0, 0)),
                                              dict(wall)]
        prm = dict(scheme=abi.SCHEME_KEP, sgs_model=abi.SGS_VREMAN, wall_model=abi.WM_MOST, nu=2.5316e-3,
                   f_const=(1.0, 0.0, 0.0), g=(0.0, 0.0, -9.80665), boussinesq=1, dt=2.0e-3, cfl_max=0.5,
                   p_tol=1e-10, p_max_iter=1000, rhie_chow_dual=0, n_scalars=1, scalar_scheme=abi.SCHEME_VANLEER_TVD,
                   scalar_diffusivity=(1.0e-3, 0, 0, 0), scalar_pr_t=(1.0, 0, 0, 0), abl_z0_m=1.0e-3,
                   abl_z0_h=1.0e-4, abl_T_surface=298.0)
        return Case(name, wall_box(32, 16, 16, L, L, 1.0, 0.25), patches, prm, "taylor_green", 1.0, n_steps=20)
    if name in ("channel", "amd", "graded"):
        # 32x16x16 wall-bounded box 2pi x 2pi x 1 with a Taylor-Green field, KEP, log-law wall
        # model, f_x = 1, one passive tracer with a Dirichlet value 1 on the bottom wall
        L = 6.283185307179586
        bump = 0.01 if name == "graded" else 0.25
        wall = {"bc": "wallModel"}
        patches = [{"bc": "periodic"}] * 4 + [dict(wall, scalar_mode=(1, 0, 0, 0), scalar_value=(1.0, 0, 0, 0)),
                                              dict(wall)]
        prm = dict(scheme=abi.SCHEME_KEP, sgs_model=abi.SGS_AMD if name == "amd" else abi.SGS_VREMAN,
                   wall_model=abi.WM_LOGLAW, nu=2.5316e-3, f_const=(1.0, 0.0, 0.0), dt=2.0e-3, cfl_max=0.5,
                   p_tol=1e-10, p_max_iter=1000, rhie_chow_dual=0, n_scalars=1,
                   scalar_scheme=abi.SCHEME_VANLEER_TVD, scalar_diffusivity=(1.0e-3, 0, 0, 0),
                   scalar_pr_t=(1.0, 0, 0, 0))
        if name == "amd":
            prm["wall_model_filter_tf_fac"] = 1.0
        return Case(name, wall_box(32, 16, 16, L, L, 1.0, bump), patches, prm, "taylor_green", 1.0, n_steps=20)
    raise KeyError(name)


REGRESSION_CASES = ("tgv", "tgv_skew", "tgv_skew_chk", "pdrop", "hydro", "hydrowall", "rb", "channel", "amd",
                    "graded", "channel_most")


def tgv_config(n=32, n_steps=200, scheme=abi.SCHEME_CDS):
    """Taylor-Green vortex, periodic [0,2pi]^3 hex box, nu=1/1600, no SGS, CDS, dt=0.01,
    Jacobi-PCG to rtol 1e-10 (first configuration)."""
    L = 2.0 * math.pi
    return Case(f"tgv{n}", uniform_box(n, n, n, L, L, L), _periodic6(),
                dict(scheme=scheme, nu=1.0 / 1600.0, dt=0.01, cfl_max=0.6, p_tol=1e-10),
                "taylor_green", 1.0, n_steps=n_steps,
                description=f"Taylor-Green vortex {n}^3 periodic hex box, CDS, nu=1/1600, dt=0.01")


def channel_config(nx=96, ny=64, nz=64, n_steps=1000, retau=395.0, noise_seed=20261203):
    """Turbulent channel 2pi x 2 x pi, tanh stretching 2.0 in y, walls at y=+-1 (log-law wall
    model), periodic x and z, Vreman SGS, KEP advection, constant streamwise pressure gradient
    u_tau^2/delta = 1 with u_tau = 1, nu = u_tau delta / Re_tau; laminar parabola with seeded
    +-10% multiplicative noise (second configuration)."""
    mesh = channel_box(nx, ny, nz, 2.0 * math.pi, 2.0, math.pi, 2.0)
    patches = [{"bc": "periodic"}, {"bc": "periodic"}, {"bc": "wallModel"}, {"bc": "wallModel"},
               {"bc": "periodic"}, {"bc": "periodic"}]
    nu = 1.0 / retau
    # bulk velocity of the log-law profile at Re_tau 395 is about 17.5 u_tau; dt keeps CFL ~0.3
    ub = 17.5
    dx = 2.0 * math.pi / nx
    dt = 0.3 * dx / (1.5 * ub)
    return Case(f"channel{nx}x{ny}x{nz}", mesh, patches,
                dict(scheme=abi.SCHEME_KEP, sgs_model=abi.SGS_VREMAN, wall_model=abi.WM_LOGLAW,
                     nu=nu, dt=dt, cfl_max=0.5, p_tol=1e-10, f_const=(1.0, 0.0, 0.0)),
                "channel", 1.5 * ub, noise=0.10, noise_seed=noise_seed, n_steps=n_steps,
                description=f"channel {nx}x{ny}x{nz} Re_tau={retau:g}, KEP, Vreman, log-law wall model")


def rb_config(nx=256, ny=256, nz=128, n_steps=10, noise_seed=20261207):
    """Rayleigh-Benard convection (fourth configuration): 4 x 4 x 1 box, periodic sides, walls at
    z = 0 (T = 1) and z = 1 (T = 0) with Bump-graded spacing, Boussinesq with g beta dT H = 1,
    Ra = 1e7 and Pr = 0.7 (nu = sqrt(Pr / Ra), kappa = nu / Pr), KEP momentum, Vreman SGS, van
    Leer TVD temperature and two passive scalars (Dirichlet 1 on the bottom wall for the first,
    on the top wall for the second).  The seeded perturbation is +-10 % multiplicative noise on a
    uniform 1e-2 drift velocity."""
    ra, pr = 1.0e7, 0.7
    nu = math.sqrt(pr / ra)
    kappa = nu / pr
    bottom = {"bc": "fixedTemp", "T": 1.0, "scalar_mode": (1, 0, 0, 0), "scalar_value": (1.0, 0, 0, 0)}
    top = {"bc": "fixedTemp", "T": 0.0, "scalar_mode": (0, 1, 0, 0), "scalar_value": (0, 1.0, 0, 0)}
    patches = [{"bc": "periodic"}] * 4 + [bottom, top]
    h = 4.0 / nx
    prm = dict(scheme=abi.SCHEME_KEP, temperature_scheme=abi.SCHEME_VANLEER_TVD, nu=nu, alpha_T=kappa, beta=1.0,
               T_ref=0.5, g=(0.0, 0.0, -1.0), boussinesq=1, dt=0.3 * h, cfl_max=0.5, p_tol=1e-10,
               p_max_iter=20000, rhie_chow_dual=0, sgs_model=abi.SGS_VREMAN, wall_model=abi.WM_NONE, n_scalars=2,
               scalar_scheme=abi.SCHEME_VANLEER_TVD, scalar_diffusivity=(kappa, kappa, 0, 0),
               scalar_pr_t=(0.85, 0.85, 0, 0))
    return Case(f"rb{nx}x{ny}x{nz}", wall_box(nx, ny, nz, 4.0, 4.0, 1.0, 0.25), patches, prm, "uniform", 1.0e-2,
                noise=0.10, noise_seed=noise_seed, n_steps=n_steps,
                description=f"Rayleigh-Benard {nx}x{ny}x{nz}, Ra=1e7, Pr=0.7, T + 2 scalars (van Leer), Vreman")


def urban_config(nx=400, ny=400, nz=125, n_blocks=200, n_steps=10, lx=1000.0, ly=1000.0, lz=300.0,
                 noise_seed=20261209, scale=1.0):
    """Urban-canopy atmospheric boundary layer (fifth configuration): lx x ly x lz metres with
    seeded cuboid obstacles carved out (urban_box), periodic lateral boundaries, MOST wall model
    on the ground (z0_m 0.1 m, z0_h 0.01 m) and the obstacles (their own z0_m 0.05 m, z0_h 0.005 m,
    the per-patch override), surface 302 K over 300 K air, Obukhov
    length -100 m (unstable) held fixed), slip top, AMD SGS, KEP momentum, Boussinesq temperature and one
    passive scalar (Dirichlet 1 on the ground) with van Leer TVD, constant streamwise pressure
    gradient u_tau^2 / lz with u_tau = 0.5 m/s.  Initial state: 5 m/s streamwise with seeded
    +-10 % multiplicative noise.  `scale` multiplies the block sizes, their margin, the roughness
    lengths and the Obukhov length (the domain lengths are given directly): a geometrically
    scaled copy whose Poisson solves are governed by the relative tolerance rather than by the
    reference's cell-volume-based absolute one, as parity tests at small sizes need."""
    mesh = urban_box(nx, ny, nz, lx, ly, lz, n_blocks, side=(10.0 * scale, 60.0 * scale),
                     height=(10.0 * scale, 80.0 * scale), margin=40.0 * scale)
    wall = {"bc": "wallModel"}
    patches = [{"bc": "periodic"}] * 4 + [dict(wall, scalar_mode=(1, 0, 0, 0), scalar_value=(1.0, 0, 0, 0)),
                                          {"bc": "slip"}, dict(wall, z0_m=0.05 * scale, z0_h=0.005 * scale)]
    dx = lx / nx
    u0 = 5.0
    prm = dict(scheme=abi.SCHEME_KEP, sgs_model=abi.SGS_AMD, wall_model=abi.WM_MOST, nu=1.5e-5, alpha_T=2.1e-5,
               beta=1.0 / 300.0, T_ref=300.0, g=(0.0, 0.0, -9.81), boussinesq=1, temperature_scheme=abi.SCHEME_VANLEER_TVD,
               f_const=(0.25 / lz, 0.0, 0.0), dt=0.3 * dx / (1.5 * u0), cfl_max=0.5, p_tol=1e-10, p_max_iter=20000,
               rhie_chow_dual=0, n_scalars=1, scalar_scheme=abi.SCHEME_VANLEER_TVD, scalar_diffusivity=(2.1e-5, 0, 0, 0),
               scalar_pr_t=(0.85, 0, 0, 0), abl_z0_m=0.1 * scale, abl_z0_h=0.01 * scale, abl_T_surface=302.0,
               abl_L_obukhov=-100.0 * scale, abl_compute_L=0)
    return Case(f"urban{nx}x{ny}x{nz}", mesh, patches, prm, "uniform", u0, noise=0.10, noise_seed=noise_seed,
                n_steps=n_steps,
                description=f"urban canopy {nx}x{ny}x{nz} ({mesh.n_cells} fluid cells, {n_blocks} blocks), MOST, AMD")


def hybrid_config(n=16, kind="mixed", n_steps=10):
    """Non-orthogonal unstructured box (third configuration, reduced size): unit cube of n^3
    jittered (+-0.2 h) hexes as a conforming mix of hexes, prisms and pyramids ("mixed") or as
    all tetrahedra ("tet"), periodic, AMD SGS, Koren TVD momentum advection, divergence-free
    curl-noise initial velocity (peak |k| = 4)."""
    mesh = mixed_box(n) if kind == "mixed" else tet_box(n)
    h = 1.0 / n
    return Case(f"hybrid_{kind}{n}", mesh, _periodic6(),
                dict(scheme=abi.SCHEME_KOREN_TVD, sgs_model=abi.SGS_AMD, wall_model=abi.WM_NONE, nu=1.0e-3,
                     dt=0.2 * h / 3.0, cfl_max=0.5, p_tol=1e-10, n_nonortho_corr=3),
                "curl_noise", 1.0, n_steps=n_steps,
                description=f"{kind} unstructured jittered unit box {n}^3, AMD, Koren")
