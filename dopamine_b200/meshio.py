"""Mesh ingestion: gmsh v4.1 ASCII files to the raw arrays dpm_create takes, and back.

The reader is the product library's (csrc/host/gmsh.cpp, dpm_gmsh_read), which follows the
reference's src/mesh/mod_gmsh_reader.f90:gmsh_read: cells are the volume elements in file order,
boundary faces the triangles and quads, patches the 2-D physical groups that hold faces.
"""
import ctypes as C

import numpy as np

from . import abi
from .cases import RawMesh
from .solver import DopamineError, lib


def _bind(L):
    if getattr(L, "_gmsh_bound", False):
        return L
    vp = C.c_void_p
    L.dpm_gmsh_read.argtypes = [C.c_char_p, C.POINTER(vp), C.c_char_p, C.c_int]
    L.dpm_gmsh_sizes.argtypes = [vp] + [C.POINTER(C.c_int64)] * 5 + [C.POINTER(C.c_int)]
    L.dpm_gmsh_fill.argtypes = [vp] + [vp] * 7
    L.dpm_gmsh_patch_name.argtypes = [vp, C.c_int]
    L.dpm_gmsh_patch_name.restype = C.c_char_p
    L.dpm_gmsh_free.argtypes = [vp]
    L.dpm_gmsh_write.argtypes = [C.c_char_p, C.POINTER(abi.RawMeshT), C.POINTER(C.c_char_p)]
    L._gmsh_bound = True
    return L


def read_gmsh(path):
    """Reads a gmsh v4.1 ASCII file into a RawMesh (patch_names from the physical groups)."""
    L = _bind(lib())
    h = C.c_void_p()
    err = C.create_string_buffer(512)
    rc = L.dpm_gmsh_read(str(path).encode(), C.byref(h), err, len(err))
    if rc != 0:
        raise DopamineError(f"dpm_gmsh_read: {err.value.decode()}", rc)
    try:
        n = [C.c_int64() for _ in range(5)]
        npatch = C.c_int()
        L.dpm_gmsh_sizes(h, *[C.byref(x) for x in n], C.byref(npatch))
        nn, nc, ncn, nb, nbn = (x.value for x in n)
        m = RawMesh(xyz=np.zeros((nn, 3)), cell_type=np.zeros(nc, np.int32), cell_off=np.zeros(nc + 1, np.int64),
                    cell_nodes=np.zeros(ncn, np.int32), bface_off=np.zeros(nb + 1, np.int64),
                    bface_nodes=np.zeros(nbn, np.int32), bface_patch=np.zeros(nb, np.int32))
        arrs = (m.xyz, m.cell_type, m.cell_off, m.cell_nodes, m.bface_off, m.bface_nodes, m.bface_patch)
        L.dpm_gmsh_fill(h, *[a.ctypes.data_as(C.c_void_p) for a in arrs])
        m.patch_names = [L.dpm_gmsh_patch_name(h, k).decode() for k in range(npatch.value)]
    finally:
        L.dpm_gmsh_free(h)
    return m


def write_gmsh(path, mesh):
    """Writes a RawMesh as a gmsh v4.1 ASCII file that read_gmsh reads back to the same mesh."""
    L = _bind(lib())
    view = abi.RawMeshView(mesh)
    names = (C.c_char_p * max(len(mesh.patch_names), 1))(*[s.encode() for s in mesh.patch_names])
    rc = L.dpm_gmsh_write(str(path).encode(), C.byref(view.struct), names)
    if rc != 0:
        raise DopamineError(f"dpm_gmsh_write failed for {path}", rc)


# ---- OpenFOAM polyMesh ---------------------------------------------------------------------------

def _bind_foam(L):
    if getattr(L, "_foam_bound", False):
        return L
    vp = C.c_void_p
    L.dpm_foam_read.argtypes = [C.c_char_p, C.POINTER(vp), C.c_char_p, C.c_int]
    L.dpm_foam_sizes.argtypes = [vp] + [C.POINTER(C.c_int64)] * 4 + [C.POINTER(C.c_int)]
    L.dpm_foam_fill.argtypes = [vp] + [vp] * 7
    L.dpm_foam_patch_name.argtypes = [vp, C.c_int]
    L.dpm_foam_patch_name.restype = C.c_char_p
    L.dpm_foam_patch_type.argtypes = [vp, C.c_int]
    L.dpm_foam_patch_type.restype = C.c_char_p
    L.dpm_foam_free.argtypes = [vp]
    L.dpm_poly_cell_geometry.argtypes = [C.POINTER(abi.PolyMeshT), C.POINTER(C.c_int), vp, vp, C.c_char_p, C.c_int]
    L._foam_bound = True
    return L


def read_foam(polymesh_dir):
    """Reads an ASCII OpenFOAM polyMesh directory into a cases.PolyMesh (patch names and types
    from the boundary file)."""
    from .cases import PolyMesh
    L = _bind_foam(lib())
    h = C.c_void_p()
    err = C.create_string_buffer(512)
    rc = L.dpm_foam_read(str(polymesh_dir).encode(), C.byref(h), err, len(err))
    if rc != 0:
        raise DopamineError(f"dpm_foam_read: {err.value.decode()}", rc)
    try:
        n = [C.c_int64() for _ in range(4)]
        npatch = C.c_int()
        L.dpm_foam_sizes(h, *[C.byref(x) for x in n], C.byref(npatch))
        npts, nf, nfn, nfi = (x.value for x in n)
        m = PolyMesh(xyz=np.zeros((npts, 3)), face_off=np.zeros(nf + 1, np.int64), face_nodes=np.zeros(nfn, np.int32),
                     owner=np.zeros(nf, np.int32), neighbour=np.zeros(nfi, np.int32),
                     patch_start=np.zeros(npatch.value, np.int64), patch_nfaces=np.zeros(npatch.value, np.int64))
        arrs = (m.xyz, m.face_off, m.face_nodes, m.owner, m.neighbour, m.patch_start, m.patch_nfaces)
        L.dpm_foam_fill(h, *[a.ctypes.data_as(C.c_void_p) for a in arrs])
        m.patch_names = [L.dpm_foam_patch_name(h, k).decode() for k in range(npatch.value)]
        m.patch_types = [L.dpm_foam_patch_type(h, k).decode() for k in range(npatch.value)]
    finally:
        L.dpm_foam_free(h)
    return m


# local faces of the gmsh element types, as csrc/host/mesh.cpp lists them
_ELEM_FACES = {4: ((0, 1, 2), (0, 1, 3), (1, 2, 3), (0, 2, 3)),
               5: ((0, 1, 2, 3), (4, 5, 6, 7), (0, 1, 5, 4), (2, 3, 7, 6), (0, 3, 7, 4), (1, 2, 6, 5)),
               6: ((0, 1, 2), (3, 4, 5), (0, 1, 4, 3), (1, 2, 5, 4), (0, 2, 5, 3)),
               7: ((0, 1, 2, 3), (0, 1, 4), (1, 2, 4), (2, 3, 4), (0, 3, 4))}


def _area_vec(xyz, nodes):
    p = xyz[list(nodes)]
    a = np.zeros(3)
    for i in range(1, len(nodes) - 1):
        a += 0.5 * np.cross(p[i] - p[0], p[i + 1] - p[0])
    return a


def to_poly(mesh):
    """The face-based (OpenFOAM) form of an element mesh (cases.RawMesh): internal faces in
    OpenFOAM's upper-triangular order (by owner, then neighbour; owner < neighbour), each oriented
    from owner to neighbour, then each patch's faces in the mesh's boundary-face order, oriented
    out of the domain."""
    from .cases import PolyMesh
    xyz = mesh.xyz
    nc = mesh.n_cells
    cen = np.array([xyz[mesh.cell_nodes[mesh.cell_off[c]:mesh.cell_off[c + 1]]].mean(axis=0) for c in range(nc)])
    faces = {}
    for c in range(nc):
        n = mesh.cell_nodes[mesh.cell_off[c]:mesh.cell_off[c + 1]]
        for lf in _ELEM_FACES[int(mesh.cell_type[c])]:
            nodes = tuple(int(n[i]) for i in lf)
            faces.setdefault(tuple(sorted(nodes)), []).append((c, nodes))
    internal = []
    for key, lst in faces.items():
        if len(lst) == 2:
            (c0, n0), (c1, _) = lst
            o, nb = (c0, c1) if c0 < c1 else (c1, c0)
            nodes = n0
            if np.dot(_area_vec(xyz, nodes), cen[nb] - cen[o]) < 0:
                nodes = tuple(reversed(nodes))
            internal.append((o, nb, nodes))
    internal.sort(key=lambda t: (t[0], t[1]))
    bnd = [[] for _ in mesh.patch_names]
    for b in range(mesh.bface_patch.shape[0]):
        nodes = tuple(int(v) for v in mesh.bface_nodes[mesh.bface_off[b]:mesh.bface_off[b + 1]])
        o = faces[tuple(sorted(nodes))][0][0]
        fc = xyz[list(nodes)].mean(axis=0)
        if np.dot(_area_vec(xyz, nodes), fc - cen[o]) < 0:
            nodes = tuple(reversed(nodes))
        bnd[int(mesh.bface_patch[b])].append((o, nodes))
    flist = [t[2] for t in internal] + [n for p in bnd for (_, n) in p]
    owner = [t[0] for t in internal] + [o for p in bnd for (o, _) in p]
    nfi = len(internal)
    starts = np.cumsum([nfi] + [len(p) for p in bnd])[:-1]
    return PolyMesh(xyz=np.ascontiguousarray(xyz, dtype=np.float64),
                    face_off=np.concatenate([[0], np.cumsum([len(f) for f in flist])]).astype(np.int64),
                    face_nodes=np.array([v for f in flist for v in f], dtype=np.int32),
                    owner=np.array(owner, dtype=np.int32),
                    neighbour=np.array([t[1] for t in internal], dtype=np.int32),
                    patch_start=np.asarray(starts, dtype=np.int64),
                    patch_nfaces=np.array([len(p) for p in bnd], dtype=np.int64),
                    patch_names=list(mesh.patch_names), patch_types=["patch"] * len(mesh.patch_names))


def _foam_header(cls, obj, note=None, binary=False, arch=None):
    s = ("FoamFile\n{\n    version     2.0;\n"
         f"    format      {'binary' if binary else 'ascii'};\n")
    if arch:
        s += f'    arch        "{arch}";\n'
    s += f"    class       {cls};\n"
    if note:
        s += f'    note        "{note}";\n'
    s += f'    location    "constant/polyMesh";\n    object      {obj};\n}}\n\n'
    return s


def write_foam(polymesh_dir, mesh, binary=False, compact=False, label_bytes=4, big_endian=False):
    """Writes a mesh (cases.PolyMesh, or an element mesh converted by to_poly) as an OpenFOAM
    polyMesh directory that read_foam reads back to the same arrays: ASCII by default, or binary
    (labels of label_bytes bytes, 64-bit scalars, little- or big-endian), faces as a faceList or a
    faceCompactList."""
    import os
    from .cases import PolyMesh
    pm = mesh if isinstance(mesh, PolyMesh) else to_poly(mesh)
    os.makedirs(polymesh_dir, exist_ok=True)
    nf = pm.owner.shape[0]
    order = ">" if big_endian else "<"
    lab = np.dtype(f"{order}i{label_bytes}")
    arch = f"{'MSB' if big_endian else 'LSB'};label={8 * label_bytes};scalar=64" if binary else None
    nc = pm.n_cells
    note = f"nPoints:{pm.xyz.shape[0]} nCells:{nc} nFaces:{nf} nInternalFaces:{pm.neighbour.shape[0]}"

    def put(name, cls, body, note_=None):
        with open(os.path.join(polymesh_dir, name), "wb") as fh:
            fh.write(_foam_header(cls, name, note_, binary, arch).encode())
            fh.write(body)

    def blist(arr, dtype):
        return f"{arr.size // (3 if dtype.kind == 'f' else 1)}\n(".encode() + np.ascontiguousarray(arr, dtype=dtype).tobytes() + b")\n"

    def alist(items):
        return (f"{len(items)}\n(\n" + "\n".join(items) + "\n)\n").encode()

    if binary:
        put("points", "vectorField", blist(pm.xyz.ravel(), np.dtype(f"{order}f8")))
    else:
        put("points", "vectorField", alist([f"({p[0]:.17g} {p[1]:.17g} {p[2]:.17g})" for p in pm.xyz]))
    if compact:
        off = np.asarray(pm.face_off, dtype=np.int64)
        if binary:
            body = (f"{off.size}\n(".encode() + off.astype(lab).tobytes() + b")\n" +
                    f"{pm.face_nodes.size}\n(".encode() + pm.face_nodes.astype(lab).tobytes() + b")\n")
        else:
            body = alist([str(int(v)) for v in off]) + alist([str(int(v)) for v in pm.face_nodes])
        put("faces", "faceCompactList", body)
    elif binary:
        parts = []
        for f in range(nf):
            nodes = pm.face_nodes[pm.face_off[f]:pm.face_off[f + 1]]
            parts.append(np.concatenate([[len(nodes)], nodes]).astype(lab).tobytes())
        put("faces", "faceList", f"{nf}\n(".encode() + b"".join(parts) + b")\n")
    else:
        put("faces", "faceList", alist([f"{pm.face_off[f + 1] - pm.face_off[f]}(" +
                                        " ".join(str(int(v)) for v in pm.face_nodes[pm.face_off[f]:pm.face_off[f + 1]]) + ")"
                                        for f in range(nf)]))
    for name, arr in (("owner", pm.owner), ("neighbour", pm.neighbour)):
        if binary:
            put(name, "labelList", f"{arr.size}\n(".encode() + arr.astype(lab).tobytes() + b")\n", note)
        else:
            put(name, "labelList", alist([str(int(v)) for v in arr]), note)
    types = pm.patch_types or ["patch"] * len(pm.patch_names)
    body = f"{len(pm.patch_names)}\n(\n"
    for k, name in enumerate(pm.patch_names):
        body += (f"    {name}\n    {{\n        type            {types[k]};\n"
                 f"        nFaces          {int(pm.patch_nfaces[k])};\n"
                 f"        startFace       {int(pm.patch_start[k])};\n    }}\n")
    body += ")\n"
    with open(os.path.join(polymesh_dir, "boundary"), "wb") as fh:  # always ASCII, as OpenFOAM writes it
        fh.write(_foam_header("polyBoundaryMesh", "boundary").encode())
        fh.write(body.encode())


def poly_cell_geometry(pm, patch_bc):
    """Cell centroids (n_cells, 3) and volumes of a cases.PolyMesh from the host polyhedral set-up
    (dpm_poly_cell_geometry); patch_bc: the bc id of every patch."""
    L = _bind_foam(lib())
    view = abi.PolyMeshView(pm)
    nc = pm.n_cells
    cen, vol = np.zeros((nc, 3)), np.zeros(nc)
    bcs = (C.c_int * max(len(patch_bc), 1))(*[int(b) for b in patch_bc])
    err = C.create_string_buffer(256)
    rc = L.dpm_poly_cell_geometry(C.byref(view.struct), bcs, cen.ctypes.data_as(C.c_void_p),
                                  vol.ctypes.data_as(C.c_void_p), err, len(err))
    if rc != 0:
        raise DopamineError(f"dpm_poly_cell_geometry: {err.value.decode()}", rc)
    return cen, vol
