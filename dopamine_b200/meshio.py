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
