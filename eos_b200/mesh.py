"""Triangle meshes from Wavefront OBJ files (eos_mesh_* of the C ABI) and scenes built from them.

The loader is the library's C++ code (host only, no GPU needed): triangulation, smooth
normals when the file has none and joining of identical vertices, as TriangleMesh::
loadFromFile gets them from assimp in the reference (src/triangleMesh.cpp:79-160).
"""
from __future__ import annotations

from ctypes import byref, c_void_p
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .scenes import LIGHT_STRIDE, SceneData, pad_materials


@dataclass
class MeshData:
    verts: np.ndarray    # [V, 3] float32
    normals: np.ndarray  # [V, 3] float32
    tris: np.ndarray     # [T, 3] uint32 vertex indices
    normals_from_file: bool
    n_faces: int
    bounds: np.ndarray   # [6] min xyz, max xyz

    @property
    def n_tris(self) -> int:
        return int(self.tris.shape[0])


def _take(lib, h: c_void_p) -> MeshData:
    try:
        info = L.MeshInfo()
        L.check(lib.eos_mesh_get_info(h, byref(info)), "eos_mesh_get_info")
        v = np.empty((info.n_verts, 3), np.float32)
        n = np.empty((info.n_verts, 3), np.float32)
        t = np.empty((info.n_tris, 3), np.uint32)
        L.check(lib.eos_mesh_get_data(h, v.ctypes.data_as(c_void_p), n.ctypes.data_as(c_void_p),
                                      t.ctypes.data_as(c_void_p)), "eos_mesh_get_data")
        return MeshData(v, n, t, bool(info.normals_from_file), int(info.n_faces),
                        np.array(list(info.bounds), np.float32))
    finally:
        lib.eos_mesh_destroy(h)


def load_obj(path: str) -> MeshData:
    lib = L.load()
    h = c_void_p()
    L.check(lib.eos_mesh_load_obj(str(path).encode(), byref(h)), f"eos_mesh_load_obj({path})")
    return _take(lib, h)


def parse_obj(text: str | bytes) -> MeshData:
    lib = L.load()
    data = text.encode() if isinstance(text, str) else bytes(text)
    h = c_void_p()
    L.check(lib.eos_mesh_parse_obj(data, len(data), byref(h)), "eos_mesh_parse_obj")
    return _take(lib, h)


def transform(mesh: MeshData, M: np.ndarray) -> MeshData:
    """Applies a 4x4 affine transform (column vectors) to positions and M^-T to normals,
    renormalised -- what createCudaScene does with a per-object transformation."""
    M = np.asarray(M, np.float64)
    v = mesh.verts.astype(np.float64) @ M[:3, :3].T + M[:3, 3]
    nt = np.linalg.inv(M[:3, :3]).T
    n = mesh.normals.astype(np.float64) @ nt.T
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    return MeshData(v.astype(np.float32), n.astype(np.float32), mesh.tris.copy(), mesh.normals_from_file,
                    mesh.n_faces, np.concatenate([v.min(0), v.max(0)]).astype(np.float32))


def scene_from_meshes(meshes: list[MeshData], materials, lights, name: str = "meshes") -> SceneData:
    """One scene from several meshes; mesh k uses material row k (object id k)."""
    verts, normals, tris, obj = [], [], [], []
    base = 0
    for k, m in enumerate(meshes):
        verts.append(m.verts)
        normals.append(m.normals)
        tris.append(m.tris.astype(np.int64) + base)
        obj.append(np.full(m.n_tris, k, np.uint32))
        base += m.verts.shape[0]
    mats = pad_materials(materials)
    if mats.shape[0] < len(meshes):
        raise ValueError("one material row per mesh")
    return SceneData(np.concatenate(verts), np.concatenate(normals), np.concatenate(tris).astype(np.uint32),
                     np.concatenate(obj), mats, np.asarray(lights, np.float32).reshape(-1, LIGHT_STRIDE), name)
