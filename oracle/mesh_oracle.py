"""OBJ mesh ingestion restated in Python -- TEST INFRASTRUCTURE (checker only).

Restates the import that TriangleMesh::loadFromFile (src/triangleMesh.cpp:79-160) gets
from assimp 3 (libassimp.so.3; not present here, so parity with assimp itself is
unpinned) with aiImportFile(aiProcess_Triangulate | aiProcess_GenSmoothNormals |
aiProcess_JoinIdenticalVertices), step by step from assimp's published algorithm:

* ObjFileParser / ObjFileImporter::createVertexArray: 'v', 'vn' and 'f' statements,
  corners i, i/t, i//n, i/t/n and negative (relative) indices; one vertex per face corner.
* TriangulateProcess: a quad is fanned from its concave corner (angles to the diagonal
  summing above pi), larger polygons from corner 0.
* GenVertexNormalsProcess (default 175-degree limit = no limit): unit face normal
  normalize(cross(v2 - v1, v3 - v1)) on each corner, then per unclaimed corner i the
  group {j : |P_j - P_i|^2 < eps^2}, eps = 1e-4 |bbox diagonal|, gets the normalised sum
  of its members' face normals (summed in corner order); members claimed earlier are
  overwritten.
* JoinVerticesProcess: equal position and normal within 1e-5 -> one vertex, first
  occurrence order.

All arithmetic is float32, one rounding per operation in the order written; numbers are
read with the C library's strtof and angles use its acosf (both through ctypes), so the
results are comparable bit for bit with the library's C++ loader.  The neighbour search
is a uniform grid of cell eps (the library sorts by x): a different search for the same
set.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

_libc = ctypes.CDLL(None)
_libc.strtof.restype = ctypes.c_float
_libc.strtof.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p)]
_libm = ctypes.CDLL("libm.so.6")
_libm.acosf.restype = ctypes.c_float
_libm.acosf.argtypes = [ctypes.c_float]

f32 = np.float32


def _strtof(tok: str) -> np.float32:
    return f32(_libc.strtof(tok.encode(), None))


def _sub(a, b):
    return (f32(a[0] - b[0]), f32(a[1] - b[1]), f32(a[2] - b[2]))


def _dot(a, b):
    return f32(f32(f32(a[0] * b[0]) + f32(a[1] * b[1])) + f32(a[2] * b[2]))


def _cross(a, b):
    return (f32(f32(a[1] * b[2]) - f32(a[2] * b[1])), f32(f32(a[2] * b[0]) - f32(a[0] * b[2])),
            f32(f32(a[0] * b[1]) - f32(a[1] * b[0])))


def _normalize_safe(v):
    ln = f32(np.sqrt(_dot(v, v)))
    if ln > 0:
        return (f32(v[0] / ln), f32(v[1] / ln), f32(v[2] / ln))
    return v


def _index(tok: str, n: int) -> int:
    i = int(tok)
    if i < 0:
        i = n + i + 1
    if i < 1 or i > n:
        raise ValueError("index out of range")
    return i - 1


def _quad_start(q) -> int:
    for i in range(4):
        v = q[i]
        left, diag, right = _sub(q[(i + 3) % 4], v), _sub(q[(i + 2) % 4], v), _sub(q[(i + 1) % 4], v)
        vs = []
        for w in (left, diag, right):
            ln = f32(np.sqrt(_dot(w, w)))
            with np.errstate(divide="ignore", invalid="ignore"):
                vs.append((f32(w[0] / ln), f32(w[1] / ln), f32(w[2] / ln)))
        left, diag, right = vs
        a = f32(f32(_libm.acosf(float(_dot(left, diag)))) + f32(_libm.acosf(float(_dot(right, diag)))))
        if a > f32(3.1415926538):
            return i
    return 0


def parse_obj(text: str):
    """Returns (verts [V,3] f32, normals [V,3] f32, tris [T,3] u32, normals_from_file, n_faces)."""
    pos, nrm, corners = [], [], []
    n_faces = 0
    all_normals = True
    for raw in text.split("\n"):
        line = raw.split("#", 1)[0].strip(" \t\r")
        if not line:
            continue
        parts = line.split()
        if parts[0] == "v":
            pos.append(tuple(_strtof(t) for t in parts[1:4]))
        elif parts[0] == "vn":
            nrm.append(tuple(_strtof(t) for t in parts[1:4]))
        elif parts[0] == "f":
            face = []
            for tok in parts[1:]:
                fields = tok.split("/")
                vi = _index(fields[0], len(pos))
                ni = _index(fields[2], len(nrm)) if len(fields) == 3 and fields[2] != "" else -1
                face.append((vi, ni))
            n_faces += 1
            if len(face) < 3:
                continue
            all_normals = all_normals and all(c[1] >= 0 for c in face)
            s = _quad_start([pos[c[0]] for c in face]) if len(face) == 4 else 0
            k = len(face)
            for t in range(1, k - 1):
                corners += [face[s], face[(s + t) % k], face[(s + t + 1) % k]]
    nc = len(corners)
    if nc == 0:
        raise ValueError("no triangles")
    cp = [pos[c[0]] for c in corners]
    P = np.array(cp, dtype=np.float32)
    lo, hi = P.min(axis=0), P.max(axis=0)
    if all_normals:
        cn = [nrm[c[1]] for c in corners]
    else:
        fn = []
        for t in range(nc // 3):
            n = _normalize_safe(_cross(_sub(cp[3 * t + 1], cp[3 * t]), _sub(cp[3 * t + 2], cp[3 * t])))
            fn += [n, n, n]
        d = _sub(tuple(hi), tuple(lo))
        eps = f32(f32(np.sqrt(_dot(d, d))) * f32(1e-4))
        eps2 = f32(eps * eps)
        cell = float(eps) * 1.001 if eps > 0 else 1.0  # a member is at most one cell away
        grid: dict = {}
        keys = []
        for j, p in enumerate(cp):
            key = (math.floor(float(p[0]) / cell), math.floor(float(p[1]) / cell), math.floor(float(p[2]) / cell))
            keys.append(key)
            grid.setdefault(key, []).append(j)
        cn = [None] * nc
        had = [False] * nc
        for i in range(nc):
            if had[i]:
                continue
            pi = cp[i]
            if eps2 == 0:
                group = [j for j in range(nc) if cp[j] == pi]
            else:
                kx, ky, kz = keys[i]
                group = []
                for dx in (-1, 0, 1):
                    for dy in (-1, 0, 1):
                        for dz in (-1, 0, 1):
                            for j in grid.get((kx + dx, ky + dy, kz + dz), ()):
                                dd = _sub(cp[j], pi)
                                if _dot(dd, dd) < eps2:
                                    group.append(j)
                group.sort()
            sx = sy = sz = f32(0)
            for j in group:
                sx, sy, sz = f32(sx + fn[j][0]), f32(sy + fn[j][1]), f32(sz + fn[j][2])
            s = _normalize_safe((sx, sy, sz))
            for j in group:
                cn[j] = s
                had[j] = True
    # join identical vertices
    uniq: dict = {}
    uv, un, tris = [], [], []
    thr = f32(f32(1e-5) * f32(1e-5))
    for c in range(nc):
        p = tuple(f32(0) if x == 0 else x for x in cp[c])
        key = tuple(float(x) for x in p)
        idx = -1
        for u in uniq.get(key, []):
            dd = _sub(un[u], cn[c])
            if _dot(dd, dd) <= thr:
                idx = u
                break
        if idx < 0:
            idx = len(uv)
            uv.append(cp[c])
            un.append(cn[c])
            uniq.setdefault(key, []).append(idx)
        tris.append(idx)
    return (np.array(uv, np.float32).reshape(-1, 3), np.array(un, np.float32).reshape(-1, 3),
            np.array(tris, np.uint32).reshape(-1, 3), int(all_normals), n_faces)
