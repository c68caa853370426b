"""CPU checkers for the render path -- TEST INFRASTRUCTURE.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
import this package.  The product (``eos_b200``) never does: it fails loudly when its
CUDA library is missing instead of falling back here.

Two checkers live here:

* :class:`Oracle` -- ``liboracle.so``, our C restatement of the reference render path
  (``eos_oracle.c``; every function cites the reference lines it follows), with
  tree-independent nearest-hit semantics, near-tie flags and an FP64 frozen-visibility
  forward + adjoint.
* :class:`RefRenderer` -- ``_ref/libeosref.so``, the reference's own CPU renderer
  (src/RayTracer.cpp, src/Scene.cpp, src/BVH.cpp, ...) compiled from its sources by
  ``oracle/Makefile`` with the two one-line fixes documented there (the shadow ray's
  uninitialised distance, the leaf index overrun).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys
from ctypes import POINTER, c_double, c_float, c_int, c_int32, c_longlong, c_uint32, c_uint8, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# EOS_ORACLE_LIB: another build of eos_oracle.c (the sanitizer test loads one built with
# AddressSanitizer and UBSan)
ORACLE_SO = os.environ.get("EOS_ORACLE_LIB") or os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libeosref.so")
# the reference's source tree, present where the checkers are built (not on the GPU box)
REF_ROOT = os.environ.get("EOS_REFERENCE_ROOT", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "src")
MAXB = 8
HIT_NONE = -1
HIT_UNTRACED = -2
FLAG_TIE, FLAG_NEAR_ORIGIN, FLAG_OUT_OF_RANGE, FLAG_AXIS_PARALLEL = 1, 2, 4, 8


def build(ref: bool = True) -> None:
    """Compile the restatement and, when the reference tree is present, the reference."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    if ref and os.path.isdir(REF_SRC):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_SRC}"], check=True)


def grid_side(spp: int) -> int:
    """n for spp = n * n samples on the reference's anti-aliasing grid."""
    n = int(round(spp ** 0.5))
    if n * n != spp:
        raise ValueError("the anti-aliasing grid needs a square number of samples")
    return n


def tree_nodes(trace_depth: int) -> int:
    """Nodes of a tree record: 2^(trace_depth + 1) - 1 (heap order)."""
    return (1 << (trace_depth + 1)) - 1


def build_reference_gpu() -> None:
    """The reference's GPU megakernel for sm_100a (oracle/_ref/libeosref_gpu.so, a comparison
    point run by oracle/ref_gpu.py) and the cached config-1 tree it renders with."""
    if not os.path.isdir(REF_SRC):
        return
    subprocess.run(["make", "-s", "-C", HERE, "refgpu", f"REF={REF_SRC}"], check=True)
    subprocess.run([sys.executable, "-m", "oracle.make_ref_tree", "--scene", "config1"], cwd=os.path.dirname(HERE),
                   check=True, capture_output=True)


def _p(a, ct):
    return a.ctypes.data_as(POINTER(ct)) if a is not None else None


_lib_oracle = None
_lib_ref = None


def lib_oracle():
    global _lib_oracle
    if _lib_oracle is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        L = ctypes.CDLL(ORACLE_SO)
        L.oracle_scene_create.restype = c_void_p
        L.oracle_scene_create.argtypes = [POINTER(c_float), POINTER(c_float), c_int, POINTER(c_uint32),
                                          POINTER(c_uint32), c_int, POINTER(c_float), c_int,
                                          POINTER(c_float), c_int]
        L.oracle_scene_destroy.argtypes = [c_void_p]
        L.oracle_scene_set_ambient.argtypes = [c_void_p, c_float]
        L.oracle_instanced_create.restype = c_void_p
        L.oracle_instanced_create.argtypes = [POINTER(c_void_p), POINTER(c_int32), POINTER(c_float), POINTER(c_int32),
                                              c_int, POINTER(c_float), c_int, POINTER(c_float), c_int]
        L.oracle_render.argtypes = [c_void_p, POINTER(c_float), c_int, c_int, c_float, c_int, c_int,
                                    c_uint32, POINTER(c_int32), c_int, c_int, POINTER(c_float),
                                    POINTER(c_int32), POINTER(c_uint32), POINTER(c_uint32),
                                    POINTER(c_longlong), c_int]
        L.oracle_closest.argtypes = [c_void_p, POINTER(c_float), c_int, POINTER(c_int32), POINTER(c_float),
                                     POINTER(c_uint8)]
        L.oracle_any.argtypes = [c_void_p, POINTER(c_float), c_int, POINTER(c_uint8)]
        L.oracle_closest_brute.argtypes = [c_void_p, POINTER(c_float), c_int, POINTER(c_int32),
                                           POINTER(c_float)]
        L.oracle_morton.argtypes = [POINTER(c_float), POINTER(c_uint32), c_int, POINTER(c_uint32),
                                    POINTER(c_int32)]
        L.oracle_frozen_f64.argtypes = [c_void_p, POINTER(c_float), c_int, c_int, c_int, c_float, c_int, c_uint32,
                                        c_int, POINTER(c_int32), POINTER(c_uint32), POINTER(c_double),
                                        POINTER(c_double), POINTER(c_double), POINTER(c_double),
                                        POINTER(c_double), POINTER(c_double), c_int, c_int, c_int]
        L.oracle_render_tree.restype = c_int
        L.oracle_render_tree.argtypes = L.oracle_render.argtypes
        _lib_oracle = L
    return _lib_oracle


def lib_ref():
    global _lib_ref
    if _lib_ref is None:
        if not os.path.exists(REF_SO):
            build(ref=True)
        if not os.path.exists(REF_SO):
            raise RuntimeError("reference CPU build unavailable (oracle/_ref/libeosref.so missing)")
        L = ctypes.CDLL(REF_SO)
        L.eosref_scene_create.restype = c_void_p
        L.eosref_scene_create.argtypes = [POINTER(c_float), POINTER(c_float), c_int, POINTER(c_uint32),
                                          POINTER(c_uint32), c_int, POINTER(c_float), c_int,
                                          POINTER(c_float), c_int, c_int, POINTER(c_double)]
        L.eosref_scene_create_transformed.restype = c_void_p
        L.eosref_scene_create_transformed.argtypes = [POINTER(c_float), POINTER(c_float), POINTER(c_uint32),
                                                      POINTER(c_uint32), c_int, POINTER(c_float), c_int,
                                                      POINTER(c_float), c_int, POINTER(c_int32), POINTER(c_float),
                                                      c_int, c_int]
        L.eosref_scene_destroy.argtypes = [c_void_p]
        L.eosref_scene_set_ambient.argtypes = [c_void_p, c_float]
        L.eosref_scene_stats.argtypes = [c_void_p, POINTER(c_int), POINTER(c_int)]
        L.eosref_render.restype = c_int
        L.eosref_render.argtypes = [c_void_p, POINTER(c_float), c_int, c_int, c_float, c_int, c_int,
                                    POINTER(c_int32), c_int, POINTER(c_float), POINTER(c_int32),
                                    POINTER(c_uint32), POINTER(c_longlong), POINTER(c_double)]
        L.eosref_render_rgba8.argtypes = [c_void_p, POINTER(c_float), c_int, c_int, c_int, c_int,
                                          POINTER(c_uint8), POINTER(c_double), c_int]
        L.eosref_render_aa.restype = c_int
        L.eosref_render_aa.argtypes = [c_void_p, POINTER(c_float), c_int, c_int, c_int, c_int, c_int,
                                       POINTER(c_int32), c_int, POINTER(c_float), POINTER(c_int32),
                                       POINTER(c_uint32), POINTER(c_longlong)]
        L.eosref_closest_hit.argtypes = [c_void_p, POINTER(c_float), c_int, POINTER(c_int32), POINTER(c_float)]
        L.eosref_any_hit.argtypes = [c_void_p, POINTER(c_float), c_int, POINTER(c_uint8)]
        L.eosref_morton3.argtypes = [POINTER(c_uint32), c_int, POINTER(c_uint32)]
        L.eosref_render_tree.restype = c_int
        L.eosref_render_tree.argtypes = [c_void_p, POINTER(c_float), c_int, c_int, c_float, c_int, c_int,
                                         POINTER(c_int32), c_int, POINTER(c_float), POINTER(c_int32),
                                         POINTER(c_uint32), POINTER(c_longlong)]
        L.eosref_tree_export.argtypes = [c_void_p, POINTER(c_int32), POINTER(c_int32)]
        L.eosref_tree_boxes.argtypes = [c_void_p, POINTER(c_float)]
        L.eosref_scene_create_from_tree.restype = c_void_p
        L.eosref_scene_create_from_tree.argtypes = [POINTER(c_float), POINTER(c_float), c_int, POINTER(c_uint32),
                                                    POINTER(c_uint32), c_int, POINTER(c_float), c_int,
                                                    POINTER(c_float), c_int, POINTER(c_int32), POINTER(c_int32),
                                                    c_int]
        _lib_ref = L
    return _lib_ref


def ref_available() -> bool:
    try:
        lib_ref()
        return True
    except (RuntimeError, OSError, subprocess.CalledProcessError):
        return False


def _scene_args(sc):
    return (_p(sc.verts, c_float), _p(sc.normals, c_float), int(sc.verts.shape[0]), _p(sc.tris, c_uint32),
            _p(sc.tri_obj, c_uint32), sc.n_tris, _p(sc.materials, c_float), sc.n_objects,
            _p(sc.lights, c_float), sc.n_lights)


def _pix(pixels):
    if pixels is None:
        return None, 0
    px = np.ascontiguousarray(pixels, dtype=np.int32)
    return px, int(px.size)


def _rays(rays):
    return np.ascontiguousarray(rays, dtype=np.float32).reshape(-1, 6)


def morton(verts: np.ndarray, tris: np.ndarray):
    """30-bit Morton codes of triangle centroids and the stable (code, id) sorted order."""
    L = lib_oracle()
    v = np.ascontiguousarray(verts, np.float32)
    t = np.ascontiguousarray(tris, np.uint32)
    n = t.shape[0]
    codes = np.zeros(n, np.uint32)
    order = np.zeros(n, np.int32)
    L.oracle_morton(_p(v, c_float), _p(t, c_uint32), n, _p(codes, c_uint32), _p(order, c_int32))
    return codes, order


class Oracle:
    """The C restatement, over one scene."""

    def __init__(self, scene):
        self.scene = scene
        self._keep = scene
        self.h = lib_oracle().oracle_scene_create(*_scene_args(scene))
        lib_oracle().oracle_scene_set_ambient(self.h, float(getattr(scene, "ambient_index", 1.0)))

    def __del__(self):
        if getattr(self, "h", None) and _lib_oracle is not None:
            _lib_oracle.oracle_scene_destroy(self.h)
            self.h = None

    def render(self, cam, trace_depth: int, pixel_offset: float = 0.5, spp: int = 1, jitter_seed: int = 0,
               pixels=None, nthreads: int | None = None, aa_grid: bool = False):
        """aa_grid: the reference's n x n anti-aliasing grid (spp = n * n), else hashed jitter."""
        L = lib_oracle()
        px, npix = _pix(pixels)
        n = npix if px is not None else cam.width * cam.height
        rgb = np.zeros((n, 3), np.float32)
        hits = np.zeros((n * spp, MAXB), np.int32)
        shadows = np.zeros((n * spp, MAXB), np.uint32)
        flags = np.zeros(n * spp, np.uint32)
        counts = np.zeros(3, np.int64)
        c12 = cam.as_array()
        L.oracle_render(self.h, _p(c12, c_float), cam.width, cam.height, pixel_offset, trace_depth, spp,
                        jitter_seed, _p(px, c_int32), npix, nthreads or os.cpu_count(), _p(rgb, c_float),
                        _p(hits, c_int32), _p(shadows, c_uint32), _p(flags, c_uint32), _p(counts, c_longlong),
                        grid_side(spp) if aa_grid else 0)
        return dict(rgb=rgb, hits=hits, shadows=shadows, flags=flags, counts=counts)

    def render_tree(self, cam, trace_depth: int, pixel_offset: float = 0.5, spp: int = 1, jitter_seed: int = 0,
                    pixels=None, nthreads: int | None = None, aa_grid: bool = False):
        """As render, with ray trees (materials both reflective and transparent trace both
        secondary rays): hits / shadows [n*spp, 2^(trace_depth+1) - 1] in heap order (node j's
        mirror child 2j + 1, transparent child 2j + 2)."""
        L = lib_oracle()
        px, npix = _pix(pixels)
        n = npix if px is not None else cam.width * cam.height
        nn = tree_nodes(trace_depth)
        rgb = np.zeros((n, 3), np.float32)
        hits = np.zeros((n * spp, nn), np.int32)
        shadows = np.zeros((n * spp, nn), np.uint32)
        flags = np.zeros(n * spp, np.uint32)
        counts = np.zeros(3, np.int64)
        c12 = cam.as_array()
        L.oracle_render_tree(self.h, _p(c12, c_float), cam.width, cam.height, pixel_offset, trace_depth, spp,
                             jitter_seed, _p(px, c_int32), npix, nthreads or os.cpu_count(), _p(rgb, c_float),
                             _p(hits, c_int32), _p(shadows, c_uint32), _p(flags, c_uint32), _p(counts, c_longlong),
                             grid_side(spp) if aa_grid else 0)
        return dict(rgb=rgb, hits=hits, shadows=shadows, flags=flags, counts=counts)

    def closest(self, rays):
        r = _rays(rays)
        n = r.shape[0]
        ids = np.zeros(n, np.int32)
        ts = np.zeros(n, np.float32)
        tie = np.zeros(n, np.uint8)
        lib_oracle().oracle_closest(self.h, _p(r, c_float), n, _p(ids, c_int32), _p(ts, c_float), _p(tie, c_uint8))
        return ids, ts, tie

    def closest_brute(self, rays):
        r = _rays(rays)
        n = r.shape[0]
        ids = np.zeros(n, np.int32)
        ts = np.zeros(n, np.float32)
        lib_oracle().oracle_closest_brute(self.h, _p(r, c_float), n, _p(ids, c_int32), _p(ts, c_float))
        return ids, ts

    def any(self, rays):
        r = _rays(rays)
        occ = np.zeros(r.shape[0], np.uint8)
        lib_oracle().oracle_any(self.h, _p(r, c_float), r.shape[0], _p(occ, c_uint8))
        return occ

    def frozen_f64(self, cams, width, height, pixel_offset, trace_depth, hits, shadows, mat_params,
                   light_params, g=None, nthreads=None, spp=1, jitter_seed=0, tree=False, aa_grid=False):
        """FP64 re-render with frozen visibility; with g, also the adjoint of <g, rgb>.

        hits / shadows: per path, V*H*W*spp of them (samples of a pixel consecutive, the
        forward's order); the colour of a pixel is the mean of its samples, whose offsets
        come from jitter_seed as in the forward pass.  Chain records (8 bounces per path)
        or, with tree=True, tree records (2^(trace_depth+1) - 1 heap-order nodes).
        mat_params: [K, 10] kd rgb, ks rgb, log shininess, reflectivity, transparency, refractive
        index (float64; rows of 8 are opaque)
        light_params: [L, 6] position xyz, colour rgb (float64)
        Returns rgb [V*H*W, 3] and, with g [V*H*W, 3], (grad_mat [K, 7], grad_light [L, 6]).
        """
        L = lib_oracle()
        cams_a = np.ascontiguousarray(np.stack([c.as_array() for c in cams]), np.float32)
        nv = len(cams)
        npx = nv * width * height
        slots = tree_nodes(trace_depth) if tree else MAXB
        h = np.ascontiguousarray(hits, np.int32).reshape(npx * spp, slots)
        s = np.ascontiguousarray(shadows, np.uint32).reshape(npx * spp, slots)
        mp = np.asarray(mat_params, np.float64)
        if mp.shape[1] == 8:  # no transparency columns: opaque, index 1
            mp = np.concatenate([mp, np.zeros((mp.shape[0], 1)), np.ones((mp.shape[0], 1))], 1)
        mp = np.ascontiguousarray(mp)
        lp = np.ascontiguousarray(light_params, np.float64)
        rgb = np.zeros((npx, 3), np.float64)
        gm = np.zeros((mp.shape[0], 7), np.float64)
        gl = np.zeros((lp.shape[0], 6), np.float64)
        ga = None if g is None else np.ascontiguousarray(g, np.float64).reshape(npx, 3)
        L.oracle_frozen_f64(self.h, _p(cams_a, c_float), nv, width, height, pixel_offset, int(spp),
                            int(jitter_seed) & 0xFFFFFFFF, trace_depth,
                            _p(h, c_int32), _p(s, c_uint32), _p(mp, c_double), _p(lp, c_double),
                            _p(rgb, c_double), _p(ga, c_double), _p(gm, c_double), _p(gl, c_double),
                            nthreads or os.cpu_count(), 1 if tree else 0, grid_side(spp) if aa_grid else 0)
        if g is None:
            return rgb
        return rgb, gm, gl


class OracleInstanced(Oracle):
    """The C restatement over a two-level scene (scenes.InstancedData): every instance's
    mesh is tested with the ray in its object space (no instance tree)."""

    def __init__(self, idata):
        L = lib_oracle()
        self.scene = idata
        self.meshes = [Oracle(m) for m in idata.meshes]
        n = len(idata.instances)
        handles = (c_void_p * len(self.meshes))(*[m.h for m in self.meshes])
        mesh_of = np.array([m for m, _, _ in idata.instances], np.int32)
        tr = np.ascontiguousarray(np.stack([np.asarray(M, np.float64).reshape(3, 4) for _, M, _ in idata.instances]),
                                  np.float32)
        base = np.array([b for _, _, b in idata.instances], np.int32)
        self._keep = (mesh_of, tr, base, idata)
        self.h = L.oracle_instanced_create(handles, _p(mesh_of, c_int32), _p(tr, c_float), _p(base, c_int32), n,
                                           _p(idata.materials, c_float), idata.materials.shape[0],
                                           _p(idata.lights, c_float), idata.lights.shape[0])
        L.oracle_scene_set_ambient(self.h, float(idata.ambient_index))


class RefRenderer:
    """The reference's own CPU renderer, compiled from its sources, over one scene.

    tree: (perm, nodes) from :meth:`export_tree` of an earlier build of the same scene;
    the tree is then restored instead of built (see :func:`ref_tree_cached`).
    transforms: (tri_xf [n_tris] int32, xforms [K, 12] row-major 3x4) for a scene of
    object-space triangles, each placed by one transformation (eosref_scene_create_transformed;
    the reference's builder bounds the placed triangles, its CPU renderer ignores them)."""

    def __init__(self, scene, build_threads: int = 1, tree=None, transforms=None):
        L = lib_ref()
        self.scene = scene
        secs = c_double(0.0)
        if transforms is not None:
            tri_xf = np.ascontiguousarray(transforms[0], np.int32)
            xf = np.ascontiguousarray(transforms[1], np.float32).reshape(-1, 12)
            a = _scene_args(scene)
            self.h = L.eosref_scene_create_transformed(a[0], a[1], a[3], a[4], a[5], a[6], a[7], a[8], a[9],
                                                       _p(tri_xf, c_int32), _p(xf, c_float), xf.shape[0],
                                                       build_threads)
            if not self.h:
                raise ValueError("transformation index out of range")
        elif tree is None:
            self.h = L.eosref_scene_create(*_scene_args(scene), build_threads, ctypes.byref(secs))
        else:
            perm = np.ascontiguousarray(tree[0], np.int32)
            nodes = np.ascontiguousarray(tree[1], np.int32).reshape(-1, 6)
            if perm.shape[0] != scene.n_tris:
                raise ValueError("tree was built for another scene")
            self.h = L.eosref_scene_create_from_tree(*_scene_args(scene), _p(perm, c_int32), _p(nodes, c_int32),
                                                     nodes.shape[0])
            if not self.h:
                raise ValueError("tree arrays do not describe a tree over this scene")
        L.eosref_scene_set_ambient(self.h, float(getattr(scene, "ambient_index", 1.0)))
        self.build_seconds = secs.value
        nn, ml = c_int(0), c_int(0)
        L.eosref_scene_stats(self.h, ctypes.byref(nn), ctypes.byref(ml))
        self.n_nodes, self.max_leaf = nn.value, ml.value

    def export_tree(self):
        """(perm [n_tris], nodes [n_nodes, 6]) of the reference's tree (eosref_tree_export)."""
        perm = np.zeros(self.scene.n_tris, np.int32)
        nodes = np.zeros((self.n_nodes, 6), np.int32)
        lib_ref().eosref_tree_export(self.h, _p(perm, c_int32), _p(nodes, c_int32))
        return perm, nodes

    def boxes(self):
        """[n_nodes, 6] boxes of the reference's flat node buffer."""
        b = np.zeros((self.n_nodes, 6), np.float32)
        lib_ref().eosref_tree_boxes(self.h, _p(b, c_float))
        return b

    def __del__(self):
        if getattr(self, "h", None) and _lib_ref is not None:
            _lib_ref.eosref_scene_destroy(self.h)
            self.h = None

    def render(self, cam, trace_depth: int, pixel_offset: float = 0.0, pixels=None, nthreads=None,
               paths: bool = True):
        L = lib_ref()
        px, npix = _pix(pixels)
        n = npix if px is not None else cam.width * cam.height
        rgb = np.zeros((n, 3), np.float32)
        hits = np.zeros((n, MAXB), np.int32) if paths else None
        shadows = np.zeros((n, MAXB), np.uint32) if paths else None
        counts = np.zeros(3, np.int64)
        secs = c_double(0.0)
        c12 = cam.as_array()
        rc = L.eosref_render(self.h, _p(c12, c_float), cam.width, cam.height, pixel_offset, trace_depth,
                             nthreads or os.cpu_count(), _p(px, c_int32), npix, _p(rgb, c_float),
                             _p(hits, c_int32), _p(shadows, c_uint32), _p(counts, c_longlong), ctypes.byref(secs))
        if rc != 0:
            raise ValueError("reference renderer rejected trace_depth (it cannot be set below 1)")
        return dict(rgb=rgb, hits=hits, shadows=shadows, counts=counts, seconds=secs.value)

    def render_tree(self, cam, trace_depth: int, pixel_offset: float = 0.0, pixels=None, nthreads=None):
        """FP32 colours and ray-tree records (heap order, tree_nodes(trace_depth) per path)."""
        L = lib_ref()
        px, npix = _pix(pixels)
        n = npix if px is not None else cam.width * cam.height
        nn = tree_nodes(trace_depth)
        rgb = np.zeros((n, 3), np.float32)
        hits = np.zeros((n, nn), np.int32)
        shadows = np.zeros((n, nn), np.uint32)
        counts = np.zeros(3, np.int64)
        c12 = cam.as_array()
        rc = L.eosref_render_tree(self.h, _p(c12, c_float), cam.width, cam.height, pixel_offset, trace_depth,
                                  nthreads or os.cpu_count(), _p(px, c_int32), npix, _p(rgb, c_float),
                                  _p(hits, c_int32), _p(shadows, c_uint32), _p(counts, c_longlong))
        if rc != 0:
            raise ValueError("reference renderer rejected trace_depth")
        return dict(rgb=rgb, hits=hits, shadows=shadows, counts=counts)

    def render_rgba8(self, cam, trace_depth: int, nthreads=None, aa: int = 0):
        """RayTracer::render into RGBA8; aa > 0 = setAASamples(aa) (its anti-aliasing grid)."""
        L = lib_ref()
        out = np.zeros((cam.height, cam.width, 4), np.uint8)
        secs = c_double(0.0)
        c12 = cam.as_array()
        L.eosref_render_rgba8(self.h, _p(c12, c_float), cam.width, cam.height, trace_depth,
                              nthreads or os.cpu_count(), _p(out, c_uint8), ctypes.byref(secs), int(aa))
        return out, secs.value

    def render_aa(self, cam, trace_depth: int, aa: int, pixels=None, nthreads=None):
        """FP32 colours and per-sample paths on the reference's aa x aa grid."""
        L = lib_ref()
        px, npix = _pix(pixels)
        n = npix if px is not None else cam.width * cam.height
        rgb = np.zeros((n, 3), np.float32)
        hits = np.zeros((n * aa * aa, MAXB), np.int32)
        shadows = np.zeros((n * aa * aa, MAXB), np.uint32)
        counts = np.zeros(3, np.int64)
        c12 = cam.as_array()
        rc = L.eosref_render_aa(self.h, _p(c12, c_float), cam.width, cam.height, trace_depth, int(aa),
                                nthreads or os.cpu_count(), _p(px, c_int32), npix, _p(rgb, c_float),
                                _p(hits, c_int32), _p(shadows, c_uint32), _p(counts, c_longlong))
        if rc != 0:
            raise ValueError("reference renderer rejected trace_depth or aa")
        return dict(rgb=rgb, hits=hits, shadows=shadows, counts=counts)

    def closest(self, rays):
        r = _rays(rays)
        ids = np.zeros(r.shape[0], np.int32)
        pts = np.zeros((r.shape[0], 3), np.float32)
        lib_ref().eosref_closest_hit(self.h, _p(r, c_float), r.shape[0], _p(ids, c_int32), _p(pts, c_float))
        return ids, pts

    def any(self, rays):
        r = _rays(rays)
        occ = np.zeros(r.shape[0], np.uint8)
        lib_ref().eosref_any_hit(self.h, _p(r, c_float), r.shape[0], _p(occ, c_uint8))
        return occ


def ref_morton3(xyz: np.ndarray) -> np.ndarray:
    """The reference's EncodeMorton3 (src/morton.h:45-48), compiled, on [n, 3] uint32."""
    a = np.ascontiguousarray(xyz, np.uint32).reshape(-1, 3)
    out = np.zeros(a.shape[0], np.uint32)
    lib_ref().eosref_morton3(_p(a, c_uint32), a.shape[0], _p(out, c_uint32))
    return out
