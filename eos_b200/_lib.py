"""ctypes binding of the C ABI in include/eos_c.h (libeos_b200.so, built in-tree).

There is no fallback: if the CUDA library is missing or fails to load, every entry
point raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_float, c_int32, c_size_t, c_uint32, c_uint64,
                    c_void_p)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libeos_b200.so")

MAX_BOUNCES = 8
MAX_LIGHTS = 32
HIT_NONE = -1
HIT_UNTRACED = -2
MODE_PLAIN = 0
MODE_WAVEFRONT = 1

STATUS = {0: "ok", 1: "invalid argument", 2: "out of device memory", 3: "CUDA error",
          4: "device loop ran out of iterations", 5: "traversal stack overflow",
          6: "ray queue overflow", 7: "unsupported", 8: "no CUDA device", 9: "file could not be read or written",
          10: "malformed input file"}


class EosError(RuntimeError):
    def __init__(self, code: int, where: str):
        super().__init__(f"{where}: {STATUS.get(code, 'unknown')} (status {code})")
        self.code = code


class Material(Structure):
    _fields_ = [("kd", c_float * 3), ("ks", c_float * 3), ("shininess", c_float), ("reflectivity", c_float),
                ("transparency", c_float), ("refractive_index", c_float)]


class Light(Structure):
    _fields_ = [("position", c_float * 3), ("color", c_float * 3)]


class Camera(Structure):
    _fields_ = [("position", c_float * 3), ("view", c_float * 3), ("right", c_float * 3), ("up", c_float * 3),
                ("width", c_int32), ("height", c_int32)]


class RenderParams(Structure):
    _fields_ = [("trace_depth", c_int32), ("pixel_offset", c_float), ("spp", c_int32), ("jitter_seed", c_uint32),
                ("mode", c_int32), ("block_size", c_int32), ("queue_chunk", c_int32), ("stack_depth", c_int32),
                ("flags", c_int32), ("row_begin", c_int32), ("row_end", c_int32)]


FLAG_STAGE_TIMING = 1
FLAG_TREE_RECORDS = 2
FLAG_AA_GRID = 4
FLAG_ASYNC = 8


class Tuning(Structure):
    _fields_ = [("block_size", c_int32), ("queue_chunk", c_int32), ("stack_depth", c_int32), ("leaf_size", c_int32),
                ("layout", c_int32), ("width", c_int32), ("builder", c_int32)]


LAYOUT_DEFAULT, LAYOUT_SAH, LAYOUT_FIXED = 0, 1, 2
BUILDER_DEFAULT, BUILDER_LBVH, BUILDER_PLOC = 0, 1, 2


class BuildParams(Structure):
    _fields_ = [("leaf_size", c_int32), ("layout", c_int32), ("width", c_int32), ("builder", c_int32)]


class PathRecord(Structure):
    _fields_ = [("hit", c_int32 * MAX_BOUNCES), ("shadow", c_uint32 * MAX_BOUNCES)]


class Stats(Structure):
    _fields_ = [("primary_rays", c_uint64), ("shadow_rays", c_uint64), ("secondary_rays", c_uint64),
                ("nodes_closest", c_uint64), ("tests_closest", c_uint64), ("nodes_shadow", c_uint64),
                ("tests_shadow", c_uint64), ("shaded_hits", c_uint64), ("gpu_ms", c_float), ("error_flags", c_int32),
                ("kernel_launches", c_uint32), ("stage_ms", c_float * 3)]


class MeshInfo(Structure):
    _fields_ = [("n_verts", c_uint32), ("n_tris", c_uint32), ("normals_from_file", c_uint32), ("n_faces", c_uint32),
                ("bounds", c_float * 6)]


class SceneInfo(Structure):
    _fields_ = [("n_tris", c_uint32), ("n_nodes", c_uint32), ("leaf_size", c_uint32), ("layout", c_uint32),
                ("width", c_uint32), ("sah_cost", c_float), ("n_objects", c_uint32), ("n_lights", c_uint32),
                ("build_ms", c_float), ("device_bytes", c_uint64), ("builder", c_uint32), ("depth", c_uint32)]


class Job(Structure):
    _fields_ = [("scene", c_void_p), ("camera", Camera), ("trace_depth", c_int32), ("pixel_offset", c_float),
                ("spp", c_int32), ("jitter_seed", c_uint32), ("rgb_out", c_void_p), ("rgba8_out", c_void_p),
                ("paths_out", c_void_p), ("row_begin", c_int32), ("row_end", c_int32)]


class Instance(Structure):
    _fields_ = [("mesh", c_void_p), ("transform", c_float * 12), ("material_base", c_uint32)]


class Limits(Structure):
    _fields_ = [("queue_entries", c_int32), ("work_budget", c_int32), ("small_stack", c_int32)]


class Grads(Structure):
    _fields_ = [("materials", c_void_p), ("lights", c_void_p)]


# every symbol declared in include/eos_c.h: (name, restype, argtypes)
SIGNATURES = [
    ("eos_abi_version", c_int32, []),
    ("eos_status_string", c_char_p, [c_int32]),
    ("eos_last_error_detail", c_char_p, []),
    ("eos_device_count", c_int32, [POINTER(c_int32)]),
    ("eos_ctx_create", c_int32, [c_int32, POINTER(c_void_p)]),
    ("eos_ctx_destroy", c_int32, [c_void_p]),
    ("eos_ctx_set_stream", c_int32, [c_void_p, c_void_p]),
    ("eos_ctx_synchronize", c_int32, [c_void_p]),
    ("eos_ctx_set_tuning", c_int32, [c_void_p, c_uint32, POINTER(Tuning)]),
    ("eos_ctx_clear_tuning", c_int32, [c_void_p]),
    ("eos_ctx_set_limits", c_int32, [c_void_p, POINTER(Limits)]),
    ("eos_scene_create", c_int32, [c_void_p, c_void_p, c_void_p, c_uint32, c_void_p, c_void_p, c_uint32,
                                   c_void_p, c_uint32, c_void_p, c_uint32, POINTER(BuildParams), POINTER(c_void_p)]),
    ("eos_scene_destroy", c_int32, [c_void_p]),
    ("eos_scene_set_materials", c_int32, [c_void_p, c_void_p, c_uint32]),
    ("eos_scene_set_lights", c_int32, [c_void_p, c_void_p, c_uint32]),
    ("eos_scene_set_ambient_index", c_int32, [c_void_p, c_float]),
    ("eos_scene_get_info", c_int32, [c_void_p, POINTER(SceneInfo)]),
    ("eos_scene_get_morton", c_int32, [c_void_p, c_void_p, c_void_p]),
    ("eos_render", c_int32, [c_void_p, c_void_p, POINTER(Camera), POINTER(RenderParams), c_void_p, c_void_p,
                             c_void_p, c_void_p, POINTER(Stats)]),
    ("eos_render_batch", c_int32, [c_void_p, POINTER(Job), c_uint32, POINTER(RenderParams), POINTER(Stats)]),
    ("eos_render_backward", c_int32, [c_void_p, c_void_p, POINTER(Camera), c_uint32, POINTER(RenderParams),
                                      c_void_p, c_void_p, POINTER(Grads)]),
    ("eos_trace_closest", c_int32, [c_void_p, c_void_p, c_void_p, c_uint32, c_void_p, c_void_p]),
    ("eos_trace_any", c_int32, [c_void_p, c_void_p, c_void_p, c_uint32, c_void_p]),
    ("eos_render_noalloc", c_int32, [c_void_p, POINTER(Camera), POINTER(RenderParams), c_void_p, c_void_p,
                                     c_void_p, POINTER(Stats)]),
    ("eos_scene_create_instanced", c_int32, [c_void_p, c_void_p, c_uint32, c_void_p, c_uint32, c_void_p, c_uint32,
                                             POINTER(c_void_p)]),
    ("eos_scene_save", c_int32, [c_void_p, c_char_p]),
    ("eos_scene_load", c_int32, [c_void_p, c_char_p, POINTER(c_void_p)]),
    ("eos_mesh_load_obj", c_int32, [c_char_p, POINTER(c_void_p)]),
    ("eos_mesh_parse_obj", c_int32, [c_char_p, c_size_t, POINTER(c_void_p)]),
    ("eos_mesh_get_info", c_int32, [c_void_p, POINTER(MeshInfo)]),
    ("eos_mesh_get_data", c_int32, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("eos_mesh_destroy", c_int32, [c_void_p]),
]

NOALLOC_MAX_PATHS = 16384
NOALLOC_MAX_LIGHTS = 8

_lib = None


def load(path: str = LIB_PATH):
    """Load libeos_b200.so and bind every C ABI symbol; raises when the library is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"CUDA library not built: {path} (run `python -m eos_b200.build`)")
    L = ctypes.CDLL(path)
    for name, res, args in SIGNATURES:
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    if L.eos_abi_version() != 1:
        raise RuntimeError("ABI version mismatch")
    _lib = L
    return L


def check(code: int, where: str) -> None:
    if code != 0:
        detail = ""
        if code in (2, 3) and _lib is not None:
            detail = (_lib.eos_last_error_detail() or b"").decode()
        raise EosError(code, where + (f" [{detail}]" if detail else ""))
