"""ctypes mirror of include/aurora_b200.h (record layouts and function signatures).

The library is loaded from aurora_b200/lib/libaurora_b200.so (built in-tree by
``aurora_b200.build``). There is no fallback: if the shared object is missing
or does not export an entry point, loading raises AuroraError.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libaurora_b200.so")


class AuroraError(RuntimeError):
    """An aurora_b200 call returned a status other than AUR_OK."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


AUR_OK = 0
STATUS_NAMES = {0: "AUR_OK", 1: "AUR_ERR_INVALID_ARG", 2: "AUR_ERR_OOM", 3: "AUR_ERR_CUDA", 4: "AUR_ERR_TIMEOUT",
                5: "AUR_ERR_QUEUE_OVERFLOW", 6: "AUR_ERR_PARSE", 7: "AUR_ERR_IO", 8: "AUR_ERR_UNSUPPORTED"}

MAT_MATTE, MAT_KELEMEN, MAT_COOKTORRANCE, MAT_METAL, MAT_CONSTANT, MAT_GLASS = 0, 1, 2, 3, 4, 5
LIGHT_SQUARE, LIGHT_SPHERE, LIGHT_ENV = 0, 1, 2
NORMAL_NONE, NORMAL_TEXTURE, NORMAL_CONSTANT = 0, 1, 2
ERR_INVALID_ARG, ERR_OOM, ERR_CUDA, ERR_TIMEOUT, ERR_QUEUE_OVERFLOW, ERR_PARSE, ERR_IO, ERR_UNSUPPORTED = range(1, 9)
FILM_PFM, FILM_EXR_HALF, FILM_EXR_FLOAT = 0, 1, 2
RENDER_PLAIN, RENDER_WAVEFRONT = 0, 1

f3 = C.c_float * 3


class Ray(C.Structure):
    _fields_ = [("org", f3), ("mint", C.c_float), ("dir", f3), ("maxt", C.c_float)]


class Hit(C.Structure):
    _fields_ = [("t", C.c_float), ("u", C.c_float), ("v", C.c_float), ("prim", C.c_int32), ("attr", C.c_int32)]


class Isect(C.Structure):
    _fields_ = [("t", C.c_float), ("u", C.c_float), ("v", C.c_float), ("prim", C.c_int32), ("attr", C.c_int32),
                ("hitP", f3), ("hitN", f3), ("st", C.c_float * 2), ("bar", f3)]


class BvhOpts(C.Structure):
    _fields_ = [("max_leaf", C.c_int32), ("cost_traverse", C.c_float), ("cost_intersect", C.c_float),
                ("ploc_radius", C.c_int32)]


class MaterialDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("diffuse", f3), ("specular", f3), ("gain", f3), ("roughness", C.c_float),
                ("roughness_b", C.c_float), ("reflectance", C.c_float), ("mix", C.c_float),
                ("diffuse_tex", C.c_int32), ("specular_tex", C.c_int32), ("roughness_tex", C.c_int32),
                ("ior", C.c_float), ("normal_kind", C.c_int32), ("normal_tex", C.c_int32), ("normal", f3)]


class LightDesc(C.Structure):
    _fields_ = [("type", C.c_int32), ("object_to_camera", C.c_float * 16), ("size_x", C.c_float),
                ("size_y", C.c_float), ("center", f3), ("radius", C.c_float), ("color", f3), ("exposure", C.c_float),
                ("tex", C.c_int32)]


class SceneDesc(C.Structure):
    _fields_ = [("verts", C.c_void_p), ("nvert", C.c_uint32), ("tri_vidx", C.c_void_p), ("tri_attr", C.c_void_p),
                ("corner_normals", C.c_void_p), ("corner_uvs", C.c_void_p), ("ntri", C.c_uint32),
                ("attr_material", C.c_void_p), ("attr_emission", C.c_void_p), ("nattr", C.c_uint32),
                ("materials", C.c_void_p), ("nmat", C.c_uint32), ("lights", C.c_void_p), ("nlight", C.c_uint32),
                ("texels", C.c_void_p), ("tex_dims", C.c_void_p), ("ntex", C.c_uint32), ("fov", C.c_float),
                ("width", C.c_int32), ("height", C.c_int32), ("tex_triplanar_scale", C.c_void_p),
                ("attr_camera_to_object", C.c_void_p)]


class RenderOpts(C.Structure):
    _fields_ = [("spp", C.c_int32), ("sample_offset", C.c_int32), ("max_depth", C.c_int32),
                ("min_depth", C.c_int32), ("seed", C.c_uint32), ("mode", C.c_int32), ("fp64_film", C.c_int32),
                ("wf_pool", C.c_int32), ("wf_block", C.c_int32), ("wf_sort", C.c_int32),
                ("count_work", C.c_int32), ("light_samples", C.c_int32)]


class RenderStats(C.Structure):
    _fields_ = [("camera_rays", C.c_uint64), ("closest_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("paths", C.c_uint64), ("node_visits", C.c_uint64), ("tri_tests", C.c_uint64),
                ("launches", C.c_uint64), ("kernel_ms", C.c_double), ("shadow_node_visits", C.c_uint64),
                ("shadow_tri_tests", C.c_uint64), ("stage_ms", C.c_double * 5), ("wf_pool", C.c_int32),
                ("wf_block", C.c_int32), ("wf_sort", C.c_int32), ("node_bytes", C.c_int32)]


vp = C.c_void_p
# aur_pass_fn: int32 (*)(void* user, const float* film, int32 samples_done)
PASS_FN = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.POINTER(C.c_float), C.c_int32)
st = C.c_int
pp = C.POINTER(C.c_void_p)

# name: (restype, argtypes) — one line per declaration of include/aurora_b200.h
SIGNATURES = {
    "aur_last_error": (C.c_char_p, []),
    "aur_status_string": (C.c_char_p, [st]),
    "aur_version": (C.c_char_p, []),
    "aur_ctx_create": (st, [C.c_int, pp]),
    "aur_ctx_destroy": (st, [vp]),
    "aur_ctx_set_stream": (st, [vp, vp]),
    "aur_ctx_synchronize": (st, [vp]),
    "aur_bvh_build": (st, [vp, vp, C.c_uint32, vp, vp, C.c_uint32, C.POINTER(BvhOpts), pp]),
    "aur_bvh_destroy": (st, [vp]),
    "aur_bvh_info": (st, [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_float)]),
    "aur_trace_closest": (st, [vp, vp, vp, C.c_uint32]),
    "aur_trace_occluded": (st, [vp, vp, vp, C.c_uint32]),
    "aur_bvh_set_shading": (st, [vp, vp, vp]),
    "aur_bvh_intersect": (st, [vp, vp, vp, C.c_uint32]),
    "aur_scene_create": (st, [vp, C.POINTER(SceneDesc), C.POINTER(BvhOpts), pp]),
    "aur_scene_load_json": (st, [vp, C.c_char_p, C.POINTER(BvhOpts), pp, C.POINTER(RenderOpts)]),
    "aur_scene_file_read": (st, [C.c_char_p, pp]),
    "aur_scene_file_desc": (st, [vp, C.POINTER(SceneDesc), C.POINTER(RenderOpts)]),
    "aur_scene_file_output": (C.c_char_p, [vp]),
    "aur_scene_file_light_samples": (C.c_int32, [vp]),
    "aur_scene_file_destroy": (st, [vp]),
    "aur_film_write": (st, [C.c_char_p, vp, C.c_int32, C.c_int32, C.c_int32]),
    "aur_scene_destroy": (st, [vp]),
    "aur_scene_info": (st, [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_uint32),
                            C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "aur_scene_bvh": (st, [vp, pp]),
    "aur_scene_set_params": (st, [vp, vp, vp]),
    "aur_scene_get_params": (st, [vp, vp, vp]),
    "aur_render": (st, [vp, C.POINTER(RenderOpts), vp, C.POINTER(RenderStats)]),
    "aur_render_progressive": (st, [vp, C.POINTER(RenderOpts), C.c_int32, vp, vp, vp, C.POINTER(RenderStats)]),
    "aur_render_f64": (st, [vp, C.POINTER(RenderOpts), vp, C.POINTER(RenderStats)]),
    "aur_render_fp64acc_noalloc": (st, [vp, C.POINTER(RenderOpts), vp, C.POINTER(RenderStats)]),
    "aur_render_batch": (st, [C.POINTER(C.c_void_p), C.POINTER(RenderOpts), C.c_uint32, C.POINTER(C.c_void_p),
                              C.POINTER(RenderStats)]),
    "aur_render_adjoint": (st, [vp, C.POINTER(RenderOpts), vp, vp, vp, C.POINTER(RenderStats)]),
    "aur_kelemen_table": (st, [vp, C.c_float, vp]),
    "aur_shading_probe": (st, [vp, vp, C.c_int, vp, C.c_uint32, vp]),
    "aur_measure_read_bandwidth": (st, [vp, C.c_uint64, C.c_int32, C.POINTER(C.c_double)]),
}

_lib = None


def lib() -> C.CDLL:
    """Loads the in-tree shared library once; raises AuroraError if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise AuroraError(8, f"{LIB_PATH} is not built (run aurora_b200.build.build())")
    handle = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(handle, name)   # AttributeError if the symbol is missing: no silent fallback
        fn.restype = res
        fn.argtypes = args
    _lib = handle
    return handle


def check(status: int, what: str) -> None:
    if status != AUR_OK:
        raise AuroraError(status, f"{what}: {lib().aur_last_error().decode(errors='replace')}")
