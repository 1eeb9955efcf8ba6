"""ctypes bindings of the C ABI declared in include/wayland_b200.h.

The shared library is wayland_b200/lib/libwayland_b200.so (built in-tree by
wayland_b200.build). There is no fallback: if the library is missing, every call raises.
"""
import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libwayland_b200.so")

WL_OK = 0
ERR_NAMES = {0: "WL_OK", 1: "WL_ERR_INVALID_ARG", 2: "WL_ERR_CUDA", 3: "WL_ERR_OOM",
             4: "WL_ERR_QUEUE_OVERFLOW", 5: "WL_ERR_TIMEOUT", 6: "WL_ERR_NOT_BUILT",
             7: "WL_ERR_UNSUPPORTED"}
STRATEGY_UPT, STRATEGY_NEE, STRATEGY_MIS, STRATEGY_BDPT = 0, 1, 2, 3
BDPT_MAX_VERTICES = 10
RNG_TEA_LCG, RNG_PCG32 = 0, 1
MATH_FAST, MATH_STRICT = 0, 1
LIGHTS_UNIFORM, LIGHTS_POWER = 0, 1
FILM_RUNNING_MEAN, FILM_FP64_SUM = 1, 2
BVH_LBVH, BVH_SAH = 0, 1
CAST_CLOSEST, CAST_ANY = 0, 1
RENDER_TRAVERSAL_STATS = 1
RENDER_GRAPH = 2
RENDER_SORT_MATERIALS = 4
INVALID = 0xFFFFFFFF


class Disney(C.Structure):
    _fields_ = [("color", C.c_float * 3), ("metallic", C.c_float), ("roughness", C.c_float),
                ("specular", C.c_float), ("specular_tint", C.c_float), ("eta", C.c_float),
                ("trans", C.c_float), ("subsurface", C.c_float), ("anisotropic", C.c_float),
                ("sheen", C.c_float), ("sheen_tint", C.c_float), ("clearcoat", C.c_float),
                ("clearcoat_gloss", C.c_float), ("texture", C.c_int32)]


class AreaLight(C.Structure):
    _fields_ = [("L", C.c_float * 3), ("two_sided", C.c_int32), ("first_tri", C.c_uint32),
                ("tri_count", C.c_uint32)]


class Camera(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("look_at", C.c_float * 3), ("up", C.c_float * 3),
                ("right", C.c_float * 3)]


class RenderParams(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32),
                ("first_frame", C.c_uint32), ("max_depth", C.c_uint32), ("rr_depth", C.c_uint32),
                ("rr_prob", C.c_float), ("eps", C.c_float), ("strategy", C.c_uint32),
                ("rng", C.c_uint32), ("math", C.c_uint32), ("lights", C.c_uint32),
                ("seed", C.c_uint64), ("env", C.c_float * 3), ("wave_paths", C.c_uint32),
                ("flags", C.c_uint32)]


class AoParams(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("spp", C.c_uint32),
                ("first_frame", C.c_uint32), ("camera_samples", C.c_uint32),
                ("ao_rays", C.c_uint32), ("radius", C.c_float), ("eps", C.c_float),
                ("rng", C.c_uint32), ("wave_paths", C.c_uint32), ("seed", C.c_uint64)]


class NrcParams(C.Structure):
    _fields_ = [("levels", C.c_uint32), ("log2_table", C.c_uint32), ("base_resolution", C.c_uint32),
                ("per_level_scale", C.c_float), ("train_paths", C.c_uint32),
                ("query_depth", C.c_uint32), ("learning_rate", C.c_float), ("seed", C.c_uint32),
                ("train_extra", C.c_uint32)]


NRC_WEIGHTS = 17408


class TuneResult(C.Structure):
    _fields_ = [("wave_paths", C.c_uint32), ("extend_ctas_per_sm", C.c_uint32),
                ("extend_refill", C.c_uint32), ("shadow_ctas_per_sm", C.c_uint32),
                ("shadow_refill", C.c_uint32), ("candidates", C.c_uint32), ("spp", C.c_uint32),
                ("ms_default", C.c_float), ("ms_tuned", C.c_float),
                ("extend_postpone", C.c_uint32), ("shadow_postpone", C.c_uint32),
                ("shadow_far_first", C.c_uint32)]


class RenderStats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("segments", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("waves", C.c_uint32), ("kernel_launches", C.c_uint32), ("ms_total", C.c_float),
                ("ms_extend", C.c_float), ("ms_shade", C.c_float), ("ms_shadow", C.c_float),
                ("ms_other", C.c_float), ("extend_node_visits", C.c_uint64),
                ("extend_tri_tests", C.c_uint64), ("shadow_node_visits", C.c_uint64),
                ("shadow_tri_tests", C.c_uint64)]


class BvhInfo(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("num_tris", C.c_uint32), ("binary_nodes", C.c_uint32),
                ("wide_nodes", C.c_uint32), ("wide_depth", C.c_uint32), ("leaf_tris", C.c_uint32),
                ("ms_build", C.c_float), ("bytes", C.c_uint64)]


DISNEY_DTYPE = np.dtype([("color", np.float32, 3), ("metallic", np.float32),
                         ("roughness", np.float32), ("specular", np.float32),
                         ("specular_tint", np.float32), ("eta", np.float32),
                         ("trans", np.float32), ("subsurface", np.float32),
                         ("anisotropic", np.float32), ("sheen", np.float32),
                         ("sheen_tint", np.float32), ("clearcoat", np.float32),
                         ("clearcoat_gloss", np.float32), ("texture", np.int32)])
LIGHT_DTYPE = np.dtype([("L", np.float32, 3), ("two_sided", np.int32),
                        ("first_tri", np.uint32), ("tri_count", np.uint32)])
RAY_DTYPE = np.dtype([("org", np.float32, 3), ("tmin", np.float32), ("dir", np.float32, 3),
                      ("tmax", np.float32)])
HIT_DTYPE = np.dtype([("t", np.float32), ("prim", np.uint32), ("u", np.float32),
                      ("v", np.float32)])
assert DISNEY_DTYPE.itemsize == C.sizeof(Disney) == 64
assert LIGHT_DTYPE.itemsize == C.sizeof(AreaLight) == 24
assert RAY_DTYPE.itemsize == 32 and HIT_DTYPE.itemsize == 16

# Every symbol include/wayland_b200.h declares, with its ctypes signature.
_P = C.c_void_p
_U32 = C.c_uint32
class NrcGridDesc(C.Structure):
    _fields_ = [("levels", C.c_uint32), ("log2_table", C.c_uint32), ("base_resolution", C.c_uint32),
                ("per_level_scale", C.c_float), ("lo", C.c_float * 3), ("inv_ext", C.c_float * 3)]


# wl_nrc_vertex (64 bytes) as a numpy record
NRC_VERTEX_DTYPE = np.dtype([("pos", np.float32, 3), ("material", np.uint32), ("wo", np.float32, 3),
                             ("pad0", np.float32), ("n", np.float32, 3), ("pad1", np.float32),
                             ("extra", np.float32, 4)])


SIGNATURES = {
    "wl_context_create": (C.c_int, [C.c_int, C.POINTER(_P)]),
    "wl_context_destroy": (C.c_int, [_P]),
    "wl_context_set_stream": (C.c_int, [_P, _P]),
    "wl_context_get_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "wl_context_sync": (C.c_int, [_P]),
    "wl_last_error_string": (C.c_char_p, []),
    "wl_version": (C.c_char_p, []),
    "wl_scene_create": (C.c_int, [_P, _P, _U32, _P, _P, _P, _U32, _P, _P, _P, _U32, _P, _U32,
                                  C.POINTER(_P)]),
    "wl_scene_destroy": (C.c_int, [_P]),
    "wl_scene_add_texture": (C.c_int, [_P, _P, _U32, _U32, C.POINTER(C.c_int32)]),
    "wl_bvh_build": (C.c_int, [_P, _U32]),
    "wl_bvh_get_info": (C.c_int, [_P, C.POINTER(BvhInfo)]),
    "wl_bvh_export_morton": (C.c_int, [_P, _P, _U32]),
    "wl_bvh_export_binary": (C.c_int, [_P, _P, _P, _P, _P, _P, _U32]),
    "wl_cast_rays": (C.c_int, [_P, _P, _P, _U32, _U32]),
    "wl_cast_rays_host": (C.c_int, [_P, _P, _P, _U32, _U32]),
    "wl_cast_rays_stats": (C.c_int, [_P, _P, _U32, _U32, C.POINTER(C.c_uint64),
                                     C.POINTER(C.c_uint64)]),
    "wl_film_create": (C.c_int, [_P, _U32, _U32, _U32, C.POINTER(_P)]),
    "wl_film_destroy": (C.c_int, [_P]),
    "wl_film_clear": (C.c_int, [_P]),
    "wl_film_download": (C.c_int, [_P, _P, _P]),
    "wl_film_download_ldr": (C.c_int, [_P, _P]),
    "wl_film_device_ptrs": (C.c_int, [_P, C.POINTER(_P), C.POINTER(_P), C.POINTER(_P)]),
    "wl_render": (C.c_int, [_P, _P, C.POINTER(Camera), C.POINTER(RenderParams), _P]),
    "wl_render_get_stats": (C.c_int, [_P, C.POINTER(RenderStats)]),
    "wl_render_params_default": (None, [C.POINTER(RenderParams), _U32, _U32, _U32]),
    "wl_debug_rng": (C.c_int, [_P, _U32, C.c_uint64, _P, _U32, _U32, _U32, _P]),
    "wl_render_noalloc": (C.c_int, [_P, _P, C.POINTER(Camera), C.POINTER(RenderParams), _P]),
    "wl_ao_params_default": (None, [C.POINTER(AoParams), _U32, _U32, _U32]),
    "wl_render_batch": (C.c_int, [_P, _U32, _P, _P, _P, _P]),
    "wl_autotune": (C.c_int, [_P, _P, C.POINTER(Camera), C.POINTER(RenderParams), C.POINTER(TuneResult)]),
    "wl_set_tune": (C.c_int, [_P, _P]),
    "wl_nrc_params_default": (None, [C.POINTER(NrcParams)]),
    "wl_nrc_create": (C.c_int, [_P, _P, C.POINTER(NrcParams), C.POINTER(_P)]),
    "wl_nrc_destroy": (C.c_int, [_P]),
    "wl_nrc_reserve": (C.c_int, [_P, _P, C.POINTER(RenderParams)]),
    "wl_render_nrc": (C.c_int, [_P, _P, C.POINTER(Camera), C.POINTER(RenderParams), _P, _P]),
    "wl_nrc_mlp_forward": (C.c_int, [_P, _P, _P, _U32]),
    "wl_nrc_train_step": (C.c_int, [_P, _P, _P, _U32, C.POINTER(C.c_float)]),
    "wl_nrc_mlp_gradients": (C.c_int, [_P, _P, _P, _U32, _P]),
    "wl_nrc_get_weights": (C.c_int, [_P, _P]),
    "wl_nrc_set_weights": (C.c_int, [_P, _P]),
    "wl_nrc_stats": (C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_float)]),
    "wl_render_ao": (C.c_int, [_P, _P, C.POINTER(Camera), C.POINTER(AoParams), _P]),
    "wl_nrc_set_wait_limit": (C.c_int, [_P, _U32]),
    "wl_nrc_kernel_times": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "wl_nrc_get_grid": (C.c_int, [_P, C.POINTER(NrcGridDesc), _P]),
    "wl_nrc_set_grid": (C.c_int, [_P, _P]),
    "wl_nrc_query": (C.c_int, [_P, _P, _U32, _P]),
    "wl_nrc_debug_encode": (C.c_int, [_P, _P, _U32, _P, _P]),
    "wl_nrc_sample_gradients": (C.c_int, [_P, _P, _U32, _P, _P, C.POINTER(C.c_float)]),
}
NOALLOC_MAX_PATHS = 65536
NRC_WAIT_POLLS = 4194304


class WlError(RuntimeError):
    def __init__(self, fn, code, msg):
        super().__init__(f"{fn} failed: {ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


_lib = None


def header_symbols():
    """Names of the functions include/wayland_b200.h declares (parsed from the header)."""
    import re
    hdr = os.path.join(os.path.dirname(PKG), "include", "wayland_b200.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"^\s*(?:WL_API\s+)?(?:int|void|const char \*)\s*(wl_\w+)\s*\(", text, re.M)))


def load(path=None):
    """Load the native library; raises if it was not built (no fallback exists)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"native library not built: {p} (run wayland_b200.build.build_all())")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(fn, code):
    if code != WL_OK:
        msg = load().wl_last_error_string()
        raise WlError(fn, code, msg.decode() if msg else "")


def call(name, *args):
    lib = load()
    code = getattr(lib, name)(*args)
    check(name, code)
