"""wayland_b200 - B200-native renderer backend (wavefront path tracer behind a C ABI).

Python host mirror of the C ABI in include/wayland_b200.h, organised like the reference's
frontend seam:
  Context          ContextManager (src/Backend/Optix/Core/ContextManager.cpp:99-157)
  Scene            SceneManager data uploaded by DeviceManager::UploadDeviceBuffer
                   (src/Frontend/Core/DeviceManager.cpp:111-181) + StaticAccelStructure
  Film             radiance + colour buffers (PathTracingProgramManager.cpp:30-32,
                   DeviceManager.cpp:80)
  PathTracer       PathTracingProgramManager{Setup, Update, End}
                   (src/Frontend/Programs/PathTracing/PathTracingProgramManager.cpp:11-55):
                   Update() renders the next frame(s) and advances frameID.
All work runs in libwayland_b200.so; nothing here computes pixels.
"""
import ctypes as C
import weakref

import numpy as np

from . import _abi
from ._abi import (BVH_LBVH, BVH_SAH, CAST_ANY, CAST_CLOSEST, FILM_FP64_SUM, INVALID,
                   LIGHTS_POWER, LIGHTS_UNIFORM, MATH_FAST, MATH_STRICT, RNG_PCG32, RNG_TEA_LCG,
                   STRATEGY_BDPT, STRATEGY_MIS, STRATEGY_NEE, STRATEGY_UPT, BDPT_MAX_VERTICES,
                   HIT_DTYPE, RAY_DTYPE, WlError)

__all__ = ["Context", "Scene", "Film", "PathTracer", "render_params", "WlError", "RAY_DTYPE",
           "HIT_DTYPE"]


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


class Context:
    """One device + one CUDA stream."""

    def __init__(self, device=0):
        self.lib = _abi.load()
        h = C.c_void_p()
        _abi.check("wl_context_create", self.lib.wl_context_create(device, C.byref(h)))
        self.handle = h
        self.device = device
        self._children = weakref.WeakSet()

    @property
    def stream(self):
        s = C.c_void_p()
        _abi.check("wl_context_get_stream", self.lib.wl_context_get_stream(self.handle, C.byref(s)))
        return s.value or 0

    def set_stream(self, stream_ptr):
        _abi.check("wl_context_set_stream",
                   self.lib.wl_context_set_stream(self.handle, C.c_void_p(stream_ptr or None)))

    def sync(self):
        _abi.check("wl_context_sync", self.lib.wl_context_sync(self.handle))

    def close(self):
        """Destroys the scenes and films still alive on this context, then the context."""
        if getattr(self, "handle", None):
            for ch in list(self._children):
                ch.close()
            _abi.check("wl_context_destroy", self.lib.wl_context_destroy(self.handle))
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def stats(self):
        s = _abi.RenderStats()
        _abi.check("wl_render_get_stats", self.lib.wl_render_get_stats(self.handle, C.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}

    def autotune(self, scene, camera, params):
        """wl_autotune: choose and keep the fastest launch shape for renders like this one."""
        r = _abi.TuneResult()
        _abi.check("wl_autotune", self.lib.wl_autotune(self.handle, scene.handle, C.byref(camera),
                                                       C.byref(params), C.byref(r)))
        return {k: getattr(r, k) for k, _ in r._fields_}

    def set_tune(self, tune=None):
        """wl_set_tune: a shape returned by autotune (dict), or None for the defaults (missing
        triangle-phase thresholds default to 12)."""
        if tune is None:
            _abi.check("wl_set_tune", self.lib.wl_set_tune(self.handle, None))
            return
        full = dict(extend_postpone=12, shadow_postpone=12)
        full.update(tune)
        r = _abi.TuneResult(**{k: full[k] for k, _ in _abi.TuneResult._fields_ if k in full})
        _abi.check("wl_set_tune", self.lib.wl_set_tune(self.handle, C.byref(r)))

    def debug_rng(self, rng, seed, d_pixels_ptr, npix, frame, count, d_out_ptr):
        _abi.check("wl_debug_rng", self.lib.wl_debug_rng(self.handle, rng, seed, C.c_void_p(d_pixels_ptr),
                                                         npix, frame, count, C.c_void_p(d_out_ptr)))


class Scene:
    """A flattened scene on the device (see wayland_b200.scenes.Scene for the fields)."""

    def __init__(self, ctx, data, build=True, bvh_kind=BVH_LBVH):
        self.ctx = ctx
        self.lib = ctx.lib
        self.data = data
        V = np.ascontiguousarray(data.V, np.float32).reshape(-1, 3)
        I = np.ascontiguousarray(data.I, np.uint32).reshape(-1, 3)
        N = None if data.N is None else np.ascontiguousarray(data.N, np.float32).reshape(-1, 3)
        tm = np.ascontiguousarray(data.tri_material, np.uint32)
        tf = None if data.tri_flags is None else np.ascontiguousarray(data.tri_flags, np.uint32)
        mats = np.ascontiguousarray(data.mats).view(_abi.DISNEY_DTYPE)
        lights = np.ascontiguousarray(data.lights).view(_abi.LIGHT_DTYPE)
        UV = getattr(data, "UV", None)
        UV = None if UV is None else np.ascontiguousarray(UV, np.float32).reshape(-1, 2)
        h = C.c_void_p()
        _abi.check("wl_scene_create", self.lib.wl_scene_create(
            ctx.handle, _p(V), len(V), _p(N), _p(UV), _p(I), len(I), _p(tm), _p(tf), _p(mats),
            len(mats), _p(lights) if len(lights) else None, len(lights), C.byref(h)))
        self.handle = h
        ctx._children.add(self)
        self.num_tris = len(I)
        for tex in (getattr(data, "textures", None) or []):
            t = np.ascontiguousarray(tex, np.uint8)
            idx = C.c_int32()
            _abi.check("wl_scene_add_texture", self.lib.wl_scene_add_texture(
                self.handle, _p(t), t.shape[1], t.shape[0], C.byref(idx)))
        if build:
            self.build_bvh(bvh_kind)

    def build_bvh(self, kind=BVH_LBVH):
        _abi.check("wl_bvh_build", self.lib.wl_bvh_build(self.handle, kind))

    def info(self):
        i = _abi.BvhInfo()
        _abi.check("wl_bvh_get_info", self.lib.wl_bvh_get_info(self.handle, C.byref(i)))
        return {k: getattr(i, k) for k, _ in i._fields_}

    def export_morton(self):
        out = np.empty(self.num_tris, np.uint64)
        _abi.check("wl_bvh_export_morton",
                   self.lib.wl_bvh_export_morton(self.handle, _p(out), self.num_tris))
        return out

    def export_binary(self):
        n = self.num_tris
        sp = np.empty(n, np.uint32)
        left = np.empty(max(n - 1, 1), np.int32)
        right = np.empty(max(n - 1, 1), np.int32)
        parent = np.empty(2 * n - 1, np.int32)
        bounds = np.empty((2 * n - 1, 6), np.float32)
        _abi.check("wl_bvh_export_binary", self.lib.wl_bvh_export_binary(
            self.handle, _p(sp), _p(left), _p(right), _p(parent), _p(bounds), n))
        return sp, left[:n - 1], right[:n - 1], parent, bounds

    def cast(self, d_rays_ptr, d_hits_ptr, n, mode=CAST_CLOSEST):
        """Device pointers (e.g. torch tensors' data_ptr()), stream ordered."""
        _abi.check("wl_cast_rays", self.lib.wl_cast_rays(self.handle, C.c_void_p(d_rays_ptr),
                                                         C.c_void_p(d_hits_ptr), n, mode))

    def cast_host(self, rays, mode=CAST_CLOSEST):
        rays = np.ascontiguousarray(rays).view(RAY_DTYPE)
        hits = np.empty(len(rays), HIT_DTYPE)
        _abi.check("wl_cast_rays_host",
                   self.lib.wl_cast_rays_host(self.handle, _p(rays), _p(hits), len(rays), mode))
        return hits

    def cast_stats(self, d_rays_ptr, n, mode=CAST_CLOSEST):
        a, b = C.c_uint64(), C.c_uint64()
        _abi.check("wl_cast_rays_stats", self.lib.wl_cast_rays_stats(
            self.handle, C.c_void_p(d_rays_ptr), n, mode, C.byref(a), C.byref(b)))
        return a.value, b.value

    def close(self):
        if getattr(self, "handle", None):
            self.lib.wl_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Film:
    def __init__(self, ctx, width, height, fp64=False):
        self.ctx = ctx
        self.lib = ctx.lib
        self.width, self.height = width, height
        self.fp64 = fp64
        h = C.c_void_p()
        _abi.check("wl_film_create", self.lib.wl_film_create(
            ctx.handle, width, height, FILM_FP64_SUM if fp64 else 0, C.byref(h)))
        self.handle = h
        ctx._children.add(self)

    def clear(self):
        _abi.check("wl_film_clear", self.lib.wl_film_clear(self.handle))

    def download(self, out=None):
        out = np.empty((self.height, self.width, 3), np.float32) if out is None else out
        _abi.check("wl_film_download", self.lib.wl_film_download(self.handle, _p(out), None))
        return out

    def download64(self):
        out = np.empty((self.height, self.width, 3), np.float64)
        _abi.check("wl_film_download", self.lib.wl_film_download(self.handle, None, _p(out)))
        return out

    def download_ldr(self):
        out = np.empty((self.height, self.width, 4), np.uint8)
        _abi.check("wl_film_download_ldr", self.lib.wl_film_download_ldr(self.handle, _p(out)))
        return out

    def save_png(self, path):
        """The tone-mapped film (AceApprox, 8-bit) as a PNG file, flipped vertically like the
        reference's output (Renderer.cpp:94-105)."""
        from .png import write_png
        write_png(path, self.download_ldr())

    def device_ptrs(self):
        a, b, c = C.c_void_p(), C.c_void_p(), C.c_void_p()
        _abi.check("wl_film_device_ptrs",
                   self.lib.wl_film_device_ptrs(self.handle, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def close(self):
        if getattr(self, "handle", None):
            self.lib.wl_film_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def render_params(width, height, spp, **kw):
    """wl_render_params with the reference's constants (wl_render_params_default), then kw."""
    p = _abi.RenderParams()
    _abi.load().wl_render_params_default(C.byref(p), width, height, spp)
    for k, v in kw.items():
        if k == "env":
            p.env[:] = [float(x) for x in v]
        else:
            setattr(p, k, v)
    return p


def ao_params(width, height, spp, **kw):
    """wl_ao_params with the reference's constants (4 camera samples, 32 rays, radius 1)."""
    p = _abi.AoParams()
    _abi.load().wl_ao_params_default(C.byref(p), width, height, spp)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def render_ao(ctx, scene, camera, params, film):
    """Ambient occlusion (AO.cu) into the film's running mean."""
    _abi.check("wl_render_ao", ctx.lib.wl_render_ao(ctx.handle, scene.handle, C.byref(camera),
                                                    C.byref(params), film.handle))


class RadianceCache:
    """The neural radiance cache (hash grid + MLP) of a scene; wl_nrc_* in the C ABI."""

    def __init__(self, ctx, scene, **kw):
        self.ctx = ctx
        self.lib = ctx.lib
        p = _abi.NrcParams()
        self.lib.wl_nrc_params_default(C.byref(p))
        for k, v in kw.items():
            setattr(p, k, v)
        self.params = p
        h = C.c_void_p()
        _abi.check("wl_nrc_create", self.lib.wl_nrc_create(ctx.handle, scene.handle, C.byref(p), C.byref(h)))
        self.handle = h
        ctx._children.add(self)

    def reserve(self, params):
        """Allocate the buffers that render_nrc with these params needs (no rendering)."""
        _abi.check("wl_nrc_reserve", self.lib.wl_nrc_reserve(self.ctx.handle, self.handle,
                                                             C.byref(params)))

    def forward(self, d_in, d_out, n):
        _abi.check("wl_nrc_mlp_forward", self.lib.wl_nrc_mlp_forward(self.handle, C.c_void_p(d_in),
                                                                     C.c_void_p(d_out), n))

    def train_step(self, d_in, d_target, n):
        loss = C.c_float()
        _abi.check("wl_nrc_train_step", self.lib.wl_nrc_train_step(
            self.handle, C.c_void_p(d_in), C.c_void_p(d_target), n, C.byref(loss)))
        return loss.value

    def gradients(self, d_in, d_target, n):
        g = np.empty(_abi.NRC_WEIGHTS, np.float32)
        _abi.check("wl_nrc_mlp_gradients", self.lib.wl_nrc_mlp_gradients(
            self.handle, C.c_void_p(d_in), C.c_void_p(d_target), n, _p(g)))
        return g

    def weights(self):
        w = np.empty(_abi.NRC_WEIGHTS, np.float32)
        _abi.check("wl_nrc_get_weights", self.lib.wl_nrc_get_weights(self.handle, _p(w)))
        return w

    def set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        _abi.check("wl_nrc_set_weights", self.lib.wl_nrc_set_weights(self.handle, _p(w)))

    def stats(self):
        a, b, l = C.c_uint32(), C.c_uint32(), C.c_float()
        _abi.check("wl_nrc_stats", self.lib.wl_nrc_stats(self.handle, C.byref(a), C.byref(b), C.byref(l)))
        return {"train_samples": a.value, "queries": b.value, "loss": l.value}

    def kernel_times(self):
        """(ms of the last query-MLP kernel, ms of the last training kernel), device time."""
        a, b = C.c_float(), C.c_float()
        _abi.check("wl_nrc_kernel_times", self.lib.wl_nrc_kernel_times(self.handle, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_wait_limit(self, polls):
        """mbarrier polls before a tensor-core wait gives up (0: at once; a test hook)."""
        _abi.check("wl_nrc_set_wait_limit", self.lib.wl_nrc_set_wait_limit(self.handle, polls))

    def grid(self, with_params=True):
        """(descriptor dict, FP32 master parameters (levels, 2^log2_table, 2) or None)."""
        d = _abi.NrcGridDesc()
        _abi.check("wl_nrc_get_grid", self.lib.wl_nrc_get_grid(self.handle, C.byref(d), None))
        desc = {"levels": d.levels, "log2_table": d.log2_table, "base_resolution": d.base_resolution,
                "per_level_scale": d.per_level_scale, "lo": list(d.lo), "inv_ext": list(d.inv_ext)}
        if not with_params:
            return desc, None
        params = np.empty((d.levels, 1 << d.log2_table, 2), np.float32)
        _abi.check("wl_nrc_get_grid", self.lib.wl_nrc_get_grid(self.handle, None, _p(params)))
        return desc, params

    def set_grid(self, params):
        params = np.ascontiguousarray(params, np.float32)
        _abi.check("wl_nrc_set_grid", self.lib.wl_nrc_set_grid(self.handle, _p(params)))

    def query(self, d_vertices, n, d_rgb):
        """Cache predictions for n device wl_nrc_vertex records into d_rgb (n x 4 floats)."""
        _abi.check("wl_nrc_query", self.lib.wl_nrc_query(self.handle, C.c_void_p(d_vertices), n,
                                                         C.c_void_p(d_rgb)))

    def debug_encode(self, d_vertices, n, d_features, d_corners=None):
        _abi.check("wl_nrc_debug_encode", self.lib.wl_nrc_debug_encode(
            self.handle, C.c_void_p(d_vertices), n, C.c_void_p(d_features),
            C.c_void_p(d_corners) if d_corners else None))

    def sample_gradients(self, d_samples, n):
        """(loss, weight gradient (17408,), grid gradient (levels, 2^log2_table, 2)) of one
        training step on n device samples, not applied."""
        desc, _ = self.grid(with_params=False)
        gw = np.empty(_abi.NRC_WEIGHTS, np.float32)
        gg = np.empty((desc["levels"], 1 << desc["log2_table"], 2), np.float32)
        loss = C.c_float()
        _abi.check("wl_nrc_sample_gradients", self.lib.wl_nrc_sample_gradients(
            self.handle, C.c_void_p(d_samples), n, _p(gw), _p(gg), C.byref(loss)))
        return loss.value, gw, gg

    def close(self):
        if getattr(self, "handle", None):
            self.lib.wl_nrc_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def render_nrc(ctx, scene, camera, params, cache, film):
    """params.spp frames with the radiance cache: query, then one training step per frame.
    film=None trains the cache without producing an image (warm-up frames)."""
    _abi.check("wl_render_nrc", ctx.lib.wl_render_nrc(ctx.handle, scene.handle, C.byref(camera),
                                                      C.byref(params), cache.handle,
                                                      film.handle if film is not None else None))


def render_batch(ctx, scenes, cameras, params, films):
    """wl_render_batch: several (scene, camera, params, film) jobs rendered together."""
    n = len(scenes)
    sh = (C.c_void_p * n)(*[s.handle for s in scenes])
    fh = (C.c_void_p * n)(*[f.handle for f in films])
    cams = (_abi.Camera * n)(*cameras)
    ps = (_abi.RenderParams * n)(*params)
    _abi.check("wl_render_batch", ctx.lib.wl_render_batch(ctx.handle, n, sh, cams, ps, fh))


def render(ctx, scene, camera, params, film):
    _abi.check("wl_render", ctx.lib.wl_render(ctx.handle, scene.handle, C.byref(camera),
                                              C.byref(params), film.handle))


class PathTracer:
    """PathTracingProgramManager: Setup() allocates the film, Update() renders `spp` more
    samples per pixel and advances frameID, End() releases the film."""

    def __init__(self, ctx, scene, camera, width, height, fp64=False, **params):
        self.ctx, self.scene, self.camera = ctx, scene, camera
        self.width, self.height, self.fp64 = width, height, fp64
        self.params = params
        self.frame = 0
        self.film = None

    def Setup(self):
        self.film = Film(self.ctx, self.width, self.height, fp64=self.fp64)
        self.frame = 0

    def Update(self, spp=1):
        p = render_params(self.width, self.height, spp, first_frame=self.frame, **self.params)
        render(self.ctx, self.scene, self.camera, p, self.film)
        self.frame += spp

    def End(self):
        if self.film is not None:
            self.film.close()
            self.film = None
