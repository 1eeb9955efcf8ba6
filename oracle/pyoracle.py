"""ctypes bindings of the CPU oracle (test infrastructure only).

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg; never by the product
path. `liboracle.so` is the project's restatement (oracle/wl_oracle.cpp); `libwlref.so` is the
reference's own src/Frontend/Device/*.h compiled on the host (oracle/ref_build), present only
where it was built.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_ORACLE = os.path.join(HERE, "_build", "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libwlref.so")
# the reference source tree (only the oracle recipes read it); WL_REFERENCE_ROOT overrides it
REF_TREE = os.environ.get("WL_REFERENCE_ROOT", "/root/reference")

ORACLE_FLAGS = ["-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fopenmp",
                "-shared", "-fPIC"]


def build_oracle(force=False):
    """Compile oracle/wl_oracle.cpp -> oracle/_build/liboracle.so."""
    src = os.path.join(HERE, "wl_oracle.cpp")
    if (not force and os.path.exists(LIB_ORACLE)
            and os.path.getmtime(LIB_ORACLE) >= max(os.path.getmtime(src),
                                                    os.path.getmtime(os.path.join(HERE, "wl_oracle.h")))):
        return LIB_ORACLE
    os.makedirs(os.path.dirname(LIB_ORACLE), exist_ok=True)
    subprocess.check_call(["g++", *ORACLE_FLAGS, src, "-o", LIB_ORACLE])
    return LIB_ORACLE


def build_ref():
    """Compile the reference's device math into oracle/_ref/libwlref.so (needs the tree)."""
    if not os.path.isdir(REF_TREE):
        return None
    subprocess.check_call(["make", "-s", "-C", os.path.join(HERE, "ref_build"), f"REF={REF_TREE}"])
    return LIB_REF


# ---- C structs mirroring include/wayland_b200.h ------------------------------------------
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


class OrScene(C.Structure):
    _fields_ = [("V", C.c_void_p), ("nV", C.c_uint32), ("N", C.c_void_p), ("I", C.c_void_p),
                ("nT", C.c_uint32), ("tri_material", C.c_void_p), ("tri_flags", C.c_void_p),
                ("mats", C.c_void_p), ("nMat", C.c_uint32), ("lights", C.c_void_p),
                ("nLight", C.c_uint32), ("UV", C.c_void_p), ("nTex", C.c_uint32),
                ("tex_rgba", C.c_void_p), ("tex_w", C.c_void_p), ("tex_h", C.c_void_p)]


RAY_DTYPE = np.dtype([("org", np.float32, 3), ("tmin", np.float32), ("dir", np.float32, 3),
                      ("tmax", np.float32)])
HIT_DTYPE = np.dtype([("t", np.float32), ("prim", np.uint32), ("u", np.float32),
                      ("v", np.float32)])
DISNEY_DTYPE = np.dtype([("color", np.float32, 3), ("metallic", np.float32),
                         ("roughness", np.float32), ("specular", np.float32),
                         ("specular_tint", np.float32), ("eta", np.float32),
                         ("trans", np.float32), ("subsurface", np.float32),
                         ("anisotropic", np.float32), ("sheen", np.float32),
                         ("sheen_tint", np.float32), ("clearcoat", np.float32),
                         ("clearcoat_gloss", np.float32), ("texture", np.int32)])
LIGHT_DTYPE = np.dtype([("L", np.float32, 3), ("two_sided", np.int32),
                        ("first_tri", np.uint32), ("tri_count", np.uint32)])
assert DISNEY_DTYPE.itemsize == C.sizeof(Disney) == 64
assert RAY_DTYPE.itemsize == 32 and HIT_DTYPE.itemsize == 16


def make_or_scene(scene):
    """Flatten a scene (attributes V, N, I, tri_material, tri_flags, mats, lights) into the
    oracle's or_scene struct. Returns (arrays to keep alive, struct)."""
    V = _f32(scene.V, (-1, 3))
    N = None if scene.N is None else _f32(scene.N, (-1, 3))
    I = np.ascontiguousarray(scene.I, np.uint32).reshape(-1, 3)
    tm = np.ascontiguousarray(scene.tri_material, np.uint32)
    tf = None if scene.tri_flags is None else np.ascontiguousarray(scene.tri_flags, np.uint32)
    mats = np.ascontiguousarray(scene.mats).view(DISNEY_DTYPE)
    lights = np.ascontiguousarray(scene.lights).view(LIGHT_DTYPE)
    UV = getattr(scene, "UV", None)
    UV = None if UV is None else _f32(UV, (-1, 2))
    texs = [np.ascontiguousarray(t, np.uint8).reshape(t.shape[0], t.shape[1], 4)
            for t in (getattr(scene, "textures", None) or [])]
    tex_ptrs = (C.c_void_p * max(len(texs), 1))(*[t.ctypes.data for t in texs])
    tw = np.array([t.shape[1] for t in texs] or [0], np.uint32)
    th = np.array([t.shape[0] for t in texs] or [0], np.uint32)
    s = OrScene(V=V.ctypes.data, nV=len(V), N=None if N is None else N.ctypes.data,
                I=I.ctypes.data, nT=len(I), tri_material=tm.ctypes.data,
                tri_flags=None if tf is None else tf.ctypes.data, mats=mats.ctypes.data,
                nMat=len(mats), lights=lights.ctypes.data if len(lights) else None,
                nLight=len(lights), UV=None if UV is None else UV.ctypes.data, nTex=len(texs),
                tex_rgba=C.cast(tex_ptrs, C.c_void_p), tex_w=tw.ctypes.data, tex_h=th.ctypes.data)
    return (V, N, I, tm, tf, mats, lights, UV, texs, tex_ptrs, tw, th), s


def ptr(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a if shape is None else a.reshape(shape)


class Oracle:
    """The project's CPU restatement (liboracle.so)."""

    def __init__(self, path=None):
        self.lib = C.CDLL(path or build_oracle())
        L = self.lib
        L.or_tea4.restype = C.c_uint32
        L.or_tea4.argtypes = [C.c_uint32, C.c_uint32]
        L.or_sinf.restype = L.or_cosf.restype = L.or_logf.restype = C.c_float
        L.or_sinf.argtypes = L.or_cosf.argtypes = L.or_logf.argtypes = [C.c_float]
        L.or_rng_stream.argtypes = [C.c_uint32, C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32,
                                    C.c_void_p]
        L.or_render.restype = C.c_uint64
        L.or_render.argtypes = [C.POINTER(OrScene), C.c_void_p, C.POINTER(Camera),
                                C.POINTER(RenderParams), C.c_int, C.c_int, C.c_void_p,
                                C.c_void_p, C.c_uint32, C.c_uint32]
        L.or_bvh_create.restype = C.c_void_p
        L.or_bvh_create.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
        L.or_bvh_destroy.argtypes = [C.c_void_p]
        L.or_cast_bvh.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]
        L.or_relmse.restype = C.c_double
        L.or_relmse.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_double]

    # -- scalar helpers
    def tea4(self, a, b):
        return self.lib.or_tea4(a, b)

    def rng_stream(self, rng, seed, pixel, frame, count):
        out = np.empty(count, np.float32)
        self.lib.or_rng_stream(rng, seed, pixel, frame, count, ptr(out))
        return out

    def lcg_stream(self, state, count):
        out = np.empty(count, np.float32)
        self.lib.or_lcg_stream(C.c_uint32(state), C.c_uint32(count), ptr(out))
        return out

    def sinf(self, x):
        return np.float32(self.lib.or_sinf(float(x)))

    def cosf(self, x):
        return np.float32(self.lib.or_cosf(float(x)))

    def logf(self, x):
        return np.float32(self.lib.or_logf(float(x)))

    # -- BSDF batches
    def disney_eval(self, mats, Ns, Ng, V, L, tex=None):
        n = len(mats)
        out = np.empty((n, 3), np.float32)
        args = [_f32(x, (n, 3)) for x in (Ns, Ng, V, L)]
        t = None if tex is None else _f32(tex, (n, 3))
        self.lib.or_disney_eval(C.c_uint32(n), ptr(mats), *[ptr(a) for a in args], ptr(t), ptr(out))
        return out

    def disney_pdf(self, mats, Ns, Ng, V, L):
        n = len(mats)
        out = np.empty(n, np.float32)
        args = [_f32(x, (n, 3)) for x in (Ns, Ng, V, L)]
        self.lib.or_disney_pdf(C.c_uint32(n), ptr(mats), *[ptr(a) for a in args], ptr(out))
        return out

    def disney_sample(self, mats, Ns, Ng, V, seeds):
        n = len(mats)
        out = np.empty((n, 3), np.float32)
        s = np.ascontiguousarray(seeds, np.uint32).copy()
        args = [_f32(x, (n, 3)) for x in (Ns, Ng, V)]
        self.lib.or_disney_sample(C.c_uint32(n), ptr(mats), *[ptr(a) for a in args], ptr(s), ptr(out))
        return out, s

    def camera_rays(self, cam, W, H, px, py, seeds):
        n = len(px)
        out = np.empty((n, 3), np.float32)
        s = np.ascontiguousarray(seeds, np.uint32).copy()
        px = np.ascontiguousarray(px, np.uint32)
        py = np.ascontiguousarray(py, np.uint32)
        self.lib.or_camera_ray(C.byref(cam), C.c_uint32(W), C.c_uint32(H), C.c_uint32(n),
                               ptr(px), ptr(py), ptr(s), ptr(out))
        return out, s

    def ace(self, rgb):
        rgb = _f32(rgb, (-1, 3))
        out = np.empty_like(rgb)
        self.lib.or_ace(C.c_uint32(len(rgb)), ptr(rgb), ptr(out))
        return out

    # -- geometry
    def cast_bruteforce(self, V, I, rays, mode=0):
        V = _f32(V); I = np.ascontiguousarray(I, np.uint32)
        hits = np.empty(len(rays), HIT_DTYPE)
        self.lib.or_cast_bruteforce(ptr(V), ptr(I), C.c_uint32(I.size // 3), ptr(rays),
                                    C.c_uint32(len(rays)), C.c_uint32(mode), ptr(hits))
        return hits

    def cast_bruteforce_f64(self, V, I, rays):
        V = _f32(V); I = np.ascontiguousarray(I, np.uint32)
        t = np.empty(len(rays), np.float64)
        p = np.empty(len(rays), np.uint32)
        self.lib.or_cast_bruteforce_f64(ptr(V), ptr(I), C.c_uint32(I.size // 3), ptr(rays),
                                        C.c_uint32(len(rays)), ptr(t), ptr(p))
        return t, p

    def morton63(self, V, I):
        V = _f32(V); I = np.ascontiguousarray(I, np.uint32)
        n = I.size // 3
        out = np.empty(n, np.uint64)
        self.lib.or_morton63(ptr(V), ptr(I), C.c_uint32(n), ptr(out))
        return out

    def lbvh(self, V, I):
        V = _f32(V); I = np.ascontiguousarray(I, np.uint32)
        n = I.size // 3
        sp = np.empty(n, np.uint32)
        left = np.full(max(n - 1, 0), -1, np.int32)
        right = np.full(max(n - 1, 0), -1, np.int32)
        parent = np.full(2 * n - 1, -1, np.int32)
        bounds = np.zeros((2 * n - 1, 6), np.float32)
        self.lib.or_lbvh(ptr(V), ptr(I), C.c_uint32(n), ptr(sp), ptr(left), ptr(right),
                         ptr(parent), ptr(bounds))
        return sp, left, right, parent, bounds

    def bvh(self, V, I):
        return OracleBVH(self, V, I)

    def render(self, scene, cam, params, prec=0, threads=0, film=None, want64=False,
               pixel_range=None):
        """Render with the oracle; returns (film_rgb[H,W,3] f32, film64 or None, segments)."""
        W, H = params.width, params.height
        film = np.zeros((H, W, 3), np.float32) if film is None else film
        f64 = np.zeros((H, W, 3), np.float64) if want64 else None
        b = self.bvh_for(scene)
        lo, hi = pixel_range or (0, W * H)
        keep, osc = make_or_scene(scene)
        segs = self.lib.or_render(C.byref(osc), b.handle, C.byref(cam), C.byref(params), prec,
                                  threads, ptr(film), ptr(f64), lo, hi)
        del keep
        return film, f64, segs

    def render_ao(self, scene, cam, params, threads=0, want64=False):
        """Ambient occlusion (AO.cu:21-130); returns (film[H,W,3] f32, film64 or None, rays)."""
        W, H = params.width, params.height
        film = np.zeros((H, W, 3), np.float32)
        f64 = np.zeros((H, W, 3), np.float64) if want64 else None
        b = self.bvh_for(scene)
        keep, osc = make_or_scene(scene)
        self.lib.or_render_ao.restype = C.c_uint64
        rays = self.lib.or_render_ao(C.byref(osc), b.handle, C.byref(cam), C.byref(params), threads,
                                     ptr(film), ptr(f64))
        del keep
        return film, f64, rays

    def render_bdpt(self, scene, cam, params, prec=0, threads=0, film=None, want64=False, max_len=0):
        """Bidirectional path tracer (BDPT.cu:42-567); returns (film_rgb[H,W,3] f32, film64 or
        None, rays). max_len > 0 keeps only the paths of at most max_len vertices after the
        camera (or_render_bdpt_len)."""
        W, H = params.width, params.height
        film = np.zeros((H, W, 3), np.float32) if film is None else film
        f64 = np.zeros((H, W, 3), np.float64) if want64 else None
        b = self.bvh_for(scene)
        keep, osc = make_or_scene(scene)
        self.lib.or_render_bdpt_len.restype = C.c_uint64
        rays = self.lib.or_render_bdpt_len(C.byref(osc), b.handle, C.byref(cam), C.byref(params),
                                           C.c_uint32(max_len), prec, threads, ptr(film), ptr(f64))
        del keep
        return film, f64, rays

    def bvh_for(self, scene):
        key = id(scene)
        c = self.__dict__.setdefault("_bvh_cache", {})
        if key not in c or c[key][0] is not scene:
            c.clear()
            c[key] = (scene, OracleBVH(self, scene.V, scene.I))
        return c[key][1]

    def relmse(self, img, ref, eps=1e-2):
        img = np.ascontiguousarray(img, np.float32).ravel()
        ref = np.ascontiguousarray(ref, np.float64).ravel()
        return self.lib.or_relmse(ptr(img), ptr(ref), C.c_uint64(img.size), eps)


class OracleBVH:
    def __init__(self, oracle, V, I):
        self.o = oracle
        self.V = _f32(V)
        self.I = np.ascontiguousarray(I, np.uint32)
        self.handle = oracle.lib.or_bvh_create(ptr(self.V), ptr(self.I), self.I.size // 3)

    def cast(self, rays, mode=0):
        hits = np.empty(len(rays), HIT_DTYPE)
        self.o.lib.or_cast_bvh(self.handle, ptr(rays), C.c_uint32(len(rays)), C.c_uint32(mode),
                               ptr(hits))
        return hits

    def __del__(self):
        try:
            self.o.lib.or_bvh_destroy(self.handle)
        except Exception:
            pass


class RefLib:
    """The reference's own device math compiled on the host (oracle/_ref/libwlref.so)."""

    def __init__(self, path=LIB_REF):
        self.lib = C.CDLL(path)
        L = self.lib
        L.ref_tea4.restype = C.c_uint32
        L.ref_tea4.argtypes = [C.c_uint32, C.c_uint32]
        L.ref_render.restype = C.c_uint64
        L.ref_render.argtypes = [C.POINTER(OrScene), C.c_void_p, C.POINTER(Camera),
                                 C.POINTER(RenderParams), C.c_int, C.c_void_p, C.c_uint32,
                                 C.c_uint32]
        L.or_bvh_create.restype = C.c_void_p
        L.or_bvh_create.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
        L.or_bvh_destroy.argtypes = [C.c_void_p]

    def tea4(self, a, b):
        return self.lib.ref_tea4(a, b)

    def rnd_stream(self, seed, count):
        out = np.empty(count, np.float32)
        self.lib.ref_rnd_stream(C.c_uint32(seed), C.c_uint32(count), ptr(out))
        return out

    def disney_eval(self, mats, Ns, Ng, V, L, tex=None):
        n = len(mats)
        out = np.empty((n, 3), np.float32)
        args = [_f32(x, (n, 3)) for x in (Ns, Ng, V, L)]
        t = None if tex is None else _f32(tex, (n, 3))
        self.lib.ref_disney_eval(C.c_uint32(n), ptr(mats), *[ptr(a) for a in args], ptr(t), ptr(out))
        return out

    def disney_pdf(self, mats, Ns, Ng, V, L):
        n = len(mats)
        out = np.empty(n, np.float32)
        args = [_f32(x, (n, 3)) for x in (Ns, Ng, V, L)]
        self.lib.ref_disney_pdf(C.c_uint32(n), ptr(mats), *[ptr(a) for a in args], ptr(out))
        return out

    def disney_sample(self, mats, Ns, Ng, V, seeds):
        n = len(mats)
        out = np.empty((n, 3), np.float32)
        s = np.ascontiguousarray(seeds, np.uint32).copy()
        args = [_f32(x, (n, 3)) for x in (Ns, Ng, V)]
        self.lib.ref_disney_sample(C.c_uint32(n), ptr(mats), *[ptr(a) for a in args], ptr(s), ptr(out))
        return out, s

    def camera_rays(self, cam, W, H, px, py, seeds):
        n = len(px)
        out = np.empty((n, 3), np.float32)
        s = np.ascontiguousarray(seeds, np.uint32).copy()
        px = np.ascontiguousarray(px, np.uint32)
        py = np.ascontiguousarray(py, np.uint32)
        self.lib.ref_camera_ray(C.byref(cam), C.c_uint32(W), C.c_uint32(H), C.c_uint32(n),
                                ptr(px), ptr(py), ptr(s), ptr(out))
        return out, s

    def ace(self, rgb):
        rgb = _f32(rgb, (-1, 3))
        out = np.empty_like(rgb)
        self.lib.ref_ace(C.c_uint32(len(rgb)), ptr(rgb), ptr(out))
        return out

    def render_ao(self, scene, cam, params, threads=0):
        W, H = params.width, params.height
        film = np.zeros((H, W, 3), np.float32)
        keep, osc = make_or_scene(scene)
        h = self.lib.or_bvh_create(osc.V, osc.I, osc.nT)
        self.lib.ref_render_ao.restype = C.c_uint64
        try:
            rays = self.lib.ref_render_ao(C.byref(osc), C.c_void_p(h), C.byref(cam), C.byref(params),
                                          threads, ptr(film))
        finally:
            self.lib.or_bvh_destroy(h)
        return film, rays

    def render(self, scene, cam, params, threads=0, film=None, pixel_range=None):
        W, H = params.width, params.height
        film = np.zeros((H, W, 3), np.float32) if film is None else film
        keep, osc = make_or_scene(scene)
        h = self.lib.or_bvh_create(osc.V, osc.I, osc.nT)
        lo, hi = pixel_range or (0, W * H)
        try:
            segs = self.lib.ref_render(C.byref(osc), h, C.byref(cam), C.byref(params),
                                       threads, ptr(film), lo, hi)
        finally:
            self.lib.or_bvh_destroy(h)
        return film, segs

    def render_bdpt(self, scene, cam, W, H, spp, first_frame=0, threads=0, radiance=None):
        """The reference's BDPT program (Programs/BDPT/BDPT.cu, run over the OptiX host emulation).
        Returns the reference's radiance buffer [H, W, 4] (FP32 running mean)."""
        rad = np.zeros((H, W, 4), np.float32) if radiance is None else radiance
        keep, osc = make_or_scene(scene)
        h = self.lib.or_bvh_create(osc.V, osc.I, osc.nT)
        L = self.lib
        L.ref_render_bdpt.restype = C.c_uint64
        L.ref_render_bdpt.argtypes = [C.POINTER(OrScene), C.c_void_p, C.POINTER(Camera), C.c_uint32,
                                      C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_void_p]
        try:
            L.ref_render_bdpt(C.byref(osc), h, C.byref(cam), W, H, spp, first_frame, threads, ptr(rad))
        finally:
            self.lib.or_bvh_destroy(h)
        del keep
        return rad

    def _program(self, fn, scene, cam, W, H, spp, first_frame, threads, radiance, extra=()):
        rad = np.zeros((H, W, 4), np.float32) if radiance is None else radiance
        keep, osc = make_or_scene(scene)
        h = self.lib.or_bvh_create(osc.V, osc.I, osc.nT)
        f = getattr(self.lib, fn)
        f.restype = C.c_uint64
        f.argtypes = [C.POINTER(OrScene), C.c_void_p, C.POINTER(Camera), C.c_uint32, C.c_uint32,
                      C.c_uint32, C.c_uint32, C.c_int, C.c_void_p] + [C.c_uint32] * len(extra)
        try:
            f(C.byref(osc), h, C.byref(cam), W, H, spp, first_frame, threads, ptr(rad), *extra)
        finally:
            self.lib.or_bvh_destroy(h)
        del keep
        return rad

    def program_pt(self, scene, cam, W, H, spp, first_frame=0, threads=0, radiance=None,
                   pixel_range=None):
        """The reference's PathTracing.cu program itself (OptiX host emulation); returns its
        radiance buffer [H, W, 4]."""
        lo, hi = pixel_range or (0, W * H)
        return self._program("ref_program_pt", scene, cam, W, H, spp, first_frame, threads, radiance,
                             (lo, hi))

    def program_ao(self, scene, cam, W, H, spp, first_frame=0, threads=0, radiance=None):
        """The reference's AO.cu program itself (views where every camera ray hits)."""
        return self._program("ref_program_ao", scene, cam, W, H, spp, first_frame, threads, radiance)
