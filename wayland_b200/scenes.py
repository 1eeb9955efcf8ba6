"""Procedural scenes for the benchmark configurations (seeded, synthetic).

The reference renders pbrt scenes (scene/*.pbrt via SceneManager, src/Frontend/Core/
SceneManager.cpp:14-49); the configurations measured here are procedural stand-ins with the
shapes, sizes and value distributions the benchmark names:

  cornell_box()        Plain PT, procedural Cornell box: unit-cube room of 5 quads, two
                       axis-aligned boxes of height 0.3 and 0.6, one 0.25 x 0.25 ceiling light
                       of radiance (17, 12, 4), matte albedos white 0.73, red (0.65, 0.05, 0.05),
                       green (0.12, 0.45, 0.15); 256 x 256, 16 spp, depth 8.
  displaced_sphere()   Plain PT at scale: icosphere subdivided to about 2M triangles displaced by
                       fBm of amplitude 0.05, on a 2-triangle ground plane; Disney parameters per
                       object from the seed; 4 quad lights and a constant environment of 0.1;
                       1920 x 1080, 64 spp, depth 16.
  door_slit_room()     Radiance-cache PT: a ~500K-triangle room lit only through a 0.05-wide
                       door slit by an area light outside (mostly indirect light), glossy Disney
                       walls with roughness U[0.1, 0.4].

Matte surfaces use the reference's matte -> Disney mapping (Material.cpp:51-67: roughness 0.5,
specular 0, sheenTint 0.5, eta 1.5), since the renderer's only surface model is that BSDF.
"""
from dataclasses import dataclass, field
import math

import numpy as np

from . import _abi

DISNEY = _abi.DISNEY_DTYPE
LIGHT = _abi.LIGHT_DTYPE


@dataclass
class Scene:
    """Flattened scene: the SceneManager fields (SceneManager.h:30-44) as the C ABI takes them."""
    name: str
    V: np.ndarray                      # (nV, 3) float32
    I: np.ndarray                      # (nT, 3) uint32
    tri_material: np.ndarray           # (nT,) uint32
    mats: np.ndarray                   # (nMat,) DISNEY
    lights: np.ndarray                 # (nLight,) LIGHT
    N: np.ndarray = None               # (nV, 3) float32 or None
    tri_flags: np.ndarray = None       # (nT,) uint32 or None
    camera: dict = field(default_factory=dict)   # pos, look_at, up, right (wl_camera)
    width: int = 256
    height: int = 256
    spp: int = 16
    max_depth: int = 8
    env: tuple = (0.0, 0.0, 0.0)
    UV: np.ndarray = None              # (nV, 2) float32 texture coordinates or None
    textures: list = field(default_factory=list)  # RGBA8 images (h, w, 4) uint8; mats' texture indexes them

    @property
    def num_tris(self):
        return int(self.I.shape[0])

    def camera_struct(self):
        c = _abi.Camera()
        for k in ("pos", "look_at", "up", "right"):
            getattr(c, k)[:] = [float(x) for x in self.camera[k]]
        return c


def disney(color, metallic=0.0, roughness=0.5, specular=0.0, specular_tint=0.0, eta=1.5,
           trans=0.0, subsurface=0.0, anisotropic=0.0, sheen=0.0, sheen_tint=0.5,
           clearcoat=0.0, clearcoat_gloss=1.0, texture=-1):
    m = np.zeros((), DISNEY)
    m["color"] = color
    for k, v in dict(metallic=metallic, roughness=roughness, specular=specular,
                     specular_tint=specular_tint, eta=eta, trans=trans, subsurface=subsurface,
                     anisotropic=anisotropic, sheen=sheen, sheen_tint=sheen_tint,
                     clearcoat=clearcoat, clearcoat_gloss=clearcoat_gloss, texture=texture).items():
        m[k] = v
    return m


def matte(color):
    """Disney(minipbrt::MatteMaterial*), Material.cpp:51-67."""
    return disney(color, metallic=0.0, roughness=0.5, specular=0.0, specular_tint=0.0, eta=1.5,
                  trans=0.0, sheen=0.0, sheen_tint=0.5, clearcoat=0.0, clearcoat_gloss=1.0)


def pinhole(pos, target, up, fov_deg, width, height):
    """PinholeCamera (Camera.cpp:15-28) + the aspect scaling of PathTracingProgramManager.cpp:28:
    lookAt = normalize(target - pos), up scaled by tan(fov/2), right = cross(lookAt, up) * W/H."""
    pos = np.asarray(pos, np.float64)
    look = np.asarray(target, np.float64) - pos
    look /= np.linalg.norm(look)
    up = np.asarray(up, np.float64)
    up = up - look * np.dot(up, look)
    up /= np.linalg.norm(up)
    up = up * math.tan(math.radians(fov_deg) / 2)
    right = np.cross(look, up) * (width / height)
    return dict(pos=pos.astype(np.float32), look_at=look.astype(np.float32),
                up=up.astype(np.float32), right=right.astype(np.float32))


def _quad(p0, p1, p2, p3):
    """Two triangles (p0, p1, p2), (p0, p2, p3); normal = cross(p1 - p0, p2 - p0)."""
    V = np.array([p0, p1, p2, p3], np.float32)
    I = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    return V, I


def _box(lo, hi):
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    faces = [
        ((x0, y0, z0), (x1, y0, z0), (x1, y0, z1), (x0, y0, z1)),  # bottom
        ((x0, y1, z0), (x0, y1, z1), (x1, y1, z1), (x1, y1, z0)),  # top
        ((x0, y0, z0), (x0, y1, z0), (x1, y1, z0), (x1, y0, z0)),  # z0
        ((x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1)),  # z1
        ((x0, y0, z0), (x0, y0, z1), (x0, y1, z1), (x0, y1, z0)),  # x0
        ((x1, y0, z0), (x1, y1, z0), (x1, y1, z1), (x1, y0, z1)),  # x1
    ]
    return [_quad(*f) for f in faces]


class _Builder:
    def __init__(self):
        self.V, self.I, self.M = [], [], []
        self.nv = 0

    def add(self, parts, mat):
        first = sum(len(i) for i in self.I)
        for V, I in parts:
            self.V.append(V)
            self.I.append(I + self.nv)
            self.M.append(np.full(len(I), mat, np.uint32))
            self.nv += len(V)
        return first, sum(len(i) for i in self.I) - first

    def arrays(self):
        return (np.concatenate(self.V).astype(np.float32), np.concatenate(self.I).astype(np.uint32),
                np.concatenate(self.M).astype(np.uint32))


def cornell_box(width=256, height=256, spp=16, max_depth=8):
    """Config 1: 10 room triangles + 24 box triangles + 2 light triangles = 36."""
    b = _Builder()
    white, red, green = 0, 1, 2
    mats = np.array([matte((0.73, 0.73, 0.73)), matte((0.65, 0.05, 0.05)),
                     matte((0.12, 0.45, 0.15))])
    # room: x, y, z in [0, 1], open towards +z where the camera is
    b.add([_quad((0, 0, 0), (1, 0, 0), (1, 0, 1), (0, 0, 1))], white)   # floor
    b.add([_quad((0, 1, 0), (0, 1, 1), (1, 1, 1), (1, 1, 0))], white)   # ceiling
    b.add([_quad((0, 0, 0), (0, 1, 0), (1, 1, 0), (1, 0, 0))], white)   # back wall
    b.add([_quad((0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0))], red)     # left wall
    b.add([_quad((1, 0, 0), (1, 1, 0), (1, 1, 1), (1, 0, 1))], green)   # right wall
    b.add(_box((0.13, 0.0, 0.53), (0.43, 0.3, 0.83)), white)            # short box
    b.add(_box((0.53, 0.0, 0.17), (0.83, 0.6, 0.47)), white)            # tall box
    # ceiling light, facing down: cross(p1 - p0, p2 - p0) = -y
    y = 0.999
    first, count = b.add([_quad((0.375, y, 0.375), (0.625, y, 0.375), (0.625, y, 0.625),
                                (0.375, y, 0.625))], white)
    V, I, M = b.arrays()
    lights = np.zeros(1, LIGHT)
    lights[0]["L"] = (17.0, 12.0, 4.0)
    lights[0]["two_sided"] = 0
    lights[0]["first_tri"] = first
    lights[0]["tri_count"] = count
    cam = pinhole((0.5, 0.5, 2.4), (0.5, 0.5, 0.0), (0, 1, 0), 39.3, width, height)
    return Scene("cornell_box", V, I, M, mats, lights, camera=cam, width=width, height=height,
                 spp=spp, max_depth=max_depth)


def checker_texture(n=32, seed=0):
    """An n x n RGBA8 test image: a two-colour checkerboard of 4 x 4 texel squares with seeded
    per-texel noise (so that bilinear filtering has something to interpolate)."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:n, 0:n]
    board = ((x // 4 + y // 4) % 2).astype(np.float64)
    a = np.array([0.85, 0.8, 0.7]) * 255
    b = np.array([0.2, 0.35, 0.6]) * 255
    img = board[..., None] * a + (1 - board[..., None]) * b + rng.uniform(-20, 20, (n, n, 3))
    out = np.empty((n, n, 4), np.uint8)
    out[..., :3] = np.clip(img, 0, 255).astype(np.uint8)
    out[..., 3] = 255
    return out


def textured_cornell_box(width=256, height=256, spp=16, max_depth=8):
    """The Cornell box with a checker texture (material 3, texture 0) tiled 4 x 4 on the floor and
    3 x 3 on the back wall, through per-vertex texture coordinates (the reference's ImageMap Kd
    path, PathTracing.cu:262-268)."""
    sc = cornell_box(width, height, spp, max_depth)
    nV = len(sc.V)
    UV = np.zeros((nV, 2), np.float32)
    # floor = vertices 0..3 (triangles 0, 1); back wall = vertices 8..11 (triangles 4, 5)
    UV[0:4] = np.array([[0, 0], [4, 0], [4, 4], [0, 4]], np.float32)
    UV[8:12] = np.array([[0, 0], [0, 3], [3, 3], [3, 0]], np.float32) + 0.37
    tex_mat = matte((0.9, 0.9, 0.9))
    tex_mat["texture"] = 0
    sc.mats = np.concatenate([sc.mats, np.array([tex_mat])])
    tm = sc.tri_material.copy()
    tm[[0, 1, 4, 5]] = len(sc.mats) - 1
    sc.tri_material = tm
    sc.UV = UV
    sc.textures = [checker_texture(32)]
    sc.name = "cornell_box_textured"
    return sc


# ---- config 2 ------------------------------------------------------------------------------
def _icosahedron():
    t = (1.0 + 5 ** 0.5) / 2.0
    V = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                  [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]],
                 np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    F = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9],
                  [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2],
                  [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11], [6, 2, 10],
                  [8, 6, 7], [9, 8, 1]], np.int64)
    return V, F


def subdivided_icosphere(n):
    """Each icosahedron face split into n^2 triangles (20 n^2 in total), vertices welded."""
    V0, F = _icosahedron()
    ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    keep = (ii + jj) <= n
    ii, jj = ii[keep], jj[keep]
    local = -np.ones((n + 1, n + 1), np.int64)
    local[ii, jj] = np.arange(len(ii))
    # triangles of one face in (i, j) lattice coordinates
    a_i, a_j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    up = (a_i + a_j) <= n - 1
    ui, uj = a_i[up], a_j[up]
    t_up = np.stack([local[ui, uj], local[ui + 1, uj], local[ui, uj + 1]], 1)
    dn = (a_i + a_j) <= n - 2
    di, dj = a_i[dn], a_j[dn]
    t_dn = np.stack([local[di + 1, dj], local[di + 1, dj + 1], local[di, dj + 1]], 1)
    tri_local = np.concatenate([t_up, t_dn])
    P, T = [], []
    for f, (a, b, c) in enumerate(F):
        A, B, Cc = V0[a], V0[b], V0[c]
        pts = A[None] + (B - A)[None] * (ii[:, None] / n) + (Cc - A)[None] * (jj[:, None] / n)
        P.append(pts)
        T.append(tri_local + f * len(ii))
    P = np.concatenate(P)
    T = np.concatenate(T)
    P /= np.linalg.norm(P, axis=1, keepdims=True)
    key = np.round(P * 1e7).astype(np.int64)
    _, first, inv = np.unique(key, axis=0, return_index=True, return_inverse=True)
    return P[first], inv.reshape(-1)[T]


def _value_noise(p, seed):
    """Smoothstep-interpolated lattice value noise in [-1, 1] (hashed integer lattice)."""
    pi = np.floor(p).astype(np.int64)
    f = p - pi
    w = f * f * (3.0 - 2.0 * f)

    def h(ix, iy, iz):
        x = (ix * 73856093) ^ (iy * 19349663) ^ (iz * 83492791) ^ (seed * 2654435761)
        x = (x ^ (x >> 13)) * 1274126177
        x = x ^ (x >> 16)
        return (x & 0xFFFF).astype(np.float64) / 32767.5 - 1.0

    out = 0.0
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                wx = w[:, 0] if dx else 1 - w[:, 0]
                wy = w[:, 1] if dy else 1 - w[:, 1]
                wz = w[:, 2] if dz else 1 - w[:, 2]
                out = out + wx * wy * wz * h(pi[:, 0] + dx, pi[:, 1] + dy, pi[:, 2] + dz)
    return out


def fbm(p, seed, octaves=5, base=2.0):
    acc, amp, freq, norm = 0.0, 1.0, base, 0.0
    for o in range(octaves):
        acc = acc + amp * _value_noise(p * freq, seed + o)
        norm += amp
        amp *= 0.5
        freq *= 2.0
    return acc / norm


def vertex_normals(V, I):
    V = V.astype(np.float64)
    fn = np.cross(V[I[:, 1]] - V[I[:, 0]], V[I[:, 2]] - V[I[:, 0]])
    N = np.zeros_like(V)
    for k in range(3):
        np.add.at(N, I[:, k], fn)
    N /= np.maximum(np.linalg.norm(N, axis=1, keepdims=True), 1e-30)
    return N.astype(np.float32)


def random_disney(rng):
    """Per-object Disney parameters from the seed: metallic, specTrans ~ U[0,1],
    roughness ~ U[0.05, 1]."""
    return disney(tuple(rng.uniform(0.2, 0.9, 3)), metallic=rng.uniform(0, 1),
                  roughness=rng.uniform(0.05, 1.0), specular=0.5, trans=rng.uniform(0, 1),
                  eta=1.5, sheen_tint=0.5)


def displaced_sphere(width=1920, height=1080, spp=64, max_depth=16, subdiv=316, seed=0,
                     amplitude=0.05):
    """Config 2: 20*subdiv^2 sphere triangles (1,997,120 at subdiv 316) + 2 ground + 8 light."""
    rng = np.random.default_rng(seed)
    P, T = subdivided_icosphere(subdiv)
    r = 1.0 + amplitude * fbm(P * 1.5, seed)
    Vs = (P * r[:, None]).astype(np.float32)
    Is = T.astype(np.uint32)
    Ns = vertex_normals(Vs, Is)
    mats = np.array([random_disney(rng), random_disney(rng), matte((0.8, 0.8, 0.8))])
    y = -1.0 - 1.5 * amplitude
    Vg, Ig = _quad((-12, y, -12), (-12, y, 12), (12, y, 12), (12, y, -12))
    Vl, Il = [], []
    lights = np.zeros(4, LIGHT)
    centers = [(-2.5, 3.0, -2.0), (2.5, 3.0, -2.0), (-2.5, 3.0, 2.5), (2.5, 3.0, 2.5)]
    for k, (cx, cy, cz) in enumerate(centers):
        h = 0.5
        v, i = _quad((cx - h, cy, cz - h), (cx + h, cy, cz - h), (cx + h, cy, cz + h),
                     (cx - h, cy, cz + h))
        Vl.append(v)
        Il.append(i + 4 * k)
        lights[k]["L"] = tuple(rng.uniform(4.0, 8.0, 3))
        lights[k]["two_sided"] = 0
    nS = len(Vs)
    V = np.concatenate([Vs, Vg, *Vl]).astype(np.float32)
    I = np.concatenate([Is, Ig + nS, *(i + nS + 4 for i in Il)]).astype(np.uint32)
    N = np.concatenate([Ns, np.tile([[0, 1, 0]], (4, 1)), np.tile([[0, -1, 0]], (16, 1))]).astype(np.float32)
    M = np.concatenate([np.zeros(len(Is), np.uint32), np.ones(2, np.uint32),
                        np.full(8, 2, np.uint32)])
    flags = np.concatenate([np.ones(len(Is), np.uint32), np.zeros(10, np.uint32)])
    first = len(Is) + 2
    for k in range(4):
        lights[k]["first_tri"] = first + 2 * k
        lights[k]["tri_count"] = 2
    cam = pinhole((0.0, 0.6, 4.2), (0.0, -0.2, 0.0), (0, 1, 0), 40.0, width, height)
    return Scene("displaced_sphere", V, I, M, mats, lights, N=N, tri_flags=flags, camera=cam,
                 width=width, height=height, spp=spp, max_depth=max_depth, env=(0.1, 0.1, 0.1))


def glass_sphere(width=1024, height=1024, spp=256, max_depth=10, subdiv=89, light_size=0.05,
                 light_L=(4000.0, 3600.0, 3000.0), roughness=0.05):
    """Bidirectional configuration: a smooth glass sphere (20 subdiv^2 triangles, 158,420 at
    subdiv 89; specular transmission 1, IOR 1.5) resting on a 2-triangle diffuse plane, lit
    only by a small one-sided quad light (light_size wide) above it, so most of the plane
    under the sphere is lit by caustics that camera paths find only by connection. The glass
    roughness is 0.05: at roughness 0 the reference's Disney lobes (GTR2 with alpha 0.001 and
    pdfs clamped to [1e-30, 1e30]) give single samples of 1e16 and more, and no estimator of
    the image converges."""
    P, T = subdivided_icosphere(subdiv)
    Vs = P.astype(np.float32)
    Is = T.astype(np.uint32)
    Ns = vertex_normals(Vs, Is)
    glass = disney((1.0, 1.0, 1.0), metallic=0.0, roughness=roughness, specular=0.5, eta=1.5,
                   trans=1.0)
    mats = np.array([glass, matte((0.7, 0.7, 0.7)), matte((0.8, 0.8, 0.8))])
    y = -1.0
    Vg, Ig = _quad((-8, y, -8), (-8, y, 8), (8, y, 8), (8, y, -8))
    h = 0.5 * light_size
    ly = 2.5
    # facing down: cross(p1 - p0, p2 - p0) = -y
    Vl, Il = _quad((-0.6 - h, ly, 0.4 - h), (-0.6 + h, ly, 0.4 - h), (-0.6 + h, ly, 0.4 + h),
                   (-0.6 - h, ly, 0.4 + h))
    nS = len(Vs)
    V = np.concatenate([Vs, Vg, Vl]).astype(np.float32)
    I = np.concatenate([Is, Ig + nS, Il + nS + 4]).astype(np.uint32)
    N = np.concatenate([Ns, np.tile([[0, 1, 0]], (4, 1)), np.tile([[0, -1, 0]], (4, 1))]).astype(np.float32)
    M = np.concatenate([np.zeros(len(Is), np.uint32), np.ones(2, np.uint32), np.full(2, 2, np.uint32)])
    flags = np.concatenate([np.ones(len(Is), np.uint32), np.zeros(4, np.uint32)])
    lights = np.zeros(1, LIGHT)
    lights[0]["L"] = light_L
    lights[0]["two_sided"] = 0
    lights[0]["first_tri"] = len(Is) + 2
    lights[0]["tri_count"] = 2
    cam = pinhole((0.0, 1.2, 4.5), (0.0, -0.4, 0.0), (0, 1, 0), 38.0, width, height)
    return Scene("glass_sphere", V, I, M, mats, lights, N=N, tri_flags=flags, camera=cam,
                 width=width, height=height, spp=spp, max_depth=max_depth)


def icosphere_soup(n):
    """Each icosahedron face split into n^2 triangles (20 n^2 in total), 3 vertices per triangle
    (not welded: fast to build for millions of triangles; flat shading)."""
    V0, F = _icosahedron()
    a_i, a_j = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    up = (a_i + a_j) <= n - 1
    ui, uj = a_i[up].astype(np.float64), a_j[up].astype(np.float64)
    dn = (a_i + a_j) <= n - 2
    di, dj = a_i[dn].astype(np.float64), a_j[dn].astype(np.float64)
    # lattice coordinates of the three corners of every triangle of one face
    ci = np.concatenate([np.stack([ui, ui + 1, ui], 1), np.stack([di + 1, di + 1, di], 1)])
    cj = np.concatenate([np.stack([uj, uj, uj + 1], 1), np.stack([dj, dj + 1, dj + 1], 1)])
    out = []
    for a, b, c in F:
        A, B, Cc = V0[a], V0[b], V0[c]
        pts = A[None, None] + (B - A)[None, None] * (ci[..., None] / n) + (Cc - A)[None, None] * (cj[..., None] / n)
        out.append(pts)
    P = np.concatenate(out).reshape(-1, 3)
    P /= np.linalg.norm(P, axis=1, keepdims=True)
    return P.astype(np.float32), np.arange(len(P), dtype=np.uint32).reshape(-1, 3)


def batch_scene(seed):
    """One job of the batched configuration: a procedural scene from its seed. Triangles
    lognormal (median 200K) clipped to [10K, 5M] on an ellipsoid soup over a ground quad;
    random Disney material; 1-8 quad lights; resolution uniform in [256, 1024] per axis; spp
    uniform in [4, 64]; depth uniform in [4, 16]."""
    rng = np.random.default_rng(1000 + seed)
    ntris = int(np.clip(rng.lognormal(np.log(2e5), 1.2), 1e4, 5e6))
    n = max(int(round(np.sqrt(ntris / 20.0))), 1)
    P, I = icosphere_soup(n)
    P = P * rng.uniform(0.7, 1.3, 3)[None].astype(np.float32)
    y = float(P[:, 1].min()) - 0.01
    Vg, Ig = _quad((-10, y, -10), (-10, y, 10), (10, y, 10), (10, y, -10))
    k = int(rng.integers(1, 9))
    Vl, Il = [], []
    lights = np.zeros(k, LIGHT)
    for j in range(k):
        cx, cz = rng.uniform(-3, 3, 2)
        cy = rng.uniform(2.0, 4.0)
        h = rng.uniform(0.1, 0.6)
        v, i = _quad((cx - h, cy, cz - h), (cx + h, cy, cz - h), (cx + h, cy, cz + h), (cx - h, cy, cz + h))
        Vl.append(v)
        Il.append(i + 4 * j)
        lights[j]["L"] = tuple(rng.uniform(2.0, 10.0, 3))
        lights[j]["two_sided"] = int(rng.integers(0, 2))
    nS = len(P)
    V = np.concatenate([P, Vg, *Vl]).astype(np.float32)
    I = np.concatenate([I, Ig + nS, *(i + nS + 4 for i in Il)]).astype(np.uint32)
    mats = np.array([random_disney(rng), matte(tuple(rng.uniform(0.3, 0.9, 3))), matte((0.8, 0.8, 0.8))])
    nT = len(I)
    M = np.concatenate([np.zeros(nT - 2 - 2 * k, np.uint32), np.ones(2, np.uint32), np.full(2 * k, 2, np.uint32)])
    first = nT - 2 * k
    for j in range(k):
        lights[j]["first_tri"] = first + 2 * j
        lights[j]["tri_count"] = 2
    W = int(rng.integers(256, 1025))
    H = int(rng.integers(256, 1025))
    ang = rng.uniform(0, 2 * np.pi)
    cam = pinhole((3.5 * np.sin(ang), 1.2, 3.5 * np.cos(ang)), (0.0, 0.0, 0.0), (0, 1, 0), 45.0, W, H)
    return Scene(f"batch_{seed}", V, I.reshape(-1, 3), M, mats, lights, camera=cam, width=W, height=H,
                 spp=int(rng.integers(4, 65)), max_depth=int(rng.integers(4, 17)))


def _grid(p0, du, dv, nu, nv):
    """Quad p0 + [0,1] du + [0,1] dv tessellated into nu x nv cells (2 nu nv triangles);
    normal = cross(du, dv)."""
    u = np.linspace(0.0, 1.0, nu + 1)
    v = np.linspace(0.0, 1.0, nv + 1)
    uu, vv = np.meshgrid(u, v, indexing="ij")
    P = (np.asarray(p0, np.float64)[None] + uu.reshape(-1, 1) * np.asarray(du, np.float64)[None]
         + vv.reshape(-1, 1) * np.asarray(dv, np.float64)[None])
    i, j = np.meshgrid(np.arange(nu), np.arange(nv), indexing="ij")
    a = (i * (nv + 1) + j).reshape(-1)
    b = ((i + 1) * (nv + 1) + j).reshape(-1)
    c = ((i + 1) * (nv + 1) + j + 1).reshape(-1)
    d = (i * (nv + 1) + j + 1).reshape(-1)
    I = np.concatenate([np.stack([a, b, c], 1), np.stack([a, c, d], 1)])
    return P.astype(np.float32), I.astype(np.uint32)


def door_slit_room(width=1920, height=1080, spp=1, max_depth=16, seed=0, cells=200,
                   slit=0.05):
    """Radiance-cache configuration: a closed room 4 x 3 x 5 whose walls are tessellated into
    about 500K triangles (cells x cells quads per wall), lit only by an area light outside,
    through a vertical slit of width `slit` in the +x wall, so most of the light is indirect.
    Glossy Disney walls (roughness ~ U[0.1, 0.4]); four boxes and a displaced sphere inside."""
    rng = np.random.default_rng(seed)
    X, Y, Z = 4.0, 3.0, 5.0
    b = _Builder()
    mats = []

    def glossy():
        mats.append(disney(tuple(rng.uniform(0.35, 0.85, 3)), metallic=0.0,
                           roughness=rng.uniform(0.1, 0.4), specular=0.5, sheen_tint=0.5))
        return len(mats) - 1

    n = cells
    # floor, ceiling, walls x = 0, z = 0, z = Z
    b.add([_grid((0, 0, 0), (0, 0, Z), (X, 0, 0), n, n)], glossy())
    b.add([_grid((0, Y, 0), (X, 0, 0), (0, 0, Z), n, n)], glossy())
    b.add([_grid((0, 0, 0), (0, Y, 0), (0, 0, Z), n, n)], glossy())
    b.add([_grid((0, 0, 0), (X, 0, 0), (0, Y, 0), n, n)], glossy())
    b.add([_grid((0, 0, Z), (0, Y, 0), (X, 0, 0), n, n)], glossy())
    # +x wall with the slit: z in [zc - slit/2, zc + slit/2], y in [0, yt]
    zc, yt = 2.5, 2.2
    z0, z1 = zc - slit / 2, zc + slit / 2
    b.add([_grid((X, 0, 0), (0, 0, z0), (0, Y, 0), n // 2, n),
           _grid((X, 0, z1), (0, 0, Z - z1), (0, Y, 0), n // 2, n),
           _grid((X, yt, z0), (0, 0, z1 - z0), (0, Y - yt, 0), 1, 4)], glossy())
    for k in range(4):
        lo = np.array([rng.uniform(0.3, 3.0), 0.0, rng.uniform(0.3, 4.0)])
        size = np.array([rng.uniform(0.3, 0.8), rng.uniform(0.3, 1.2), rng.uniform(0.3, 0.8)])
        b.add(_box(tuple(lo), tuple(np.minimum(lo + size, [X - 0.4, Y - 0.2, Z - 0.2]))), glossy())
    P, T = subdivided_icosphere(40)
    r = 1.0 + 0.05 * fbm(P * 1.5, seed)
    Vs = (P * r[:, None] * 0.6 + np.array([1.2, 0.7, 3.4])).astype(np.float32)
    b.add([(Vs, T.astype(np.uint32))], glossy())
    # the light: a 1.2 x 2.0 quad at x = X + 1.5 facing -x (towards the slit), radiance ~60
    lx = X + 1.5
    first, count = b.add([_quad((lx, 0.1, zc - 0.6), (lx, 0.1, zc + 0.6), (lx, 2.1, zc + 0.6),
                                (lx, 2.1, zc - 0.6))], 0)
    V, I, M = b.arrays()
    lights = np.zeros(1, LIGHT)
    lights[0]["L"] = (60.0, 55.0, 45.0)
    lights[0]["two_sided"] = 0
    lights[0]["first_tri"] = first
    lights[0]["tri_count"] = count
    cam = pinhole((0.6, 1.6, 0.5), (3.0, 1.0, 4.2), (0, 1, 0), 60.0, width, height)
    return Scene("door_slit_room", V, I, M, np.array(mats), lights, camera=cam, width=width,
                 height=height, spp=spp, max_depth=max_depth)


def random_triangles(n, seed=0, spread=1.0, size=0.1):
    """Random triangle soup in [-spread, spread]^3 for traversal parity tests."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(-spread, spread, (n, 1, 3))
    V = (c + rng.normal(0, size, (n, 3, 3))).reshape(-1, 3).astype(np.float32)
    I = np.arange(3 * n, dtype=np.uint32).reshape(-1, 3)
    return V, I
