"""pbrt-v3 scene files -> the flattened scene of the C ABI (wayland_b200.scenes.Scene).

The reference's frontend reads pbrt-v3 files with minipbrt and converts them in
SceneManager::TransformScene (src/Frontend/Core/SceneManager.cpp:45-246). This loader reads the
subset that conversion accepts and converts it the same way:

- Camera "perspective" (PinholeCamera, Camera.cpp:15-28): position, up (scaled by tan(fov / 2)),
  look direction and right = cross(look, up) from camera-to-world (the inverse of the transform
  current at the Camera directive), right scaled by width / height
  (PathTracingProgramManager.cpp:26).
- Materials matte, plastic, glass, disney, mapped to Disney parameters as Material.cpp:33-107
  does; named materials (MakeNamedMaterial / NamedMaterial) and anonymous ones.
- Textures "imagemap" (PNG or TGA files) bound to Kd / Kt / color; "scale" textures are left
  out as SceneManager.cpp:144-146 does.
- Shape "trianglemesh" (P, indices, optional N and "float uv") and "plymesh" (ASCII or binary
  little-endian PLY with x y z [nx ny nz] [u v | s t], triangle or quad faces). Vertices and
  normals are transformed by the shape's object-to-world matrix as points, as
  TriangleMesh::TriangleMesh does (Shape.cpp:17-40).
- AreaLightSource "diffuse" (L, twosided) bound to the shapes of its attribute block.
- Film x/yresolution, Sampler pixelsamples, Integrator maxdepth; Transform, ConcatTransform,
  Translate, Scale, Rotate, LookAt, Identity, AttributeBegin/End, TransformBegin/End, Include.

minipbrt's own rules are kept where they differ from pbrt-v3's specification: its parameter
defaults (matte Kd and disney color (1, 1, 1)), texture coordinates only as "float uv", PLY
quads split into (0, 1, 3), (2, 3, 1) and larger faces by its ear clipping, and its
single-precision matrix arithmetic (Mat4 translate / rotate / lookAt / inverse) followed by the
frontend's glm float arithmetic for vertices and the camera frame. The arrays this loader
returns equal, bit for bit, what the reference's own SceneManager (built from its sources)
hands to the C ABI through the integration guide's DeviceManager (tests/test_frontend.py).
"""
import math
import os
import re
import struct

import numpy as np

from . import scenes

_TOKEN = re.compile(r'"[^"]*"|\[|\]|[^\s\[\]"#]+|#[^\n]*')


def _tokens(text):
    for m in _TOKEN.finditer(text):
        t = m.group(0)
        if not t.startswith("#"):
            yield t


class _Stream:
    def __init__(self, toks):
        self.toks = list(toks)
        self.i = 0

    def peek(self):
        return self.toks[self.i] if self.i < len(self.toks) else None

    def next(self):
        t = self.toks[self.i]
        self.i += 1
        return t

    def done(self):
        return self.i >= len(self.toks)

    def numbers(self, n):
        out = []
        if self.peek() == "[":
            self.next()
            while self.peek() != "]":
                out.append(float(self.next()))
            self.next()
        else:
            for _ in range(n):
                out.append(float(self.next()))
        return out

    def string(self):
        return self.next().strip('"')

    def params(self):
        """The parameter list after a directive: {name: (type, values)}."""
        out = {}
        while not self.done() and self.peek().startswith('"'):
            decl = self.string().split()
            if len(decl) != 2:
                raise ValueError(f"bad parameter declaration {decl}")
            typ, name = decl
            vals = []
            if self.peek() == "[":
                self.next()
                while self.peek() != "]":
                    vals.append(self.next())
                self.next()
            else:
                vals.append(self.next())
            if typ in ("string", "texture", "bool"):
                vals = [v.strip('"') for v in vals]
                if typ == "bool":
                    vals = [v == "true" for v in vals]
            else:
                vals = [float(v) for v in vals]
            out[name] = (typ, vals)
        return out


F32 = np.float32


def _libm():
    """glibc's single-precision sinf / cosf / tanf, the functions minipbrt and the reference's
    frontend call through std::sin / std::cos / glm::tan on float arguments."""
    import ctypes
    import ctypes.util
    lib = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
    for name in ("sinf", "cosf", "tanf"):
        f = getattr(lib, name)
        f.restype = ctypes.c_float
        f.argtypes = [ctypes.c_float]
    return lib


_LIBM = _libm()


def _f(x):
    return F32(x)


def _v_normalize(v):
    """minipbrt's normalize: v / sqrt((x x + y y) + z z), in float."""
    x, y, z = (_f(c) for c in v)
    n = F32(np.sqrt(F32(F32(x * x + y * y) + z * z)))
    return (x / n, y / n, z / n)


def _v_cross(a, b):
    return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])


class _Mat4:
    """minipbrt's Mat4 (row-major, float) and the operations its parser applies to the current
    transform (Mat4::translate / scale / rotate / lookAt / concatTransform and inverse), in the
    same float operation order, so the transforms equal the reference frontend's bit for bit."""

    def __init__(self, rows=None):
        self.r = [[_f(1.0 if i == j else 0.0) for j in range(4)] for i in range(4)] if rows is None \
            else [[_f(x) for x in row] for row in rows]

    def copy(self):
        return _Mat4(self.r)

    @staticmethod
    def from_column_major(vals):
        # Transform / ConcatTransform arguments are column-major (rows[r][c] = arg[4 c + r])
        return _Mat4([[vals[4 * c + r] for c in range(4)] for r in range(4)])

    def translate(self, v):
        v = [_f(x) for x in v]
        for r in self.r:
            r[3] = r[3] + ((r[0] * v[0] + r[1] * v[1]) + r[2] * v[2])

    def scale(self, v):
        v = [_f(x) for x in v]
        for r in self.r:
            for c in range(3):
                r[c] = r[c] * v[c]

    def rotate(self, degrees, axis):
        ang = F32(F32(_f(degrees) * F32(math.pi)) / F32(180.0))  # degrees_to_radians
        c, s = F32(_LIBM.cosf(float(ang))), F32(_LIBM.sinf(float(ang)))
        ux, uy, uz = _v_normalize(axis)
        k = F32(1.0) - c
        b = [[ux * ux * k + c, ux * uy * k - uz * s, ux * uz * k + uy * s],
             [uy * ux * k + uz * s, uy * uy * k + c, uy * uz * k - ux * s],
             [uz * ux * k - uy * s, uz * uy * k + ux * s, uz * uz * k + c]]
        a = [row[:] for row in self.r]
        for i in range(4):
            for j in range(3):
                self.r[i][j] = (a[i][0] * b[0][j] + a[i][1] * b[1][j]) + a[i][2] * b[2][j]

    def concat(self, m):
        a = [row[:] for row in self.r]
        for i in range(4):
            for j in range(4):
                self.r[i][j] = ((a[i][0] * m.r[0][j] + a[i][1] * m.r[1][j]) + a[i][2] * m.r[2][j]) + \
                    a[i][3] * m.r[3][j]

    def look_at(self, pos, target, up):
        pos, target = [_f(x) for x in pos], [_f(x) for x in target]
        d = _v_normalize([target[k] - pos[k] for k in range(3)])
        x = _v_normalize(_v_cross(_v_normalize(up), d))
        y = _v_normalize(_v_cross(d, x))
        m = _Mat4([[x[0], y[0], d[0], pos[0]], [x[1], y[1], d[1], pos[1]], [x[2], y[2], d[2], pos[2]],
                   [0, 0, 0, 1]])
        self.concat(m.inverse())

    def _d2(self, r0, r1, c0, c1):
        r = self.r
        return r[r0][c0] * r[r1][c1] - r[r0][c1] * r[r1][c0]

    def inverse(self):
        m = self.r
        d = self._d2
        A, B, C, D, E, Fv = d(2, 3, 2, 3), d(2, 3, 1, 3), d(2, 3, 1, 2), d(2, 3, 0, 3), d(2, 3, 0, 2), d(2, 3, 0, 1)
        G, H, I, J, K, L = d(1, 3, 2, 3), d(1, 3, 1, 3), d(1, 3, 1, 2), d(1, 3, 0, 3), d(1, 3, 0, 2), d(1, 3, 0, 1)
        M, N, O, P, Q, R = d(1, 2, 2, 3), d(1, 2, 1, 3), d(1, 2, 1, 2), d(1, 2, 0, 3), d(1, 2, 0, 2), d(1, 2, 0, 1)

        def t(a, x, b, y, c, z):
            return (a * x - b * y) + c * z
        inv = [[+t(m[1][1], A, m[1][2], B, m[1][3], C), -t(m[0][1], A, m[0][2], B, m[0][3], C),
                +t(m[0][1], G, m[0][2], H, m[0][3], I), -t(m[0][1], M, m[0][2], N, m[0][3], O)],
               [-t(m[1][0], A, m[1][2], D, m[1][3], E), +t(m[0][0], A, m[0][2], D, m[0][3], E),
                -t(m[0][0], G, m[0][2], J, m[0][3], K), +t(m[0][0], M, m[0][2], P, m[0][3], Q)],
               [+t(m[1][0], B, m[1][1], D, m[1][3], Fv), -t(m[0][0], B, m[0][1], D, m[0][3], Fv),
                +t(m[0][0], H, m[0][1], J, m[0][3], L), -t(m[0][0], N, m[0][1], P, m[0][3], R)],
               [-t(m[1][0], C, m[1][1], E, m[1][2], Fv), +t(m[0][0], C, m[0][1], E, m[0][2], Fv),
                -t(m[0][0], I, m[0][1], K, m[0][2], L), +t(m[0][0], O, m[0][1], Q, m[0][2], R)]]
        det = ((m[0][0] * inv[0][0] + m[0][1] * inv[1][0]) + m[0][2] * inv[2][0]) + m[0][3] * inv[3][0]
        inv_det = F32(1.0) / det
        return _Mat4([[x * inv_det for x in row] for row in inv])

    def apply(self, P, w):
        """The reference frontend's TransformVec3(transpose(make_mat4(rows)), p, w): glm's
        mat4 * vec4, (r0 x + r1 y) + (r2 z + r3 w) per row, in float, for an (n, 3) array."""
        P = np.asarray(P, F32)
        x, y, z = P[:, 0], P[:, 1], P[:, 2]
        wf = F32(w)
        out = np.empty((len(P), 3), F32)
        for i in range(3):
            r = self.r[i]
            out[:, i] = (r[0] * x + r[1] * y) + (r[2] * z + r[3] * wf)
        return out

    def apply4(self, v):
        """glm's mat4 * vec4 for one 4-vector (float)."""
        v = [_f(c) for c in v]
        return [(r[0] * v[0] + r[1] * v[1]) + (r[2] * v[2] + r[3] * v[3]) for r in self.r]


def _glm_normalize4(v):
    """glm::normalize of a vec4: v * (1 / sqrt((x x + y y) + (z z + w w)))."""
    dot = (v[0] * v[0] + v[1] * v[1]) + (v[2] * v[2] + v[3] * v[3])
    k = F32(1.0) / F32(np.sqrt(dot))
    return [c * k for c in v]


def _glm_normalize3(v):
    """glm::normalize of a vec3: v * (1 / sqrt((x x + y y) + z z))."""
    dot = (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]
    k = F32(1.0) / F32(np.sqrt(dot))
    return [c * k for c in v]


def _camera_frame(c2w, fov, W, H):
    """PinholeCamera(fov, cameraToWorld) (Camera.cpp:15-28) and the aspect scaling of
    PathTracingProgramManager.cpp:28, in the reference frontend's float operation order."""
    pos = c2w.apply4([0, 0, 0, 1])[:3]
    up = _glm_normalize4(c2w.apply4([0, 1, 0, 0]))[:3]
    look = _glm_normalize3(c2w.apply4([0, 0, 1, 0])[:3])
    half = F32(_f(fov) / F32(2.0))
    rad = F32(np.float64(half * F32(math.pi)) / 180.0)  # AngleToRadian: (a * PI) / 180.0
    t = F32(_LIBM.tanf(float(rad)))
    up = [t * c for c in up]
    right = [look[1] * up[2] - up[1] * look[2], look[2] * up[0] - up[2] * look[0],
             look[0] * up[1] - up[0] * look[1]]  # glm::cross(look, up)
    aspect = F32(F32(W) / F32(H))
    right = [c * aspect for c in right]
    return {"pos": np.array(pos, F32), "look_at": np.array(look, F32), "up": np.array(up, F32),
            "right": np.array(right, F32)}


def _color(params, name, default):
    if name in params:
        typ, v = params[name]
        if typ in ("rgb", "color", "spectrum") and len(v) == 3:
            return [float(x) for x in v]
        if typ == "float":
            return [float(v[0])] * 3
    return list(default)


def _float(params, name, default):
    return float(params[name][1][0]) if name in params else default


def _tex(params, name, tex_index):
    if name in params and params[name][0] == "texture":
        return tex_index.get(params[name][1][0], -1)
    return -1


def material_to_disney(kind, params, tex_index):
    """Material.cpp:33-107 (Disney(...) constructors) with minipbrt's parameter defaults (which
    the reference reads; a texture-bound colour keeps its default value)."""
    if kind == "matte":
        m = scenes.matte(tuple(_color(params, "Kd", (1.0, 1.0, 1.0))))
        m["texture"] = _tex(params, "Kd", tex_index)
    elif kind == "plastic":
        kd = np.array(_color(params, "Kd", (0.25, 0.25, 0.25)), np.float32)
        ks = np.array(_color(params, "Ks", (0.25, 0.25, 0.25)), np.float32)
        m = scenes.disney(tuple(kd + ks), metallic=float(np.clip(np.linalg.norm(ks), 0.0, 1.0)),
                          roughness=_float(params, "roughness", 0.1), specular=0.0,
                          specular_tint=0.0, eta=1.5, trans=0.0, sheen_tint=0.5)
        m["texture"] = _tex(params, "Kd", tex_index)
    elif kind == "glass":
        kr = np.array(_color(params, "Kr", (1, 1, 1)), np.float32)
        kt = np.array(_color(params, "Kt", (1, 1, 1)), np.float32)
        m = scenes.disney(tuple((kr + kt) / 2.0), metallic=0.0, roughness=0.01, specular=0.5,
                          specular_tint=0.0, eta=_float(params, "eta", 1.5), trans=1.0,
                          sheen_tint=0.5)
        m["texture"] = _tex(params, "Kt", tex_index)
    elif kind == "disney":
        m = scenes.disney(tuple(_color(params, "color", (1.0, 1.0, 1.0))),
                          metallic=_float(params, "metallic", 0.0),
                          roughness=_float(params, "roughness", 0.5), specular=0.0,
                          specular_tint=_float(params, "speculartint", 0.0),
                          eta=_float(params, "eta", 1.5), trans=_float(params, "spectrans", 0.0),
                          subsurface=0.0, anisotropic=_float(params, "anisotropic", 0.0),
                          sheen=_float(params, "sheen", 0.0), sheen_tint=_float(params, "sheentint", 0.5),
                          clearcoat=_float(params, "clearcoat", 0.0),
                          clearcoat_gloss=_float(params, "clearcoatgloss", 1.0))
        m["texture"] = _tex(params, "color", tex_index)
    else:
        raise ValueError(f"unsupported material type {kind!r} (the reference accepts matte, "
                         "plastic, glass, disney)")
    return m


def read_ply(path):
    """(P, N or None, UV or None, triangles) of an ASCII or binary little-endian PLY mesh."""
    with open(path, "rb") as f:
        data = f.read()
    end = data.index(b"end_header") + len(b"end_header")
    while data[end:end + 1] in (b"\r", b"\n"):
        end += 1
        if data[end - 1:end] == b"\n":
            break
    header = data[:end].decode("ascii", "replace").splitlines()
    fmt, elements = None, []
    for line in header:
        w = line.split()
        if not w:
            continue
        if w[0] == "format":
            fmt = w[1]
        elif w[0] == "element":
            elements.append([w[1], int(w[2]), []])
        elif w[0] == "property":
            elements[-1][2].append(w[1:])
    types = {"char": "b", "int8": "b", "uchar": "B", "uint8": "B", "short": "h", "int16": "h",
             "ushort": "H", "uint16": "H", "int": "i", "int32": "i", "uint": "I", "uint32": "I",
             "float": "f", "float32": "f", "double": "d", "float64": "d"}
    body = data[end:]
    verts, faces = None, []
    if fmt == "ascii":
        words = body.split()
        k = 0
        for name, count, props in elements:
            rows = []
            for _ in range(count):
                row = []
                for p in props:
                    if p[0] == "list":
                        n = int(words[k]); k += 1
                        row.append([float(x) for x in words[k:k + n]]); k += n
                    else:
                        row.append(float(words[k])); k += 1
                rows.append(row)
            if name == "vertex":
                verts = (props, rows)
            elif name == "face":
                faces = [r[0] for r in rows]
    elif fmt == "binary_little_endian":
        k = 0
        for name, count, props in elements:
            if all(p[0] != "list" for p in props):
                st = struct.Struct("<" + "".join(types[p[0]] for p in props))
                arr = np.frombuffer(body, np.dtype([(p[1], "<" + st.format[1 + i])
                                                    for i, p in enumerate(props)]), count, k)
                k += st.size * count
                if name == "vertex":
                    verts = (props, arr)
            else:
                rows = []
                for _ in range(count):
                    row = []
                    for p in props:
                        if p[0] == "list":
                            cs = struct.Struct("<" + types[p[1]])
                            n, = cs.unpack_from(body, k); k += cs.size
                            es = struct.Struct("<" + types[p[2]] * n)
                            row.append(list(es.unpack_from(body, k))); k += es.size
                        else:
                            s1 = struct.Struct("<" + types[p[0]])
                            row.append(s1.unpack_from(body, k)[0]); k += s1.size
                    rows.append(row)
                if name == "face":
                    idx = [i for i, p in enumerate(props) if p[0] == "list"][0]
                    faces = [r[idx] for r in rows]
    else:
        raise ValueError(f"unsupported PLY format {fmt!r}")
    props, rows = verts
    names = [p[-1] for p in props]

    def col(n):
        if isinstance(rows, np.ndarray):
            return np.asarray(rows[n], np.float64)
        return np.array([r[names.index(n)] for r in rows], np.float64)

    P = np.stack([col("x"), col("y"), col("z")], 1)
    N = np.stack([col("nx"), col("ny"), col("nz")], 1) if "nx" in names else None
    UV = None
    for a, b in (("u", "v"), ("s", "t"), ("texture_u", "texture_v")):
        if a in names and b in names:
            UV = np.stack([col(a), col(b)], 1)
    tris = []
    for f in faces:
        tris.extend(triangulate_polygon([int(x) for x in f], P))
    return P, N, UV, np.array(tris, np.int64).reshape(-1, 3)


def _angle_at_vert(i, pts, prev, nxt):
    """minipbrt's angle_at_vert: the angle at a remaining polygon vertex, 10000 when reflex."""
    x = pts[nxt[i]] - pts[i]
    x = (x / np.float32(np.sqrt(np.float32(x @ x)))).astype(np.float32)
    y = np.array([-x[1], x[0]], np.float32)
    p = (pts[prev[i]] - pts[i]).astype(np.float32)
    a = float(np.arctan2(np.float32(p @ y), np.float32(p @ x)))
    return 10000.0 if a <= 0.0 or a >= math.pi else a


def triangulate_polygon(idx, P):
    """The triangles minipbrt makes of a PLY face (miniply triangulate_polygon): a triangle as is,
    a quad as (0, 1, 3), (2, 3, 1), larger polygons by ear clipping at the sharpest remaining
    vertex of the face projected on its plane."""
    n = len(idx)
    if n < 3:
        return []
    if n == 3:
        return [idx]
    if n == 4:
        return [[idx[0], idx[1], idx[3]], [idx[2], idx[3], idx[1]]]
    V = np.asarray(P, np.float32)

    def unit(v):
        return (v / np.float32(np.sqrt(np.float32(v @ v)))).astype(np.float32)

    o = V[idx[0]]
    u = unit(V[idx[1]] - o)
    nrm = unit(np.cross(u, unit(V[idx[n - 1]] - o)).astype(np.float32))
    v = unit(np.cross(nrm, u).astype(np.float32))
    pts = [np.zeros(2, np.float32)] + [np.array([(V[idx[i]] - o) @ u, (V[idx[i]] - o) @ v], np.float32)
                                       for i in range(1, n)]
    nxt = [(i + 1) % n for i in range(n)]
    prev = [(i - 1) % n for i in range(n)]
    first, out = 0, []
    while n > 3:
        best, best_a = first, _angle_at_vert(first, pts, prev, nxt)
        i = nxt[first]
        while i != first:
            a = _angle_at_vert(i, pts, prev, nxt)
            if a < best_a:
                best, best_a = i, a
            i = nxt[i]
        ni, pi = nxt[best], prev[best]
        out.append([idx[best], idx[ni], idx[pi]])
        if best == first:
            first = ni
        nxt[pi], prev[ni] = ni, pi
        n -= 1
    out.append([idx[first], idx[nxt[first]], idx[prev[first]]])
    return out


def load(path, width=None, height=None):
    """Read a pbrt-v3 file into a scenes.Scene (the SceneManager fields, flattened)."""
    base = os.path.dirname(os.path.abspath(path))
    state = {"ctm": _Mat4(), "material": None, "light": None, "reverse": False}
    stack, tstack = [], []
    named_mats, mats, tex_index, textures = {}, [], {}, []
    meshes = []          # (P, N, UV, tris, material, light)
    lights = []          # (L, two_sided)
    cam = {"c2w": None, "fov": 90.0}
    film = {"x": 640, "y": 480}
    opts = {"spp": 16, "maxdepth": 5}

    def current_material():
        if state["material"] is None:
            mats.append(scenes.matte((0.5, 0.5, 0.5)))
            state["material"] = len(mats) - 1
        return state["material"]

    def run(text, cwd):
        s = _Stream(_tokens(text))
        while not s.done():
            d = s.next()
            if d == "Transform":
                state["ctm"] = _Mat4.from_column_major(s.numbers(16))
            elif d == "ConcatTransform":
                state["ctm"].concat(_Mat4.from_column_major(s.numbers(16)))
            elif d == "Translate":
                state["ctm"].translate(s.numbers(3))
            elif d == "Scale":
                state["ctm"].scale(s.numbers(3))
            elif d == "Rotate":
                v = s.numbers(4)
                state["ctm"].rotate(v[0], v[1:])
            elif d == "LookAt":
                v = s.numbers(9)
                state["ctm"].look_at(v[0:3], v[3:6], v[6:9])
            elif d == "Identity":
                state["ctm"] = _Mat4()
            elif d == "Camera":
                kind = s.string()
                p = s.params()
                if kind != "perspective":
                    raise ValueError(f"unsupported camera {kind!r} (the reference accepts perspective)")
                cam["c2w"] = state["ctm"].inverse()
                cam["fov"] = _float(p, "fov", 90.0)
            elif d == "Film":
                s.string()
                p = s.params()
                film["x"] = int(_float(p, "xresolution", 640))
                film["y"] = int(_float(p, "yresolution", 480))
            elif d == "Sampler":
                s.string()
                p = s.params()
                opts["spp"] = int(_float(p, "pixelsamples", 16))
            elif d == "Integrator":
                s.string()
                p = s.params()
                opts["maxdepth"] = int(_float(p, "maxdepth", 5))
            elif d in ("PixelFilter", "Accelerator", "CoordinateSystem", "CoordSysTransform",
                       "ColorSpace", "Option"):
                if d in ("CoordinateSystem", "CoordSysTransform"):
                    s.string()
                else:
                    s.string()
                    s.params()
            elif d == "WorldBegin":
                state["ctm"] = _Mat4()
            elif d == "WorldEnd":
                pass
            elif d == "AttributeBegin":
                stack.append(dict(state, ctm=state["ctm"].copy()))
            elif d == "AttributeEnd":
                state.update(stack.pop())
            elif d == "TransformBegin":
                tstack.append(state["ctm"].copy())
            elif d == "TransformEnd":
                state["ctm"] = tstack.pop()
            elif d == "ReverseOrientation":
                state["reverse"] = not state["reverse"]
            elif d == "Material":
                kind = s.string()
                mats.append(material_to_disney(kind, s.params(), tex_index))
                state["material"] = len(mats) - 1
            elif d == "MakeNamedMaterial":
                name = s.string()
                p = s.params()
                kind = p.pop("type")[1][0]
                mats.append(material_to_disney(kind, p, tex_index))
                named_mats[name] = len(mats) - 1
            elif d == "NamedMaterial":
                state["material"] = named_mats[s.string()]
            elif d == "Texture":
                name = s.string()
                s.string()
                kind = s.string()
                p = s.params()
                if kind == "scale":
                    continue  # SceneManager.cpp:144-146 leaves scale textures out ("TBD")
                if kind != "imagemap":
                    raise ValueError(f"unsupported texture {kind!r} (the reference accepts imagemap)")
                textures.append(_load_image(os.path.join(cwd, p["filename"][1][0])))
                tex_index[name] = len(textures) - 1
            elif d == "AreaLightSource":
                kind = s.string()
                p = s.params()
                if kind != "diffuse":
                    raise ValueError("only diffuse area lights")
                lights.append((_color(p, "L", (1, 1, 1)),
                               bool(p["twosided"][1][0]) if "twosided" in p else False))
                state["light"] = len(lights) - 1
            elif d == "LightSource":
                s.string()
                s.params()  # point/spot/infinite lights: the reference converts area lights only
            elif d == "Shape":
                kind = s.string()
                p = s.params()
                if kind == "trianglemesh":
                    P = np.array(p["P"][1], np.float64).reshape(-1, 3)
                    tris = np.array(p["indices"][1], np.int64).reshape(-1, 3)
                    N = np.array(p["N"][1], np.float64).reshape(-1, 3) if "N" in p else None
                    # minipbrt reads texture coordinates only as "float uv" (a "point2 uv" or
                    # "st" list is not a float parameter there and is dropped)
                    UV = np.array(p["uv"][1], np.float64).reshape(-1, 2) \
                        if "uv" in p and p["uv"][0] == "float" else None
                elif kind == "plymesh":
                    P, N, UV, tris = read_ply(os.path.join(cwd, p["filename"][1][0]))
                else:
                    raise ValueError(f"unsupported shape {kind!r} (the reference accepts triangle meshes)")
                meshes.append((P, N, UV, tris, state["ctm"].copy(), current_material(), state["light"]))
            elif d == "Include":
                inc = os.path.join(cwd, s.string())
                with open(inc) as f:
                    run(f.read(), os.path.dirname(inc))
            elif d in ("MakeNamedMedium", "MediumInterface", "ObjectBegin", "ObjectEnd",
                       "ObjectInstance"):
                raise ValueError(f"unsupported directive {d}")
            else:
                raise ValueError(f"unknown directive {d!r}")

    with open(path) as f:
        run(f.read(), base)
    if cam["c2w"] is None:
        raise ValueError("the scene has no camera")
    W = width or film["x"]
    H = height or film["y"]
    # meshes -> flattened arrays (SceneManager mesh order; light meshes keep their triangles
    # contiguous, which every mesh does)
    Vs, Ns, UVs, Is, Ms, flags = [], [], [], [], [], []
    light_ranges = {}
    nv = nt = 0
    has_n = any(m[1] is not None for m in meshes)
    has_uv = any(m[2] is not None for m in meshes)
    for P, N, UV, tris, o2w, mat, light in meshes:
        Vs.append(o2w.apply(P, 1.0))
        if has_n:
            if N is not None:
                Ns.append(o2w.apply(N, 1.0))  # as points (Shape.cpp:39)
            else:
                Ns.append(np.zeros((len(P), 3)))
        if has_uv:
            UVs.append(UV if UV is not None else np.zeros((len(P), 2)))
        Is.append(tris + nv)
        Ms.append(np.full(len(tris), mat, np.uint32))
        flags.append(np.full(len(tris), 1 if N is not None else 0, np.uint32))
        if light is not None:
            if light in light_ranges:
                raise ValueError("one area light bound to several meshes is not supported")
            light_ranges[light] = (nt, len(tris))
        nv += len(P)
        nt += len(tris)
    larr = np.zeros(len(light_ranges), scenes.LIGHT)
    for k, (li, (first, count)) in enumerate(sorted(light_ranges.items())):
        L, two = lights[li]
        larr[k]["L"] = L
        larr[k]["two_sided"] = int(two)
        larr[k]["first_tri"] = first
        larr[k]["tri_count"] = count
    camera = _camera_frame(cam["c2w"], cam["fov"], W, H)
    sc = scenes.Scene(os.path.basename(path), np.concatenate(Vs).astype(np.float32),
                      np.concatenate(Is).astype(np.uint32), np.concatenate(Ms),
                      np.array(mats) if mats else np.array([scenes.matte((0.5, 0.5, 0.5))]), larr,
                      N=np.concatenate(Ns).astype(np.float32) if has_n else None,
                      tri_flags=np.concatenate(flags) if has_n else None, camera=camera,
                      width=W, height=H, spp=opts["spp"], max_depth=opts["maxdepth"])
    if has_uv:
        sc.UV = np.concatenate(UVs).astype(np.float32)
    sc.textures = textures
    return sc


def _load_image(path):
    """RGBA8 (h, w, 4) of a PNG (8-bit RGB, RGBA or palette) or TGA file, first row = top.
    The reference decodes any format with stbi_load (Texture.cpp:13-16); images in other formats
    are read from a PNG file of the same name next to them when there is one."""
    from .png import read_png_any
    with open(path, "rb") as f:
        magic = f.read(8)
    if path.lower().endswith(".tga"):
        return read_tga(path)
    if magic != b"\x89PNG\r\n\x1a\n":
        alt = os.path.splitext(path)[0] + ".png"
        if os.path.exists(alt):
            path = alt
        else:
            raise ValueError(f"{path}: only PNG images can be read (no PNG copy next to it)")
    return read_png_any(path)


def read_tga(path):
    """RGBA8 (h, w, 4) of a truecolour TGA file (types 2 and 10: uncompressed and run-length
    encoded, 24 or 32 bits), first row = the top of the image."""
    with open(path, "rb") as f:
        data = f.read()
    idlen, cmtype, itype = data[0], data[1], data[2]
    w, h = struct.unpack("<HH", data[12:16])
    bpp, desc = data[16], data[17]
    if itype not in (2, 10) or bpp not in (24, 32) or cmtype != 0:
        raise ValueError(f"{path}: only truecolour TGA (24/32-bit, raw or RLE)")
    n = bpp // 8
    pos = 18 + idlen
    count = w * h
    if itype == 2:
        px = np.frombuffer(data, np.uint8, count * n, pos).reshape(count, n)
    else:
        px = np.empty((count, n), np.uint8)
        k = 0
        while k < count:
            head = data[pos]
            pos += 1
            run = (head & 0x7F) + 1
            if head & 0x80:
                px[k:k + run] = np.frombuffer(data, np.uint8, n, pos)
                pos += n
            else:
                px[k:k + run] = np.frombuffer(data, np.uint8, run * n, pos).reshape(run, n)
                pos += run * n
            k += run
    img = np.full((count, 4), 255, np.uint8)
    img[:, 0], img[:, 1], img[:, 2] = px[:, 2], px[:, 1], px[:, 0]
    if n == 4:
        img[:, 3] = px[:, 3]
    img = img.reshape(h, w, 4)
    if not (desc & 0x20):  # origin at the bottom left
        img = img[::-1]
    return np.ascontiguousarray(img)
