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
- Shape "trianglemesh" (P, indices, optional N and uv/st) and "plymesh" (ASCII or binary
  little-endian PLY with x y z [nx ny nz] [u v | s t], triangle or quad faces). Vertices and
  normals are transformed by the shape's object-to-world matrix as points, as
  TriangleMesh::TriangleMesh does (Shape.cpp:17-40).
- AreaLightSource "diffuse" (L, twosided) bound to the shapes of its attribute block.
- Film x/yresolution, Sampler pixelsamples, Integrator maxdepth; Transform, ConcatTransform,
  Translate, Scale, Rotate, LookAt, Identity, AttributeBegin/End, TransformBegin/End, Include.
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


def _translate(d):
    m = np.eye(4)
    m[:3, 3] = d
    return m


def _scale(s):
    return np.diag([s[0], s[1], s[2], 1.0])


def _rotate(angle, axis):
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    s, c = math.sin(math.radians(angle)), math.cos(math.radians(angle))
    x, y, z = a
    m = np.eye(4)
    m[:3, :3] = [[x * x + (1 - x * x) * c, x * y * (1 - c) - z * s, x * z * (1 - c) + y * s],
                 [x * y * (1 - c) + z * s, y * y + (1 - y * y) * c, y * z * (1 - c) - x * s],
                 [x * z * (1 - c) - y * s, y * z * (1 - c) + x * s, z * z + (1 - z * z) * c]]
    return m


def _look_at(eye, look, up):
    """World-to-camera of pbrt-v3's LookAt (camera looks along +z, x = normalize(up) x dir)."""
    eye, look, up = (np.asarray(v, np.float64) for v in (eye, look, up))
    d = look - eye
    d = d / np.linalg.norm(d)
    right = np.cross(up / np.linalg.norm(up), d)
    right = right / np.linalg.norm(right)
    new_up = np.cross(d, right)
    c2w = np.eye(4)
    c2w[:3, 0], c2w[:3, 1], c2w[:3, 2], c2w[:3, 3] = right, new_up, d, eye
    return np.linalg.inv(c2w)


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
    """Material.cpp:33-107 (Disney(...) constructors) with pbrt-v3's parameter defaults."""
    if kind == "matte":
        m = scenes.matte(tuple(_color(params, "Kd", (0.5, 0.5, 0.5))))
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
        m = scenes.disney(tuple(_color(params, "color", (0.5, 0.5, 0.5))),
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
        f = [int(x) for x in f]
        for j in range(1, len(f) - 1):
            tris.append([f[0], f[j], f[j + 1]])
    return P, N, UV, np.array(tris, np.int64).reshape(-1, 3)


def load(path, width=None, height=None):
    """Read a pbrt-v3 file into a scenes.Scene (the SceneManager fields, flattened)."""
    base = os.path.dirname(os.path.abspath(path))
    state = {"ctm": np.eye(4), "material": None, "light": None, "reverse": False}
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
                state["ctm"] = np.array(s.numbers(16), np.float64).reshape(4, 4).T
            elif d == "ConcatTransform":
                state["ctm"] = state["ctm"] @ np.array(s.numbers(16), np.float64).reshape(4, 4).T
            elif d == "Translate":
                state["ctm"] = state["ctm"] @ _translate(s.numbers(3))
            elif d == "Scale":
                state["ctm"] = state["ctm"] @ _scale(s.numbers(3))
            elif d == "Rotate":
                v = s.numbers(4)
                state["ctm"] = state["ctm"] @ _rotate(v[0], v[1:])
            elif d == "LookAt":
                v = s.numbers(9)
                state["ctm"] = state["ctm"] @ _look_at(v[0:3], v[3:6], v[6:9])
            elif d == "Identity":
                state["ctm"] = np.eye(4)
            elif d == "Camera":
                kind = s.string()
                p = s.params()
                if kind != "perspective":
                    raise ValueError(f"unsupported camera {kind!r} (the reference accepts perspective)")
                cam["c2w"] = np.linalg.inv(state["ctm"])
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
                state["ctm"] = np.eye(4)
            elif d == "WorldEnd":
                pass
            elif d == "AttributeBegin":
                stack.append(dict(state))
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
                    uvk = "uv" if "uv" in p else ("st" if "st" in p else None)
                    UV = np.array(p[uvk][1], np.float64).reshape(-1, 2) if uvk else None
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
        Ph = np.concatenate([P, np.ones((len(P), 1))], 1) @ o2w.T
        Vs.append(Ph[:, :3])
        if has_n:
            if N is not None:
                Nh = np.concatenate([N, np.ones((len(N), 1))], 1) @ o2w.T  # as points (Shape.cpp:39)
                Ns.append(Nh[:, :3])
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
    c2w = cam["c2w"]
    pos = c2w @ np.array([0, 0, 0, 1.0])
    up = c2w @ np.array([0, 1.0, 0, 0])
    look = c2w @ np.array([0, 0, 1.0, 0])
    up = up[:3] / np.linalg.norm(up[:3]) * math.tan(math.radians(cam["fov"] / 2))
    look = look[:3] / np.linalg.norm(look[:3])
    right = np.cross(look, up) * (W / H)
    camera = {"pos": pos[:3].astype(np.float32), "look_at": look.astype(np.float32),
              "up": up.astype(np.float32), "right": right.astype(np.float32)}
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
