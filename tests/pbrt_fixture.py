"""A small pbrt-v3 scene written by the tests (trianglemesh, binary PLY, named and anonymous
materials of every kind the reference converts, an imagemap texture, a transformed shape and a
diffuse area light)."""
import struct

import numpy as np

from wayland_b200.png import write_png
from wayland_b200.scenes import checker_texture

SCENE = """# test scene
LookAt 0 1 4.5  0 0.7 0  0 1 0
Camera "perspective" "float fov" [ 40 ]
Film "image" "integer xresolution" [ 40 ] "integer yresolution" [ 32 ]
    "string filename" [ "out.png" ]
Sampler "random" "integer pixelsamples" [ 4 ]
Integrator "path" "integer maxdepth" [ 6 ]
WorldBegin
Texture "checks" "spectrum" "imagemap" "string filename" [ "tex.png" ]
Texture "scaled" "spectrum" "scale" "texture tex1" "checks" "float tex2" [ 0.5 ]
MakeNamedMaterial "floor" "string type" [ "matte" ] "texture Kd" "checks"
MakeNamedMaterial "shiny" "string type" [ "plastic" ] "rgb Kd" [ 0.3 0.2 0.1 ]
    "rgb Ks" [ 0.2 0.2 0.2 ] "float roughness" [ 0.05 ]
NamedMaterial "floor"
Shape "trianglemesh" "point3 P" [ -3 0 -3  3 0 -3  3 0 3  -3 0 3 ]
    "integer indices" [ 0 2 1 0 3 2 ] "float uv" [ 0 0 4 0 4 4 0 4 ]
AttributeBegin
  Translate 0 0.5 0
  Rotate 30 0 1 0
  NamedMaterial "shiny"
  Shape "plymesh" "string filename" [ "box.ply" ]
AttributeEnd
AttributeBegin
  Translate 1.2 0.4 0.3
  Material "disney" "rgb color" [ 0.2 0.5 0.8 ] "float metallic" [ 0.3 ] "float roughness" [ 0.4 ]
      "float spectrans" [ 0.2 ] "float clearcoat" [ 0.5 ]
  Shape "trianglemesh" "point3 P" [ -0.3 0 0  0.3 0 0  0 0.6 0  0 0 0.3 ]
      "integer indices" [ 0 1 2  1 3 2  3 0 2 ] "normal N" [ -1 0 0  1 0 0  0 1 0  0 0 1 ]
AttributeEnd
AttributeBegin
  Material "glass" "float eta" [ 1.33 ]
  Shape "trianglemesh" "point3 P" [ -1.5 0.01 0.5  -0.9 0.01 0.5  -1.2 0.8 0.8 ]
      "integer indices" [ 0 1 2 ]
AttributeEnd
AttributeBegin
  AreaLightSource "diffuse" "rgb L" [ 8 7 6 ]
  Material "matte" "rgb Kd" [ 0 0 0 ]
  Shape "trianglemesh" "point3 P" [ -0.5 2.5 -0.5  0.5 2.5 -0.5  0.5 2.5 0.5  -0.5 2.5 0.5 ]
      "integer indices" [ 0 1 2 0 2 3 ]
AttributeEnd
WorldEnd
"""


def box_ply(path, half=0.4):
    """A box as a binary little-endian PLY with quad faces."""
    h = half
    P = np.array([[-h, -h, -h], [h, -h, -h], [h, h, -h], [-h, h, -h],
                  [-h, -h, h], [h, -h, h], [h, h, h], [-h, h, h]], np.float32)
    F = [[0, 3, 2, 1], [4, 5, 6, 7], [0, 1, 5, 4], [2, 3, 7, 6], [1, 2, 6, 5], [0, 4, 7, 3]]
    head = ("ply\nformat binary_little_endian 1.0\nelement vertex 8\nproperty float x\n"
            "property float y\nproperty float z\nelement face 6\n"
            "property list uchar int vertex_indices\nend_header\n").encode()
    body = P.tobytes() + b"".join(struct.pack("<B4i", 4, *f) for f in F)
    with open(path, "wb") as f:
        f.write(head + body)
    return P


def write_scene(dirpath):
    write_png(dirpath / "tex.png", checker_texture(16), flip=False)
    box_ply(dirpath / "box.ply")
    path = dirpath / "test.pbrt"
    path.write_text(SCENE)
    return path
