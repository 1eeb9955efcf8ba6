"""pbrt-v3 ingestion (wayland_b200.pbrt) against the reference's conversion rules
(SceneManager.cpp, Material.cpp, Camera.cpp, Shape.cpp). Host code, no GPU."""
import math
import os

import numpy as np
import pytest

from wayland_b200 import pbrt
from pbrt_fixture import write_scene

REF_CBOX = os.path.join(os.environ.get("WL_REFERENCE_ROOT", "/root/reference"),
                        "scene", "cornell-box", "cbox.pbrt")


def test_synthetic_scene(tmp_path):
    sc = pbrt.load(str(write_scene(tmp_path)))
    assert (sc.width, sc.height, sc.spp, sc.max_depth) == (40, 32, 4, 6)
    # floor 2 + box 12 (6 quads) + disney tetrahedron 3 + glass 1 + light 2
    assert sc.num_tris == 20
    assert len(sc.lights) == 1 and sc.lights[0]["first_tri"] == 18 and sc.lights[0]["tri_count"] == 2
    assert tuple(sc.lights[0]["L"]) == (8, 7, 6) and sc.lights[0]["two_sided"] == 0
    # materials in creation order: floor (textured matte), shiny (plastic), disney, glass, light
    m = sc.mats
    # a texture-bound Kd keeps minipbrt's default value (1, 1, 1), which the reference reads
    assert m[0]["texture"] == 0 and np.allclose(m[0]["color"], 1.0)
    assert np.allclose(m[1]["color"], [0.5, 0.4, 0.3]) and math.isclose(m[1]["metallic"], math.sqrt(0.12), rel_tol=1e-6)
    assert math.isclose(m[1]["roughness"], 0.05, rel_tol=1e-6) and m[1]["texture"] == -1
    assert np.allclose(m[2]["color"], [0.2, 0.5, 0.8]) and math.isclose(m[2]["trans"], 0.2, rel_tol=1e-6)
    assert m[2]["specular"] == 0 and math.isclose(m[2]["clearcoat"], 0.5)
    assert m[3]["trans"] == 1 and math.isclose(m[3]["eta"], 1.33, rel_tol=1e-6) and math.isclose(m[3]["roughness"], 0.01, rel_tol=1e-6)
    assert list(sc.tri_material) == [0, 0] + [1] * 12 + [2] * 3 + [3] + [4, 4]
    # the box is rotated and lifted: its vertices stay within the rotated box around y = 0.5
    box = sc.V[sc.I[2:14].reshape(-1)]
    assert np.allclose(box[:, 1].min(), 0.1, atol=1e-5) and np.allclose(box[:, 1].max(), 0.9, atol=1e-5)
    # normals only on the tetrahedron, transformed as points (Shape.cpp:39)
    assert list(sc.tri_flags) == [0] * 14 + [1] * 3 + [0] * 3
    assert np.allclose(sc.N[sc.I[14, 0]], [-1 + 1.2, 0.4, 0.3])
    # texture coordinates and the texture itself (16 x 16 RGBA8)
    assert sc.UV is not None and np.allclose(sc.UV[sc.I[0]], [[0, 0], [4, 4], [4, 0]])
    assert len(sc.textures) == 1 and sc.textures[0].shape == (16, 16, 4)
    # camera (Camera.cpp:15-28, PathTracingProgramManager.cpp:26)
    eye, target = np.array([0, 1, 4.5]), np.array([0, 0.7, 0])
    d = (target - eye) / np.linalg.norm(target - eye)
    assert np.allclose(sc.camera["pos"], eye, atol=1e-6)
    assert np.allclose(sc.camera["look_at"], d, atol=1e-6)
    t = math.tan(math.radians(20))
    assert math.isclose(float(np.linalg.norm(sc.camera["up"])), t, rel_tol=1e-5)
    assert np.allclose(sc.camera["right"], np.cross(sc.camera["look_at"], sc.camera["up"]) * 40 / 32, atol=1e-6)


def test_unsupported_inputs(tmp_path):
    p = tmp_path / "bad.pbrt"
    p.write_text('Camera "orthographic"\nWorldBegin\nWorldEnd\n')
    with pytest.raises(ValueError, match="perspective"):
        pbrt.load(str(p))
    p.write_text('Camera "perspective"\nWorldBegin\nShape "sphere" "float radius" [ 1 ]\nWorldEnd\n')
    with pytest.raises(ValueError, match="sphere"):
        pbrt.load(str(p))
    p.write_text('Camera "perspective"\nWorldBegin\nMaterial "metal"\nWorldEnd\n')
    with pytest.raises(ValueError, match="metal"):
        pbrt.load(str(p))


@pytest.mark.skipif(not os.path.exists(REF_CBOX), reason="needs the reference's scene files")
def test_reference_cornell_box():
    """The reference's own scene/cornell-box/cbox.pbrt (available where the reference tree is)."""
    sc = pbrt.load(REF_CBOX)
    assert sc.num_tris == 36 and (sc.width, sc.height) == (1024, 1024)
    assert len(sc.lights) == 1 and tuple(sc.lights[0]["L"]) == (50, 35, 15)
    assert np.allclose(sc.camera["pos"], [0, 1, 6.8])
    assert np.allclose(sc.camera["look_at"], [0, 0, -1])
