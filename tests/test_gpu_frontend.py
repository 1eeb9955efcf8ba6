"""The drop-in path end to end on the GPU: the reference's own frontend (minipbrt + SceneManager
compiled from the reference's sources into oracle/_ref/wl_frontend) parses the test scene (every
material kind the reference converts, a PLY mesh, rotated and translated shapes, vertex normals,
an imagemap texture with float uv, an area light), the integration guide's DeviceManager hands it
to the C ABI, and Renderer::Run's frame loop renders 4 frames of one sample per pixel in strict
math. The film equals the CPU oracle's render of the same arrays and camera bit for bit."""
import numpy as np
import pytest

import frontend_dump
import pyoracle as po
import wayland_b200 as wl
from pbrt_fixture import write_scene
from wayland_b200 import pbrt

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not frontend_dump.available(),
                                 reason="oracle/_ref/wl_frontend not built (needs the reference tree)")]


def test_reference_frontend_renders_through_the_abi(oracle, tmp_path):
    path = write_scene(tmp_path)
    ref_scene = pbrt.load(str(path))
    sc, film = frontend_dump.run(path, ref_scene.width, ref_scene.height, tmp_path / "dump.bin", frames=4,
                                 depth=6, strict=True)
    assert film is not None and film.mean() > 0.01
    assert len(sc.textures) == 1 and sc.UV is not None and sc.UV.any()
    p = wl.render_params(sc.width, sc.height, 4, max_depth=6, math=wl.MATH_STRICT)
    cam = po.Camera()
    for k in ("pos", "look_at", "up", "right"):
        getattr(cam, k)[:] = [float(x) for x in sc.camera[k]]
    q = po.RenderParams()
    for k, _ in q._fields_:
        if k == "env":
            q.env[:] = list(p.env)
        else:
            setattr(q, k, getattr(p, k))
    img, _, _ = oracle.render(sc, cam, q)
    assert np.array_equal(film.view(np.uint32), np.ascontiguousarray(img, np.float32).view(np.uint32))
