"""The reference's own frontend (minipbrt + SceneManager, SceneManager.cpp:14-246, compiled in
place into oracle/_ref/wl_frontend) against the project's Python restatement of it
(wayland_b200/pbrt.py): the arrays the integration guide's DeviceManager hands to wl_scene_create
and the camera frame must be equal bit for bit, on the test scene (every material kind the
reference converts, a PLY mesh, a transformed shape, vertex normals, texture coordinates, an
imagemap texture, an area light) and on the reference's own cbox.pbrt. Parse only: no GPU."""
import os

import numpy as np
import pytest

import frontend_dump
from pbrt_fixture import write_scene
from wayland_b200 import pbrt

REF_CBOX = os.path.join(os.environ.get("WL_REFERENCE_ROOT", "/root/reference"), "scene", "cornell-box",
                        "cbox.pbrt")
pytestmark = pytest.mark.skipif(not frontend_dump.available(),
                                reason="oracle/_ref/wl_frontend not built (needs the reference tree)")


def same_scene(a, b):
    assert np.array_equal(a.V, b.V)
    assert np.array_equal(a.I, b.I)
    assert np.array_equal(a.tri_material, b.tri_material)
    assert a.mats.tobytes() == b.mats.tobytes()
    assert a.lights.tobytes() == b.lights.tobytes()
    if b.N is not None:
        flags = b.tri_flags if b.tri_flags is not None else np.ones(b.num_tris, np.uint32)
        assert np.array_equal(a.tri_flags, flags)
        used = np.unique(b.I[flags == 1])
        assert np.array_equal(a.N[used], b.N[used])
    else:
        assert not a.tri_flags.any()
    if b.UV is not None:
        assert np.array_equal(a.UV, b.UV)
    assert len(a.textures) == len(b.textures)
    for ta, tb in zip(a.textures, b.textures):
        assert np.array_equal(ta, tb)
    for k in ("pos", "look_at", "up", "right"):
        assert np.array_equal(a.camera[k], np.asarray(b.camera[k], np.float32)), k


def test_frontend_matches_python_loader_on_test_scene(tmp_path):
    path = write_scene(tmp_path)
    ref = pbrt.load(str(path))
    got, film = frontend_dump.run(path, ref.width, ref.height, tmp_path / "dump.bin")
    assert film is None
    same_scene(got, ref)


@pytest.mark.skipif(not os.path.exists(REF_CBOX), reason="needs the reference's scene files")
def test_frontend_matches_python_loader_on_cbox(tmp_path):
    ref = pbrt.load(REF_CBOX)
    got, _ = frontend_dump.run(REF_CBOX, ref.width, ref.height, tmp_path / "dump.bin")
    same_scene(got, ref)
