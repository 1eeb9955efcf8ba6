"""The oracle against the golden vectors generated from the reference's own device code
(tests/golden/make_golden.py). Bit-exact: every comparison is on the float bit patterns."""
import os

import numpy as np
import pytest

import pyoracle as po
from wayland_b200 import scenes

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def gold():
    return dict(np.load(os.path.join(GOLD, "device_math.npz")))


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_tea4(oracle, gold):
    got = np.array([oracle.tea4(int(a), int(b)) for a, b in gold["tea_in"]], np.uint32)
    assert np.array_equal(got, gold["tea_out"])


def test_lcg_stream(oracle, gold):
    for s, ref in zip(gold["rnd_seed"], gold["rnd_out"]):
        assert np.array_equal(bits(oracle.lcg_stream(int(s), 64)), bits(ref))


def test_disney_eval(oracle, gold):
    g = gold
    got = oracle.disney_eval(g["mats"], g["Ns"], g["Ng"], g["V"], g["L"], g["tex"])
    assert np.array_equal(bits(got), bits(g["eval"]))
    assert (np.abs(g["eval"]) > 0).any(axis=1).mean() > 0.2  # the cases exercise the lobes


def test_disney_pdf(oracle, gold):
    g = gold
    got = oracle.disney_pdf(g["mats"], g["Ns"], g["Ng"], g["V"], g["L"])
    assert np.array_equal(bits(got), bits(g["pdf"]))


def test_disney_sample(oracle, gold):
    g = gold
    got, seeds = oracle.disney_sample(g["mats"], g["Ns"], g["Ng"], g["V"], g["sample_seed"])
    assert np.array_equal(bits(got), bits(g["sample"]))
    assert np.array_equal(seeds, g["sample_seed_out"])
    # transmission, diffuse and specular branches are all present
    refl = (np.einsum("ij,ij->i", g["sample"], g["Ns"]) * np.einsum("ij,ij->i", g["V"], g["Ns"]))
    assert (refl < 0).sum() > 100 and (refl > 0).sum() > 100


def test_camera(oracle, gold):
    g = gold
    cam = po.Camera()
    for i, k in enumerate(("pos", "look_at", "up", "right")):
        getattr(cam, k)[:] = [float(x) for x in g["cam"][i]]
    d, s = oracle.camera_rays(cam, 256, 256, g["cam_px"], g["cam_py"], g["cam_seed"])
    assert np.array_equal(bits(d), bits(g["cam_dir"]))
    assert np.array_equal(s, g["cam_seed_out"])


def test_ace(oracle, gold):
    assert np.array_equal(bits(oracle.ace(gold["ace_in"])), bits(gold["ace_out"]))


def test_cornell_image(oracle):
    """The oracle's path tracer reproduces the reference-math render of the Cornell box."""
    g = dict(np.load(os.path.join(GOLD, "cornell_32x32_4spp.npz")))

    class S:
        V, I, tri_material, mats, lights = g["V"], g["I"], g["tri_material"], g["mats"], g["lights"]
        N = None
        tri_flags = None

    cam = po.Camera()
    for i, k in enumerate(("pos", "look_at", "up", "right")):
        getattr(cam, k)[:] = [float(x) for x in g["cam"][i]]
    p = po.RenderParams(width=32, height=32, spp=4, first_frame=0, max_depth=25, rr_depth=5,
                        rr_prob=0.9, eps=1e-3, strategy=2, rng=0, math=1, lights=0, seed=0)
    img, _, segs = oracle.render(S(), cam, p)
    assert np.array_equal(bits(img), bits(g["image"]))
    assert segs == int(g["segments"])
    assert img.mean() > 0.05


def test_own_transcendentals(oracle):
    """The project's sin/cos/log are within a few ulp of the double-precision values."""
    xs = np.linspace(0, 2 * np.pi, 4001, dtype=np.float32)
    s = np.array([oracle.sinf(x) for x in xs])
    c = np.array([oracle.cosf(x) for x in xs])
    assert np.abs(s - np.sin(xs.astype(np.float64))).max() < 2e-7
    assert np.abs(c - np.cos(xs.astype(np.float64))).max() < 2e-7
    ys = np.exp(np.linspace(-25, 10, 4001)).astype(np.float32)
    lg = np.array([oracle.logf(y) for y in ys])
    assert (np.abs(lg - np.log(ys.astype(np.float64))) / np.maximum(1.0, np.abs(np.log(ys)))).max() < 3e-7
    assert np.isnan(oracle.logf(-1.0)) and np.isneginf(oracle.logf(0.0))


class _GoldScene:
    def __init__(self, g):
        self.V, self.I, self.N = g["V"], g["I"], g.get("N")
        self.tri_flags = g.get("tri_flags")
        self.tri_material = np.zeros(len(self.I), np.uint32)
        self.mats = np.zeros(1, po.DISNEY_DTYPE)
        self.lights = np.zeros(0, po.LIGHT_DTYPE)


def test_ao_image(oracle):
    """The oracle's ambient occlusion reproduces AO.cu's loop over the reference's arithmetic."""
    g = dict(np.load(os.path.join(GOLD, "ao_sphere_40x24.npz")))
    cam = po.Camera()
    for i, k in enumerate(("pos", "look_at", "up", "right")):
        getattr(cam, k)[:] = [float(x) for x in g["cam"][i]]
    p = po.AoParams(width=40, height=24, spp=2, first_frame=0, camera_samples=4, ao_rays=32,
                    radius=1.0, eps=1e-3, rng=0, wave_paths=0, seed=0)
    img, _, rays = oracle.render_ao(_GoldScene(g), cam, p)
    assert np.array_equal(bits(img), bits(g["image"]))
    assert rays == int(g["rays"])


@pytest.mark.parametrize("name,make", [
    ("bdpt_cornell_32x32_4spp.npz", lambda: scenes.cornell_box(32, 32)),
    ("bdpt_glass_40x40_4spp.npz", lambda: scenes.glass_sphere(40, 40, subdiv=12)),
])
def test_bdpt_image(oracle, name, make):
    """The oracle's bidirectional path tracer reproduces the reference's BDPT program
    (Programs/BDPT/BDPT.cu run over the OptiX host emulation) bit for bit."""
    g = dict(np.load(os.path.join(GOLD, name)))
    sc = make()
    assert np.array_equal(sc.V, g["V"]) and np.array_equal(sc.I, g["I"])
    cam = po.Camera()
    for i, k in enumerate(("pos", "look_at", "up", "right")):
        getattr(cam, k)[:] = [float(x) for x in g["cam"][i]]
    p = po.RenderParams(width=sc.width, height=sc.height, spp=4, first_frame=0, max_depth=10,
                        rr_depth=5, rr_prob=0.9, eps=1e-3, strategy=3, rng=0, math=1, lights=0,
                        seed=0)
    img, _, rays = oracle.render_bdpt(sc, cam, p)
    assert np.isfinite(g["image"]).all() and g["image"].max() > 0
    assert np.array_equal(bits(img), bits(g["image"]))


def test_program_pt_image(oracle):
    """The oracle's path tracer reproduces the reference's PathTracing.cu program itself (run
    over the OptiX host emulation) bit for bit: vertex normals, Disney lobes, four lights."""
    g = dict(np.load(os.path.join(GOLD, "program_pt_sphere_48x32_4spp.npz")))
    sc = scenes.displaced_sphere(48, 32, subdiv=24, seed=3)
    assert np.array_equal(sc.V, g["V"]) and np.array_equal(sc.I, g["I"])
    cam = po.Camera()
    for k in ("pos", "look_at", "up", "right"):
        getattr(cam, k)[:] = [float(x) for x in sc.camera[k]]
    p = po.RenderParams(width=48, height=32, spp=4, first_frame=0, max_depth=25, rr_depth=5,
                        rr_prob=0.9, eps=1e-3, strategy=2, rng=0, math=1, lights=0, seed=0)
    img, _, _ = oracle.render(sc, cam, p)
    assert g["image"].max() > 0
    assert np.array_equal(bits(img), bits(g["image"]))


def test_program_ao_image(oracle):
    """The oracle's ambient occlusion reproduces the reference's AO.cu program itself in a
    closed room (every camera ray hits)."""
    g = dict(np.load(os.path.join(GOLD, "program_ao_room_32x24_2spp.npz")))
    sc = scenes.door_slit_room(32, 24, cells=8, slit=0.0)
    assert np.array_equal(sc.V, g["V"]) and np.array_equal(sc.I, g["I"])
    cam = po.Camera()
    for k in ("pos", "look_at", "up", "right"):
        getattr(cam, k)[:] = [float(x) for x in sc.camera[k]]
    p = po.AoParams(width=32, height=24, spp=2, first_frame=0, camera_samples=4, ao_rays=32,
                    radius=1.0, eps=1e-3, rng=0, wave_paths=0, seed=0)
    img, _, _ = oracle.render_ao(sc, cam, p)
    assert np.array_equal(bits(img), bits(g["image"]))
