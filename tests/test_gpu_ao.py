"""Ambient occlusion (AO.cu:21-130) on the GPU through the C ABI: bit-identical to the golden
image made from the reference's own arithmetic and to the oracle, for both random streams, any
wave size and multi-call accumulation."""
import os

import numpy as np
import pytest

import pyoracle as po
import wayland_b200 as wl
from wayland_b200 import scenes

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def oparams(p):
    q = po.AoParams()
    for k, _ in q._fields_:
        setattr(q, k, getattr(p, k))
    return q


def ocam(sc):
    c = po.Camera()
    for k in ("pos", "look_at", "up", "right"):
        getattr(c, k)[:] = [float(x) for x in sc.camera[k]]
    return c


def test_ao_golden(ctx):
    g = dict(np.load(os.path.join(GOLD, "ao_sphere_40x24.npz")))
    sph = scenes.displaced_sphere(40, 24, subdiv=12, seed=5)
    assert np.array_equal(sph.V, g["V"]) and np.array_equal(sph.I, g["I"])
    s = wl.Scene(ctx, sph)
    film = wl.Film(ctx, 40, 24)
    wl.render_ao(ctx, s, sph.camera_struct(), wl.ao_params(40, 24, 2), film)
    assert np.array_equal(bits(film.download()), bits(g["image"]))


@pytest.mark.parametrize("rng", [wl.RNG_TEA_LCG, wl.RNG_PCG32])
def test_ao_vs_oracle(ctx, oracle, rng):
    sc = scenes.cornell_box(48, 40)
    s = wl.Scene(ctx, sc)
    p = wl.ao_params(48, 40, 3, rng=rng, seed=5, radius=0.1, ao_rays=8, camera_samples=3)
    film = wl.Film(ctx, 48, 40, fp64=True)
    wl.render_ao(ctx, s, sc.camera_struct(), p, film)
    ref, ref64, _ = oracle.render_ao(sc, ocam(sc), oparams(p), want64=True)
    assert np.array_equal(bits(film.download()), bits(ref))
    assert np.array_equal(film.download64().view(np.uint64), ref64.view(np.uint64))
    # small waves (one camera-sample group of 3 per slot, waves cut inside a frame) and two
    # calls (frames 0-1, then 2) give the same image
    f2 = wl.Film(ctx, 48, 40)
    wl.render_ao(ctx, s, sc.camera_struct(), wl.ao_params(48, 40, 2, rng=rng, seed=5, radius=0.1,
                                                          ao_rays=8, camera_samples=3, wave_paths=999), f2)
    wl.render_ao(ctx, s, sc.camera_struct(), wl.ao_params(48, 40, 1, first_frame=2, rng=rng, seed=5,
                                                          radius=0.1, ao_rays=8, camera_samples=3), f2)
    assert np.array_equal(bits(f2.download()), bits(ref))


def test_ao_program_golden(ctx):
    """GPU strict AO == the reference's AO.cu program itself, closed room, bit for bit."""
    g = dict(np.load(os.path.join(GOLD, "program_ao_room_32x24_2spp.npz")))
    sc = scenes.door_slit_room(32, 24, cells=8, slit=0.0)
    assert np.array_equal(sc.V, g["V"]) and np.array_equal(sc.I, g["I"])
    s = wl.Scene(ctx, sc)
    film = wl.Film(ctx, 32, 24)
    wl.render_ao(ctx, s, sc.camera_struct(), wl.ao_params(32, 24, 2), film)
    assert np.array_equal(bits(film.download()), bits(g["image"]))
    film.close()
    s.close()
