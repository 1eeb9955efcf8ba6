"""Edge cases of the render entry points against the oracle, in WL_MATH_STRICT mode (bit for bit):
images of one pixel and of sizes that divide into nothing (7 x 3, 33 x 17), one sample per
pixel and more samples than one wave holds, a scene without lights (environment only: next-event
estimation is skipped, BDPT traces no light subpath), and the same scene lit by nothing at all
(a black image)."""
import dataclasses

import numpy as np
import pytest

import pyoracle as po
import wayland_b200 as wl
from wayland_b200 import scenes

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def ocam(sc):
    c = po.Camera()
    for k in ("pos", "look_at", "up", "right"):
        getattr(c, k)[:] = [float(x) for x in sc.camera[k]]
    return c


def oparams(p):
    q = po.RenderParams()
    for k, _ in q._fields_:
        if k == "env":
            q.env[:] = list(p.env)
        else:
            setattr(q, k, getattr(p, k))
    return q


def render(ctx, sc, p):
    s = wl.Scene(ctx, sc)
    film = wl.Film(ctx, p.width, p.height)
    wl.render(ctx, s, sc.camera_struct(), p, film)
    img = film.download()
    film.close()
    s.close()
    return img


def lightless(W, H):
    """The Cornell box with its light's triangles kept as geometry but no light records."""
    sc = scenes.cornell_box(W, H)
    return dataclasses.replace(sc, lights=np.zeros(0, sc.lights.dtype))


@pytest.mark.parametrize("W,H,spp,wave", [(1, 1, 3, 0), (7, 3, 2, 0), (33, 17, 5, 0), (33, 17, 5, 600)])
def test_ragged_sizes_strict_vs_oracle(ctx, oracle, W, H, spp, wave):
    sc = scenes.cornell_box(W, H)
    p = wl.render_params(W, H, spp, math=wl.MATH_STRICT, wave_paths=wave)
    img = render(ctx, sc, p)
    ref, _, _ = oracle.render(sc, ocam(sc), oparams(p))
    assert np.array_equal(bits(img), bits(ref))


@pytest.mark.parametrize("strategy", [wl.STRATEGY_MIS, wl.STRATEGY_BDPT])
def test_scene_without_lights_strict_vs_oracle(ctx, oracle, strategy):
    sc = lightless(24, 16)
    kw = dict(max_depth=6) if strategy == wl.STRATEGY_BDPT else {}
    p = wl.render_params(24, 16, 3, math=wl.MATH_STRICT, strategy=strategy, env=(0.3, 0.2, 0.1), **kw)
    img = render(ctx, sc, p)
    if strategy == wl.STRATEGY_BDPT:
        ref, _, _ = oracle.render_bdpt(sc, ocam(sc), oparams(p))
    else:
        ref, _, _ = oracle.render(sc, ocam(sc), oparams(p))
    assert np.array_equal(bits(img), bits(ref))


def test_nothing_emits(ctx):
    sc = lightless(16, 16)
    p = wl.render_params(16, 16, 2, math=wl.MATH_STRICT)
    img = render(ctx, sc, p)
    assert np.isfinite(img).all() and not img.any()
