"""The wavefront bidirectional path tracer (wl_render with WL_STRATEGY_BDPT) against the
reference's BDPT program and the oracle.

WL_MATH_STRICT renders are compared bit for bit: with the golden images made by the reference's
own Programs/BDPT/BDPT.cu (run on the host over an emulation of its OptiX calls), and with the
oracle's restatement for both random streams, subpath caps from 1 to 10, vertex normals,
transmission and metallic lobes, four lights, multi-call accumulation and small waves.
WL_MATH_FAST is compared with the FP64 oracle by relMSE at equal spp (tolerance 2e-3)."""
import os

import numpy as np
import pytest

import pyoracle as po
import wayland_b200 as wl
from wayland_b200 import scenes

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FAST_RELMSE_TOL = 2e-3


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def same(img, ref):
    """Bit equality, with the share of differing pixels in the failure message."""
    d = (bits(img) != bits(ref)).any(axis=-1)
    return not d.any(), f"{int(d.sum())} of {d.size} pixels differ; first {np.argwhere(d)[:4].tolist()}"


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


def bdpt_params(W, H, spp, **kw):
    kw.setdefault("max_depth", 10)
    return wl.render_params(W, H, spp, strategy=wl.STRATEGY_BDPT, **kw)


def gpu_bdpt(ctx, sc, p, fp64=False, calls=1):
    s = wl.Scene(ctx, sc)
    film = wl.Film(ctx, p.width, p.height, fp64=fp64)
    spp, first = p.spp, p.first_frame
    per = spp // calls
    for k in range(calls):
        p.first_frame = first + k * per
        p.spp = per if k < calls - 1 else spp - per * (calls - 1)
        wl.render(ctx, s, sc.camera_struct(), p, film)
    p.spp, p.first_frame = spp, first
    img = film.download()
    img64 = film.download64() if fp64 else None
    film.close()
    s.close()
    return img, img64


@pytest.mark.parametrize("name,make", [
    ("bdpt_cornell_32x32_4spp.npz", lambda: scenes.cornell_box(32, 32)),
    ("bdpt_glass_40x40_4spp.npz", lambda: scenes.glass_sphere(40, 40, subdiv=12)),
])
def test_golden_bdpt_strict(ctx, name, make):
    """GPU strict mode == the reference's BDPT program, bit for bit."""
    g = dict(np.load(os.path.join(GOLD, name)))
    sc = make()
    assert np.array_equal(sc.V, g["V"]) and np.array_equal(sc.I, g["I"])
    img, _ = gpu_bdpt(ctx, sc, bdpt_params(sc.width, sc.height, 4, math=wl.MATH_STRICT))
    ok, msg = same(img, g["image"])
    assert ok, msg


@pytest.mark.parametrize("rng", [wl.RNG_TEA_LCG, wl.RNG_PCG32])
@pytest.mark.parametrize("max_depth", [1, 2, 3, 10])
def test_cornell_bdpt_strict_vs_oracle(ctx, oracle, rng, max_depth):
    sc = scenes.cornell_box(40, 36)
    p = bdpt_params(40, 36, 3, math=wl.MATH_STRICT, rng=rng, seed=11, max_depth=max_depth)
    img, _ = gpu_bdpt(ctx, sc, p)
    ref, _, _ = oracle.render_bdpt(sc, ocam(sc), oparams(p))
    ok, msg = same(img, ref)
    assert ok, msg


def test_sphere_bdpt_strict_vs_oracle(ctx, oracle):
    """Vertex normals, random Disney materials (metallic, transmission), four lights."""
    sc = scenes.displaced_sphere(width=48, height=32, subdiv=24, seed=3)
    p = bdpt_params(48, 32, 4, math=wl.MATH_STRICT)
    img, _ = gpu_bdpt(ctx, sc, p)
    ref, _, _ = oracle.render_bdpt(sc, ocam(sc), oparams(p))
    ok, msg = same(img, ref)
    assert ok, msg
    assert img.max() > 0


def test_bdpt_strict_calls_and_waves(ctx, oracle):
    """Two render calls continue the running mean; waves smaller than one frame give the same
    image as one wave."""
    sc = scenes.glass_sphere(36, 30, subdiv=10)
    p = bdpt_params(36, 30, 6, math=wl.MATH_STRICT, first_frame=2)
    ref, _, _ = oracle.render_bdpt(sc, ocam(sc), oparams(p))
    img, _ = gpu_bdpt(ctx, sc, p, calls=2)
    ok, msg = same(img, ref)
    assert ok, msg
    p.wave_paths = 1024
    img2, _ = gpu_bdpt(ctx, sc, p)
    ok, msg = same(img2, ref)
    assert ok, msg


def test_bdpt_fast_vs_fp64_oracle(ctx, oracle):
    sc = scenes.cornell_box(64, 64)
    p = bdpt_params(64, 64, 32)
    img, img64 = gpu_bdpt(ctx, sc, p, fp64=True)
    _, ref64, _ = oracle.render_bdpt(sc, ocam(sc), oparams(p), prec=1, want64=True)
    rel = float(((img64 - ref64) ** 2 / (ref64 ** 2 + 1e-2)).mean())
    assert rel < FAST_RELMSE_TOL
    assert np.isfinite(img).all()


def test_bdpt_rejects_long_subpaths(ctx):
    sc = scenes.cornell_box(8, 8)
    s = wl.Scene(ctx, sc)
    film = wl.Film(ctx, 8, 8)
    with pytest.raises(wl.WlError):
        wl.render(ctx, s, sc.camera_struct(), bdpt_params(8, 8, 1, max_depth=wl.BDPT_MAX_VERTICES + 1), film)
    film.close()
    s.close()
