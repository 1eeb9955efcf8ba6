"""The radiance cache on the bidirectional program's camera subpaths (wl_render_nrc with
WL_STRATEGY_BDPT).

A frame renders one sample per pixel by BDPT over the paths of at most t = query_depth vertices
after the camera, plus the cache's prediction at the t-th eye vertex (times the eye subpath's
throughput) for every longer path.

- Exactness of the bidirectional part: with the cache's weights at zero and a learning rate of
  zero the prediction is exactly 0, so a WL_MATH_STRICT render must equal, bit for bit, the
  oracle's BDPT restricted to paths of at most t vertices (eye subpaths of t vertices, light
  subpaths of t - 1, connections (i, j) with i + j + 2 <= t), for several t.
- What the cache adds: after online training, the image's mean brightness is within 10 % of
  the plain (unrestricted) BDPT at high spp, while the restricted part alone is measurably
  darker (the cache carries the longer paths)."""
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


@pytest.mark.parametrize("t", [1, 2, 3, 4])
def test_restricted_bdpt_strict_vs_oracle(ctx, oracle, t):
    sc = scenes.cornell_box(24, 24)
    s = wl.Scene(ctx, sc)
    c = wl.RadianceCache(ctx, s, log2_table=12, train_paths=64, query_depth=t, learning_rate=0.0)
    c.set_weights(np.zeros(wl._abi.NRC_WEIGHTS, np.float32))
    film = wl.Film(ctx, 24, 24)
    p = wl.render_params(24, 24, 3, strategy=wl.STRATEGY_BDPT, max_depth=10, math=wl.MATH_STRICT)
    wl.render_nrc(ctx, s, sc.camera_struct(), p, c, film)
    img = film.download()
    film.close()
    ref, _, _ = oracle.render_bdpt(sc, ocam(sc), oparams(p), max_len=t)
    d = (bits(img) != bits(ref)).any(axis=-1)
    assert not d.any(), f"t={t}: {int(d.sum())} of {d.size} pixels differ; first {np.argwhere(d)[:4].tolist()}"
    assert np.abs(c.weights()).max() == 0.0  # learning rate 0 leaves the zero network as it was
    c.close()
    s.close()


def test_cache_carries_long_paths(ctx, oracle):
    W = H = 48
    sc = scenes.cornell_box(W, H)
    s = wl.Scene(ctx, sc)
    cam = sc.camera_struct()
    t = 3
    # plain BDPT (subpaths of up to 10 vertices) at high spp: the reference brightness
    ref_film = wl.Film(ctx, W, H)
    wl.render(ctx, s, cam, wl.render_params(W, H, 256, strategy=wl.STRATEGY_BDPT, max_depth=10), ref_film)
    ref = float(ref_film.download().mean())
    ref_film.close()
    # the restricted part alone (oracle, paths of at most t vertices): darker than the full image
    part, _, _ = oracle.render_bdpt(sc, ocam(sc), oparams(wl.render_params(W, H, 16, strategy=wl.STRATEGY_BDPT,
                                                                            max_depth=10)), max_len=t)
    part_mean = float(part.mean())
    assert part_mean < 0.9 * ref, (part_mean, ref)
    # with the cache, trained online (warm-up frames without a film, then the image)
    c = wl.RadianceCache(ctx, s, log2_table=16, train_paths=1024, query_depth=t)
    p = wl.render_params(W, H, 32, strategy=wl.STRATEGY_BDPT, max_depth=10)
    wl.render_nrc(ctx, s, cam, p, c, None)
    film = wl.Film(ctx, W, H)
    p.first_frame = 0
    wl.render_nrc(ctx, s, cam, p, c, film)
    img = film.download()
    st = c.stats()
    film.close()
    c.close()
    s.close()
    assert np.isfinite(img).all()
    assert st["train_samples"] > 500 and np.isfinite(st["loss"])
    assert abs(float(img.mean()) - ref) < 0.1 * ref, (float(img.mean()), part_mean, ref)
