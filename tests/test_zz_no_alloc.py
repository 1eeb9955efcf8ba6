"""wl_render_noalloc: the render entry point for callers that must not allocate device memory
once they are running (a host that reserves its whole device budget up front, a real-time loop
that cannot absorb an allocation's implicit synchronisation). Its path queues live in a static
device array instead of cudaMalloc'd memory.

The test calls it through the C ABI twice in a row and checks each result against wl_render's
on the same inputs. In WL_MATH_STRICT mode the tolerance is zero (bit-identical), the same
tolerance every strict-mode render test here uses. The render spans several waves of the
static scratch. The test also checks that a second call leaves the device's free memory
unchanged, and that an oversized wave is refused. This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest
import torch

import wayland_b200 as wl
from wayland_b200 import _abi, scenes

pytestmark = pytest.mark.gpu


def noalloc(ctx, scene, camera, params, film):
    _abi.check("wl_render_noalloc", ctx.lib.wl_render_noalloc(
        ctx.handle, scene.handle, C.byref(camera), C.byref(params), film.handle))


@pytest.fixture(scope="module")
def own_ctx():
    c = wl.Context(0)
    yield c
    c.close()


def test_noalloc_matches_render_twice(own_ctx):
    ctx = own_ctx
    sc = scenes.cornell_box(320, 240)          # 76,800 pixels x 2 spp: three waves of scratch
    scene = wl.Scene(ctx, sc)
    cam = sc.camera_struct()
    p = wl.render_params(320, 240, 2, math=wl.MATH_STRICT, max_depth=8)
    ref_film = wl.Film(ctx, 320, 240, fp64=True)
    wl.render(ctx, scene, cam, p, ref_film)
    ref = ref_film.download()
    ref64 = ref_film.download64()
    assert ref.mean() > 0.01
    for call in range(2):
        film = wl.Film(ctx, 320, 240, fp64=True)
        # the context reserved the scratch when it was created: neither the first call nor the
        # second changes the device's free memory
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        noalloc(ctx, scene, cam, p, film)
        ctx.sync()
        assert torch.cuda.mem_get_info()[0] == free_before, f"call {call} allocated"
        got = film.download()
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), f"call {call}"
        assert np.array_equal(film.download64().view(np.uint64), ref64.view(np.uint64))
        film.close()


def test_noalloc_fast_mode_and_limit(own_ctx):
    ctx = own_ctx
    sc = scenes.cornell_box(96, 64)
    scene = wl.Scene(ctx, sc)
    cam = sc.camera_struct()
    p = wl.render_params(96, 64, 4, math=wl.MATH_FAST, max_depth=8)
    a = wl.Film(ctx, 96, 64)
    wl.render(ctx, scene, cam, p, a)
    b = wl.Film(ctx, 96, 64)
    noalloc(ctx, scene, cam, p, b)
    # identical kernels and random streams; only the queue memory differs
    assert np.array_equal(a.download().view(np.uint32), b.download().view(np.uint32))
    big = wl.render_params(96, 64, 4, wave_paths=_abi.NOALLOC_MAX_PATHS + 1)
    with pytest.raises(wl.WlError, match="INVALID_ARG.*static scratch limit"):
        noalloc(ctx, scene, cam, big, b)
    # flags it cannot honour are refused rather than ignored
    for flag in (_abi.RENDER_GRAPH, _abi.RENDER_TRAVERSAL_STATS):
        with pytest.raises(wl.WlError, match="INVALID_ARG.*SORT_MATERIALS"):
            noalloc(ctx, scene, cam, wl.render_params(96, 64, 4, flags=flag), b)
    # the bidirectional program needs more memory than the static array holds
    with pytest.raises(wl.WlError, match="INVALID_ARG.*path tracer only"):
        noalloc(ctx, scene, cam, wl.render_params(96, 64, 4, strategy=wl.STRATEGY_BDPT, max_depth=6), b)
    # the caller's current device is the same after the call
    torch.cuda.set_device(0)
    noalloc(ctx, scene, cam, p, b)
    assert torch.cuda.current_device() == 0
