"""The wavefront path tracer through the C ABI against the oracle.

WL_MATH_STRICT renders are compared bit for bit: with the golden image made from the reference's
own device code (TEA+LCG, Cornell box), and with the oracle's path tracer for both random streams,
all three strategies, a scene with vertex normals, transmission, metallic lobes, an environment
and four lights, multi-call accumulation and any wave size. WL_MATH_FAST (the benchmark mode)
is compared with the FP64 oracle by relMSE at equal spp: tolerance 2e-3 (fast-math sin/cos/log
and approximate division change a few paths; the statistics do not change)."""
import os

import numpy as np
import pytest
import torch

import pyoracle as po
import wayland_b200 as wl
from wayland_b200 import scenes

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FAST_RELMSE_TOL = 2e-3


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


def gpu_render(ctx, scene_data, p, fp64=False, scene=None):
    sc = scene or wl.Scene(ctx, scene_data)
    film = wl.Film(ctx, p.width, p.height, fp64=fp64)
    wl.render(ctx, sc, scene_data.camera_struct(), p, film)
    img = film.download()
    img64 = film.download64() if fp64 else None
    return img, img64, film, sc


def small_sphere(W=48, H=32):
    return scenes.displaced_sphere(width=W, height=H, subdiv=24, seed=3)


def test_golden_cornell_strict(ctx):
    """GPU strict mode == the reference's device code (via oracle/_ref), bit for bit."""
    g = dict(np.load(os.path.join(GOLD, "cornell_32x32_4spp.npz")))
    sc = scenes.cornell_box(32, 32)
    assert np.array_equal(sc.V, g["V"]) and np.array_equal(sc.I, g["I"])
    p = wl.render_params(32, 32, 4, math=wl.MATH_STRICT)
    img, _, film, s = gpu_render(ctx, sc, p)
    assert np.array_equal(bits(img), bits(g["image"]))
    assert ctx.stats()["segments"] == int(g["segments"])


@pytest.mark.parametrize("rng", [wl.RNG_TEA_LCG, wl.RNG_PCG32])
@pytest.mark.parametrize("strategy", [wl.STRATEGY_MIS, wl.STRATEGY_NEE, wl.STRATEGY_UPT])
def test_cornell_strict_vs_oracle(ctx, oracle, rng, strategy):
    sc = scenes.cornell_box(48, 40)
    p = wl.render_params(48, 40, 3, math=wl.MATH_STRICT, rng=rng, strategy=strategy, seed=7,
                         max_depth=8)
    img, _, _, _ = gpu_render(ctx, sc, p)
    ref, _, segs = oracle.render(sc, ocam(sc), oparams(p))
    assert np.array_equal(bits(img), bits(ref))
    assert ctx.stats()["segments"] == segs


@pytest.mark.parametrize("rng", [wl.RNG_TEA_LCG, wl.RNG_PCG32])
def test_sphere_strict_vs_oracle(ctx, oracle, rng):
    """Vertex normals, random Disney (transmission, metallic), 4 lights, environment 0.1."""
    sc = small_sphere()
    p = wl.render_params(sc.width, sc.height, 2, math=wl.MATH_STRICT, rng=rng, max_depth=16,
                         env=sc.env, seed=11)
    img, _, _, _ = gpu_render(ctx, sc, p)
    ref, _, segs = oracle.render(sc, ocam(sc), oparams(p))
    assert np.array_equal(bits(img), bits(ref))
    assert img.mean() > 0.01


def test_accumulation_and_waves(ctx, oracle):
    """Two calls (frames 0-1, 2-4) == one call of 5 frames == many small waves; FP64 film equals
    the oracle's FP64 mean."""
    sc = scenes.cornell_box(40, 24)
    s = wl.Scene(ctx, sc)
    cam = sc.camera_struct()
    film = wl.Film(ctx, 40, 24, fp64=True)
    wl.render(ctx, s, cam, wl.render_params(40, 24, 2, math=wl.MATH_STRICT), film)
    wl.render(ctx, s, cam, wl.render_params(40, 24, 3, first_frame=2, math=wl.MATH_STRICT), film)
    a = film.download()
    p5 = wl.render_params(40, 24, 5, math=wl.MATH_STRICT)
    one, one64, _, _ = gpu_render(ctx, sc, p5, fp64=True, scene=s)
    small = wl.render_params(40, 24, 5, math=wl.MATH_STRICT, wave_paths=1000)
    b, _, _, _ = gpu_render(ctx, sc, small, scene=s)
    ref, ref64, _ = oracle.render(sc, ocam(sc), oparams(p5), want64=True)
    assert np.array_equal(bits(a), bits(ref))
    assert np.array_equal(bits(one), bits(ref))
    assert np.array_equal(bits(b), bits(ref))
    assert np.array_equal(one64.view(np.uint64), ref64.view(np.uint64))


def test_fast_mode_relmse(ctx, oracle):
    """Benchmark arithmetic vs the FP64 oracle at equal spp and the same random streams."""
    sc = scenes.cornell_box(64, 64)
    p = wl.render_params(64, 64, 16, math=wl.MATH_FAST, max_depth=8)
    img, _, _, _ = gpu_render(ctx, sc, p)
    _, ref64, _ = oracle.render(sc, ocam(sc), oparams(p), prec=1, want64=True)
    rel = oracle.relmse(img, ref64)
    assert rel < FAST_RELMSE_TOL, rel
    sc2 = small_sphere()
    p2 = wl.render_params(sc2.width, sc2.height, 8, math=wl.MATH_FAST, max_depth=16, env=sc2.env)
    img2, _, _, _ = gpu_render(ctx, sc2, p2)
    _, ref2, _ = oracle.render(sc2, ocam(sc2), oparams(p2), prec=1, want64=True)
    assert oracle.relmse(img2, ref2) < 5 * FAST_RELMSE_TOL


BENCH_FAST_TOL = 1e-2


def test_fast_mode_bench_scene(ctx, oracle):
    """The benchmark's own arithmetic on the benchmark's own scene: the 1,997,130-triangle
    displaced sphere with its 4 lights and environment 0.1, depth 16, MIS, TEA+LCG, fast math,
    binned-SAH BVH, at 96x54 x 16 spp (the bench's 1920x1080 view at 1/20 scale) against the FP64
    oracle with the same random streams. relMSE below BENCH_FAST_TOL, and below a tenth of the
    relMSE of an independent 16-spp render (other frames) against the same oracle image: the
    fast-math deviation is far below the Monte-Carlo noise of an image at the same spp."""
    sc = scenes.displaced_sphere(96, 54, 16, 16)
    assert sc.num_tris == 1997130
    s = wl.Scene(ctx, sc, bvh_kind=wl.BVH_SAH)
    p = wl.render_params(96, 54, 16, math=wl.MATH_FAST, max_depth=16, env=sc.env)
    img, _, _, _ = gpu_render(ctx, sc, p, scene=s)
    _, ref64, _ = oracle.render(sc, ocam(sc), oparams(p), prec=1, want64=True)
    q = wl.render_params(96, 54, 16, math=wl.MATH_FAST, max_depth=16, env=sc.env, first_frame=1000)
    other, _, _, _ = gpu_render(ctx, sc, q, scene=s)
    rel = oracle.relmse(img, ref64)
    noise = oracle.relmse(other, ref64)
    print(f"bench scene fast vs FP64 oracle relMSE {rel:.3e}, independent render {noise:.3e}")
    assert ref64.mean() > 0.01
    assert rel < BENCH_FAST_TOL, rel
    assert rel < 0.1 * noise, (rel, noise)
    s.close()


@pytest.mark.parametrize("rng", [wl.RNG_TEA_LCG, wl.RNG_PCG32])
def test_rng_streams(ctx, oracle, rng):
    pix = np.array([0, 1, 77, 65535, 1 << 20, 2073599], np.uint32)
    d_pix = torch.from_numpy(pix.view(np.int32)).cuda()
    out = torch.empty(len(pix) * 40, dtype=torch.float32, device="cuda")
    ctx.debug_rng(rng, 12345, d_pix.data_ptr(), len(pix), 9, 40, out.data_ptr())
    ctx.sync()
    got = out.cpu().numpy().reshape(len(pix), 40)
    for i, px in enumerate(pix):
        assert np.array_equal(bits(got[i]), bits(oracle.rng_stream(rng, 12345, int(px), 9, 40)))


def test_ldr_tonemap(ctx, oracle):
    sc = scenes.cornell_box(32, 32)
    p = wl.render_params(32, 32, 2, math=wl.MATH_STRICT)
    img, _, film, _ = gpu_render(ctx, sc, p)
    ldr = film.download_ldr()
    rad = np.clip(img.reshape(-1, 3), 0, 1e30)
    exp = (oracle.ace(rad) * np.float32(255.0)).astype(np.uint8).reshape(32, 32, 3)
    assert np.array_equal(ldr[..., :3], exp) and (ldr[..., 3] == 255).all()


def test_render_errors(ctx):
    sc = scenes.cornell_box(16, 16)
    s = wl.Scene(ctx, sc, build=False)
    film = wl.Film(ctx, 16, 16)
    with pytest.raises(wl.WlError, match="NOT_BUILT"):
        wl.render(ctx, s, sc.camera_struct(), wl.render_params(16, 16, 1), film)
    s.build_bvh()
    with pytest.raises(wl.WlError, match="INVALID_ARG"):
        wl.render(ctx, s, sc.camera_struct(), wl.render_params(16, 8, 1), film)
    with pytest.raises(wl.WlError, match="INVALID_ARG"):
        wl.render(ctx, s, sc.camera_struct(), wl.render_params(16, 16, 0), film)


def test_path_tracer_program(ctx, oracle):
    """PathTracingProgramManager-style use: Setup, Update per frame, End."""
    sc = scenes.cornell_box(24, 24)
    s = wl.Scene(ctx, sc)
    pt = wl.PathTracer(ctx, s, sc.camera_struct(), 24, 24, math=wl.MATH_STRICT)
    pt.Setup()
    for _ in range(3):
        pt.Update(1)
    img = pt.film.download()
    pt.End()
    ref, _, _ = oracle.render(sc, ocam(sc), oparams(wl.render_params(24, 24, 3, math=wl.MATH_STRICT)))
    assert np.array_equal(bits(img), bits(ref))


def test_program_pt_golden_strict(ctx):
    """GPU strict mode == the reference's PathTracing.cu program itself (vertex normals, Disney
    lobes, four lights; the program's background is 0), bit for bit."""
    g = dict(np.load(os.path.join(GOLD, "program_pt_sphere_48x32_4spp.npz")))
    sc = small_sphere(48, 32)
    assert np.array_equal(sc.V, g["V"]) and np.array_equal(sc.I, g["I"])
    p = wl.render_params(48, 32, 4, math=wl.MATH_STRICT, env=(0.0, 0.0, 0.0))
    img, _, _, _ = gpu_render(ctx, sc, p)
    assert np.array_equal(bits(img), bits(g["image"]))


@pytest.mark.parametrize("strategy", [wl.STRATEGY_MIS, wl.STRATEGY_BDPT])
def test_graph_replay_matches_launches(ctx, strategy):
    """WL_RENDER_GRAPH: every wave replays one captured graph (several waves per call, two calls
    reusing the graph with new frames); the image equals direct launches bit for bit."""
    sc = small_sphere(40, 30)
    kw = dict(math=wl.MATH_STRICT, strategy=strategy, wave_paths=1500,
              max_depth=10 if strategy == wl.STRATEGY_BDPT else 12)
    imgs = []
    for flags in (0, wl._abi.RENDER_GRAPH):
        s = wl.Scene(ctx, sc)
        film = wl.Film(ctx, 40, 30)
        for first in (0, 3):
            p = wl.render_params(40, 30, 3, first_frame=first, flags=flags, **kw)
            wl.render(ctx, s, sc.camera_struct(), p, film)
        imgs.append(film.download())
        film.close()
        s.close()
    assert imgs[0].max() > 0
    assert np.array_equal(bits(imgs[0]), bits(imgs[1]))


def test_sorted_shading_keeps_the_image(ctx):
    """WL_RENDER_SORT_MATERIALS (each shading block counting-sorted by miss / emitter / material
    before shading): the same strict image as unsorted shading, bit for bit, for a single render
    and for a batch mixing two scenes."""
    sc = small_sphere(40, 30)
    cb = scenes.cornell_box(24, 20)
    imgs = []
    for flags in (0, wl._abi.RENDER_SORT_MATERIALS):
        s = wl.Scene(ctx, sc)
        film = wl.Film(ctx, 40, 30)
        p = wl.render_params(40, 30, 3, math=wl.MATH_STRICT, env=sc.env, flags=flags, wave_paths=1500)
        wl.render(ctx, s, sc.camera_struct(), p, film)
        imgs.append(film.download())
        film.close()
        jobs = [(sc, s), (cb, wl.Scene(ctx, cb))]
        films = [wl.Film(ctx, d.width, d.height) for d, _ in jobs]
        ps = [wl.render_params(d.width, d.height, 2, math=wl.MATH_STRICT, env=d.env, flags=flags)
              for d, _ in jobs]
        wl.render_batch(ctx, [o for _, o in jobs], [d.camera_struct() for d, _ in jobs], ps, films)
        imgs += [f.download() for f in films]
        for f in films:
            f.close()
        for _, o in jobs:
            o.close()
    assert imgs[0].max() > 0
    for a, b in zip(imgs[:3], imgs[3:]):
        assert np.array_equal(bits(a), bits(b))


def test_tuned_shapes_keep_the_image(ctx):
    """The autotuner's knobs change scheduling only: any shape renders the same strict image,
    and wl_autotune returns a valid shape that it keeps for later renders."""
    sc = small_sphere(48, 32)
    s = wl.Scene(ctx, sc)
    p = wl.render_params(48, 32, 4, math=wl.MATH_STRICT)
    imgs = []
    for tune in (None, dict(wave_paths=1 << 12, extend_ctas_per_sm=4, extend_refill=8,
                            shadow_ctas_per_sm=6, shadow_refill=24, extend_postpone=0,
                            shadow_postpone=32, shadow_far_first=1),
                 dict(wave_paths=1 << 13, extend_ctas_per_sm=0, extend_refill=4,
                      shadow_ctas_per_sm=0, shadow_refill=4, extend_postpone=32,
                      shadow_postpone=0)):
        ctx.set_tune(tune)
        film = wl.Film(ctx, 48, 32)
        wl.render(ctx, s, sc.camera_struct(), p, film)
        imgs.append(film.download())
        film.close()
    assert np.array_equal(bits(imgs[0]), bits(imgs[1]))
    assert np.array_equal(bits(imgs[0]), bits(imgs[2]))
    r = ctx.autotune(s, sc.camera_struct(), wl.render_params(48, 32, 64))
    assert r["candidates"] >= 40 and r["extend_refill"] in (4, 6, 8, 12, 16, 24)
    assert 0 < r["ms_tuned"] <= r["ms_default"] * 1.5
    film = wl.Film(ctx, 48, 32)
    wl.render(ctx, s, sc.camera_struct(), p, film)
    assert np.array_equal(bits(film.download()), bits(imgs[0]))
    film.close()
    # the bidirectional program's connection rays take the shadow pass's any-hit order
    bp = wl.render_params(48, 32, 2, strategy=wl.STRATEGY_BDPT, max_depth=6, math=wl.MATH_STRICT)
    bimgs = []
    for far in (0, 1):
        ctx.set_tune(dict(wave_paths=0, extend_ctas_per_sm=0, extend_refill=12, shadow_ctas_per_sm=0,
                          shadow_refill=12, shadow_far_first=far))
        film = wl.Film(ctx, 48, 32)
        wl.render(ctx, s, sc.camera_struct(), bp, film)
        bimgs.append(film.download())
        film.close()
    assert bimgs[0].max() > 0 and np.array_equal(bits(bimgs[0]), bits(bimgs[1]))
    ctx.set_tune(None)
    s.close()


def test_batch_matches_separate_renders(ctx):
    """wl_render_batch: jobs of different scenes, sizes, spp, depths and random streams share
    waves (small waves make jobs span several, and waves span several jobs); every film equals
    the film of a separate wl_render call bit for bit."""
    jobs = [
        (scenes.cornell_box(40, 30), dict(spp=3, max_depth=8)),
        (small_sphere(48, 32), dict(spp=5, max_depth=12, rng=wl.RNG_PCG32, seed=9)),
        (scenes.glass_sphere(32, 32, subdiv=10), dict(spp=2, max_depth=6, first_frame=4)),
        (scenes.cornell_box(17, 13), dict(spp=7, max_depth=3, strategy=wl.STRATEGY_NEE)),
    ]
    ctx.set_tune(dict(wave_paths=1500, extend_ctas_per_sm=0, extend_refill=12,
                      shadow_ctas_per_sm=0, shadow_refill=12))
    try:
        objs, params, films, refs = [], [], [], []
        for sc, kw in jobs:
            kw = dict(kw)
            spp = kw.pop("spp")
            p = wl.render_params(sc.width, sc.height, spp, math=wl.MATH_STRICT, env=sc.env, **kw)
            s = wl.Scene(ctx, sc)
            objs.append(s)
            params.append(p)
            films.append(wl.Film(ctx, sc.width, sc.height))
            rf = wl.Film(ctx, sc.width, sc.height)
            wl.render(ctx, s, sc.camera_struct(), p, rf)
            refs.append(rf.download())
            rf.close()
        wl.render_batch(ctx, objs, [sc.camera_struct() for sc, _ in jobs], params, films)
        for f, r in zip(films, refs):
            assert r.max() > 0
            assert np.array_equal(bits(f.download()), bits(r))
        for f in films:
            f.close()
        # WL_RENDER_GRAPH: the whole batch is one captured graph, replayed by a second call with
        # other frames (the jobs table changes, the graph does not); both equal separate renders
        for shift in (0, 11):
            gparams, gfilms, grefs = [], [], []
            for (sc, _), s, p in zip(jobs, objs, params):
                q = wl.render_params(p.width, p.height, p.spp, math=wl.MATH_STRICT, env=sc.env,
                                     max_depth=p.max_depth, rng=p.rng, seed=p.seed,
                                     strategy=p.strategy, first_frame=p.first_frame + shift,
                                     flags=wl._abi.RENDER_GRAPH)
                gparams.append(q)
                gfilms.append(wl.Film(ctx, sc.width, sc.height))
                rf = wl.Film(ctx, sc.width, sc.height)
                r = wl.render_params(p.width, p.height, p.spp, math=wl.MATH_STRICT, env=sc.env,
                                     max_depth=p.max_depth, rng=p.rng, seed=p.seed,
                                     strategy=p.strategy, first_frame=p.first_frame + shift)
                wl.render(ctx, s, sc.camera_struct(), r, rf)
                grefs.append(rf.download())
                rf.close()
            wl.render_batch(ctx, objs, [sc.camera_struct() for sc, _ in jobs], gparams, gfilms)
            for f, r in zip(gfilms, grefs):
                assert np.array_equal(bits(f.download()), bits(r))
                f.close()
        # batches run the path tracer; a bidirectional job is refused, not rendered another way
        sc0 = jobs[0][0]
        bd = wl.render_params(sc0.width, sc0.height, 2, strategy=wl.STRATEGY_BDPT, max_depth=6)
        bf = wl.Film(ctx, sc0.width, sc0.height)
        with pytest.raises(wl.WlError, match="INVALID_ARG.*path tracer"):
            wl.render_batch(ctx, objs[:1], [sc0.camera_struct()], [bd], [bf])
        bf.close()
        for s in objs:
            s.close()
    finally:
        ctx.set_tune(None)


def test_textured_strict_vs_oracle(ctx, oracle, tmp_path):
    """A texture (bilinear, wrapping, normalised RGBA8) on two walls: strict mode (software filter
    with the texture unit's documented arithmetic) equals the oracle bit for bit; fast mode (the
    texture unit itself) is within the relMSE tolerance of the FP64 oracle; the film's PNG has
    the film's size."""
    sc = scenes.textured_cornell_box(48, 40)
    p = wl.render_params(48, 40, 4, math=wl.MATH_STRICT, max_depth=8)
    img, _, film, _ = gpu_render(ctx, sc, p)
    ref, _, _ = oracle.render(sc, ocam(sc), oparams(p))
    assert np.array_equal(bits(img), bits(ref))
    plain = scenes.cornell_box(48, 40)
    ref_plain, _, _ = oracle.render(plain, ocam(plain), oparams(p))
    assert np.abs(ref - ref_plain).max() > 0.05  # the texture shows
    film.save_png(tmp_path / "t.png")
    from wayland_b200.png import read_png
    assert read_png(tmp_path / "t.png").shape == (40, 48, 4)
    pf = wl.render_params(48, 40, 64, max_depth=8)
    _, img64, _, _ = gpu_render(ctx, sc, pf, fp64=True)
    _, ref64, _ = oracle.render(sc, ocam(sc), oparams(pf), prec=1, want64=True)
    rel = float(((img64 - ref64) ** 2 / (ref64 ** 2 + 1e-2)).mean())
    assert rel < FAST_RELMSE_TOL


def test_pbrt_scene_strict_vs_oracle(ctx, oracle, tmp_path):
    """A scene read from a pbrt-v3 file (trianglemesh, binary PLY, matte/plastic/disney/glass,
    texture, area light) renders bit-exactly like the oracle in strict mode."""
    from wayland_b200 import pbrt
    from pbrt_fixture import write_scene
    sc = pbrt.load(str(write_scene(tmp_path)))
    p = wl.render_params(sc.width, sc.height, sc.spp, math=wl.MATH_STRICT, max_depth=sc.max_depth)
    img, _, _, _ = gpu_render(ctx, sc, p)
    ref, _, _ = oracle.render(sc, ocam(sc), oparams(p))
    assert img.max() > 0
    assert np.array_equal(bits(img), bits(ref))


def test_distributed_film_reduction_one_rank(ctx):
    """render_distributed over an NCCL group of one rank: the film's FP64 sums are all-reduced on
    the device (through the CUDA array interface) and equal the single render's FP64 mean."""
    import socket
    import torch
    import torch.distributed as dist
    from wayland_b200 import multi
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        sc = scenes.cornell_box(40, 30)
        s = wl.Scene(ctx, sc)
        p = wl.render_params(40, 30, 6, max_depth=8)
        film = wl.Film(ctx, 40, 30, fp64=True)
        img, n = multi.render_distributed(wl, ctx, s, sc.camera_struct(), p, film, 0, 1)
        assert n == 6
        ref = wl.Film(ctx, 40, 30, fp64=True)
        wl.render(ctx, s, sc.camera_struct(), p, ref)
        assert np.allclose(img.cpu().numpy(), ref.download64(), rtol=1e-12, atol=1e-14)
        film.close()
        ref.close()
        s.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("rng", [wl.RNG_TEA_LCG, wl.RNG_PCG32])
def test_power_lights_strict_vs_oracle(ctx, oracle, rng):
    """WL_LIGHTS_POWER: emissive triangles chosen from the FP64 CDF (built on the GPU in a fixed
    order, area x luminance weights); strict mode equals the oracle bit for bit, and the image
    converges to the uniform-selection image (same expectation, different noise)."""
    sc = small_sphere(48, 32)
    sc.lights["L"] = np.array([[20, 18, 16], [1, 1, 1], [5, 2, 1], [0.5, 3, 6]], np.float32)
    p = wl.render_params(48, 32, 4, math=wl.MATH_STRICT, lights=wl.LIGHTS_POWER, rng=rng, seed=3)
    img, _, _, _ = gpu_render(ctx, sc, p)
    ref, _, _ = oracle.render(sc, ocam(sc), oparams(p))
    assert np.array_equal(bits(img), bits(ref))
    a = wl.render_params(48, 32, 256, lights=wl.LIGHTS_POWER)
    b = wl.render_params(48, 32, 256, lights=wl.LIGHTS_UNIFORM)
    _, ia, _, _ = gpu_render(ctx, sc, a, fp64=True)
    _, ib, _, _ = gpu_render(ctx, sc, b, fp64=True)
    assert abs(ia.mean() - ib.mean()) < 0.02 * ib.mean()


def test_user_stream_orders_the_whole_render(ctx):
    """A render issued on a caller's stream (wl_context_set_stream) is ordered on that stream as a
    whole: the library's second stream, which runs the shadow passes, joins back before the
    render's last kernel. A copy of the film enqueued on the caller's stream right after the call,
    with no other synchronisation, reads the finished image: the strict image of the same render
    on the context's own stream, bit for bit."""
    from wayland_b200.multi import _DeviceArray
    sc = small_sphere(48, 32)
    s = wl.Scene(ctx, sc)
    p = wl.render_params(48, 32, 8, math=wl.MATH_STRICT, env=sc.env)
    ref = wl.Film(ctx, 48, 32)
    wl.render(ctx, s, sc.camera_struct(), p, ref)
    expected = ref.download()
    ref.close()
    user = torch.cuda.Stream()
    ctx.set_stream(user.cuda_stream)
    try:
        film = wl.Film(ctx, 48, 32)
        wl.render(ctx, s, sc.camera_struct(), p, film)
        rgb = film.device_ptrs()[0]
        with torch.cuda.stream(user):
            view = torch.as_tensor(_DeviceArray(rgb, (32, 48, 3), "<f4"), device="cuda")
            got = view.clone()
        user.synchronize()
        got = got.cpu().numpy()
        film.close()
    finally:
        ctx.set_stream(None)
    assert expected.max() > 0
    assert np.array_equal(bits(got), bits(expected))
    s.close()
