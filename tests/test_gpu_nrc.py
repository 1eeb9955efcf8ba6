"""The radiance-cache network on the GPU against the FP64 CPU oracle (oracle/nrc_oracle.py):
forward outputs and weight gradients, a training run that fits a target function, and a render
in which the cache answers the queries. Tolerances: outputs within 2e-2 relative (bfloat16
activations can round differently when FP32 and FP64 sums straddle a rounding boundary; the
median error must be below 1e-4); gradients within 5e-3 of the largest entry."""
import numpy as np
import pytest
import torch

import nrc_oracle
import wayland_b200 as wl
from wayland_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cache(ctx):
    sc = scenes.cornell_box(32, 32)
    s = wl.Scene(ctx, sc)
    c = wl.RadianceCache(ctx, s, log2_table=16)
    yield c, s, sc
    c.close()
    s.close()


def batch(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, (n, 64)).astype(np.float32)
    x[:, 59] = 1.0
    t = np.zeros((n, 4), np.float32)
    t[:, 0] = np.abs(np.sin(3 * x[:, 0]) + x[:, 1] ** 2)
    t[:, 1] = np.abs(np.cos(2 * x[:, 2])) * 0.5
    t[:, 2] = np.abs(x[:, 3] * x[:, 4])
    return x, t


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_forward_matches_oracle(cache):
    c, _, _ = cache
    x, _ = batch(4096, 1)
    out = torch.empty((4096, 4), dtype=torch.float32, device="cuda")
    dx = dev(x)
    c.forward(dx.data_ptr(), out.data_ptr(), 4096)
    c.ctx.sync()
    got = out.cpu().numpy()[:, :3]
    ref, _ = nrc_oracle.forward(c.weights(), x)
    ref = ref[:, :3]
    err = np.abs(got - ref) / (np.abs(ref) + 1e-2)
    assert np.median(err) < 1e-4 and err.max() < 2e-2, (np.median(err), err.max())


def test_gradients_match_oracle(cache):
    c, _, _ = cache
    x, t = batch(3000, 2)
    dx, dt = dev(x), dev(t)
    g = c.gradients(dx.data_ptr(), dt.data_ptr(), 3000)
    loss, ref = nrc_oracle.gradients(c.weights(), x, t)
    scale = np.abs(ref).max()
    assert scale > 0
    assert np.abs(g - ref).max() < 5e-3 * scale, (np.abs(g - ref).max(), scale)


@pytest.mark.parametrize("n", [20000, 40000, 65536])
def test_gradients_many_tiles_per_cta(cache, n):
    """Batches of 2 to 4 tiles of 128 rows per CTA (the training kernel keeps two in flight and
    accumulates every tile's weight gradient in tensor memory), with a ragged last tile: the
    gradient matches the oracle and is the same bit for bit on a second run (fixed order)."""
    c, _, _ = cache
    x, t = batch(n, 10 + n)
    dx, dt = dev(x), dev(t)
    g = c.gradients(dx.data_ptr(), dt.data_ptr(), n)
    _, ref = nrc_oracle.gradients(c.weights(), x, t)
    scale = np.abs(ref).max()
    assert scale > 0
    assert np.abs(g - ref).max() < 5e-3 * scale, (np.abs(g - ref).max(), scale)
    g2 = c.gradients(dx.data_ptr(), dt.data_ptr(), n)
    assert np.array_equal(g.view(np.uint32), g2.view(np.uint32))


def test_training_fits(ctx):
    sc = scenes.cornell_box(16, 16)
    s = wl.Scene(ctx, sc)
    c = wl.RadianceCache(ctx, s, log2_table=12, learning_rate=5e-3)
    x, t = batch(16384, 3)
    dx, dt = dev(x), dev(t)
    first = c.train_step(dx.data_ptr(), dt.data_ptr(), 16384)
    for _ in range(300):
        last = c.train_step(dx.data_ptr(), dt.data_ptr(), 16384)
    assert last < 0.25 * first, (first, last)
    c.close()
    s.close()


def test_render_with_cache(ctx):
    sc = scenes.cornell_box(64, 48)
    s = wl.Scene(ctx, sc)
    c = wl.RadianceCache(ctx, s, log2_table=16, train_paths=512)
    film = wl.Film(ctx, 64, 48)
    p = wl.render_params(64, 48, 8, max_depth=8)
    wl.render_nrc(ctx, s, sc.camera_struct(), p, c, film)
    img = film.download()
    st = c.stats()
    assert np.isfinite(img).all() and img.mean() > 0.01
    assert st["train_samples"] > 100 and st["queries"] > 1000
    assert np.isfinite(st["loss"])
    c.close()
    s.close()


def test_reserve_and_warmup_without_film(ctx):
    """wl_nrc_reserve allocates up front; frames without a film train the cache only."""
    sc = scenes.cornell_box(48, 32)
    s = wl.Scene(ctx, sc)
    c = wl.RadianceCache(ctx, s, log2_table=14, train_paths=256)
    p = wl.render_params(48, 32, 3, max_depth=8)
    c.reserve(p)
    wl.render_nrc(ctx, s, sc.camera_struct(), p, c, None)
    st = c.stats()
    assert st["train_samples"] > 50 and np.isfinite(st["loss"])
    film = wl.Film(ctx, 48, 32)
    wl.render_nrc(ctx, s, sc.camera_struct(), wl.render_params(48, 32, 2, max_depth=8), c, film)
    img = film.download()
    assert np.isfinite(img).all() and img.mean() > 0.01
    film.close()
    c.close()
    s.close()


def test_self_training_matches_full_paths(ctx):
    """Training paths that end at the cache after train_extra vertices and full-length training
    paths converge to images of the same brightness (the cache learns the multi-bounce tail)."""
    sc = scenes.cornell_box(48, 48)
    s = wl.Scene(ctx, sc)
    means = []
    for extra in (0, 3):
        c = wl.RadianceCache(ctx, s, log2_table=16, train_paths=1024, train_extra=extra)
        wl.render_nrc(ctx, s, sc.camera_struct(), wl.render_params(48, 48, 32, max_depth=12), c, None)
        film = wl.Film(ctx, 48, 48)
        wl.render_nrc(ctx, s, sc.camera_struct(), wl.render_params(48, 48, 32, max_depth=12), c, film)
        means.append(float(film.download().mean()))
        film.close()
        c.close()
    ref_film = wl.Film(ctx, 48, 48)
    wl.render(ctx, s, sc.camera_struct(), wl.render_params(48, 48, 256, max_depth=12), ref_film)
    ref = float(ref_film.download().mean())
    ref_film.close()
    s.close()
    for m in means:
        assert abs(m - ref) < 0.1 * ref, (means, ref)


def test_wait_timeout_reported(ctx):
    """A tensor-core wait that gives up is reported, and the cache keeps working: with the wait
    limit at 0 polls every mbarrier wait of the forward kernel gives up at once; the kernel
    records the error, drains the tensor-core work it issued, frees its tensor memory and
    returns; wl_nrc_stats returns WL_ERR_TIMEOUT once. With the limit restored the next forward
    pass is correct again."""
    sc = scenes.cornell_box(16, 16)
    s = wl.Scene(ctx, sc)
    c = wl.RadianceCache(ctx, s, log2_table=12)
    x, _ = batch(1024, 5)
    out = torch.zeros((1024, 4), dtype=torch.float32, device="cuda")
    dx = dev(x)
    c.set_wait_limit(0)
    c.forward(dx.data_ptr(), out.data_ptr(), 1024)
    ctx.sync()
    with pytest.raises(wl.WlError, match="TIMEOUT"):
        c.stats()
    c.stats()  # reported once
    c.set_wait_limit(wl._abi.NRC_WAIT_POLLS)
    c.forward(dx.data_ptr(), out.data_ptr(), 1024)
    ctx.sync()
    ref, _ = nrc_oracle.forward(c.weights(), x)
    err = np.abs(out.cpu().numpy()[:, :3] - ref[:, :3]) / (np.abs(ref[:, :3]) + 1e-2)
    assert err.max() < 2e-2
    c.stats()
    c.close()
    s.close()
