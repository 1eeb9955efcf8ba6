"""The radiance cache's hash-grid half on the GPU against the FP64 CPU oracle
(oracle/nrc_oracle.py), on surface points of the door-slit room (the cache's benchmark scene):

- the table entry of every level's 8 cell corners: bit-exact;
- the 64 encoded inputs as the query pass stores them (bfloat16): each within one bfloat16 rounding
  step of the oracle's value plus 1e-6 (the device interpolates in FP32, the oracle in FP64: a sum
  next to a rounding boundary may round the other way, and a sum that cancels to nearly zero keeps
  the FP32 rounding error of its 8 terms, below 8 x 2^-24 for features of magnitude <= 1);
- the render's query path (encode into tiles, tcgen05 MLP): predictions within 5e-2 relative,
  99 % of them within 1e-2 and the median below 1e-4 (an input that rounds one bfloat16 step
  apart moves the outputs by up to a few percent);
- one training step through the render's training path (encode, fused tensor-core forward and
  backward, grid scatter): weight gradients and hash-grid gradients within 1e-2 of the largest
  entry (FP32 atomics sum the grid gradient in an arbitrary order), loss within 1e-3 relative.
"""
import numpy as np
import pytest
import torch

import nrc_oracle
import wayland_b200 as wl
from wayland_b200 import _abi, scenes

pytestmark = pytest.mark.gpu

N = 4096


def surface_vertices(sc, n, seed):
    """n uniform points on the scene's triangles (area weighted) with the geometric normal
    facing a random outgoing direction of its hemisphere, the triangle's material and
    targets drawn in [0, 2)."""
    rng = np.random.default_rng(seed)
    V, I = sc.V.astype(np.float64), sc.I.astype(np.int64)
    a, b, c = V[I[:, 0]], V[I[:, 1]], V[I[:, 2]]
    area = 0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1)
    t = rng.choice(len(I), size=n, p=area / area.sum())
    s1 = np.sqrt(rng.uniform(size=(n, 1)))
    s2 = rng.uniform(size=(n, 1))
    p = a[t] * (1 - s1) + b[t] * (s1 * (1 - s2)) + c[t] * (s1 * s2)
    ng = np.cross(b[t] - a[t], c[t] - a[t])
    ng /= np.linalg.norm(ng, axis=1, keepdims=True)
    wo = rng.normal(size=(n, 3))
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    wo = np.where((wo * ng).sum(1, keepdims=True) < 0, -wo, wo)
    v = np.zeros(n, _abi.NRC_VERTEX_DTYPE)
    v["pos"] = p
    v["material"] = sc.tri_material[t]
    v["wo"] = wo
    v["n"] = ng
    v["extra"][:, :3] = rng.uniform(0.0, 2.0, (n, 3))
    return v


@pytest.fixture(scope="module")
def setup(ctx):
    sc = scenes.door_slit_room(64, 64)
    scene = wl.Scene(ctx, sc)
    cache = wl.RadianceCache(ctx, scene, log2_table=14)
    desc, _ = cache.grid(with_params=False)
    rng = np.random.default_rng(7)
    params = rng.uniform(-1.0, 1.0, (desc["levels"], 1 << desc["log2_table"], 2)).astype(np.float32)
    cache.set_grid(params)
    g = nrc_oracle.GridDesc(desc["levels"], desc["log2_table"], desc["base_resolution"],
                            desc["per_level_scale"], desc["lo"], desc["inv_ext"])
    v = surface_vertices(sc, N, 3)
    dv = torch.from_numpy(v.view(np.uint8).copy()).cuda()
    yield cache, g, params, v, dv, sc
    cache.close()
    scene.close()


def test_corner_indices_bit_exact(setup):
    cache, g, params, v, dv, sc = setup
    feat = torch.empty((N, 64), dtype=torch.float32, device="cuda")
    corners = torch.empty((N, g.levels, 8), dtype=torch.int32, device="cuda")
    cache.debug_encode(dv.data_ptr(), N, feat.data_ptr(), corners.data_ptr())
    cache.ctx.sync()
    idx, _ = nrc_oracle.grid_corners(g, v["pos"])
    got = corners.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, idx)
    # both index paths occur: dense coarse levels and hashed fine levels
    dense = [(g.res(l) + 1) ** 3 <= (1 << g.log2T) for l in range(g.levels)]
    assert any(dense) and not all(dense)


def test_encoded_inputs_match_oracle(setup):
    cache, g, params, v, dv, sc = setup
    feat = torch.empty((N, 64), dtype=torch.float32, device="cuda")
    cache.debug_encode(dv.data_ptr(), N, feat.data_ptr())
    cache.ctx.sync()
    got = feat.cpu().numpy().astype(np.float64)
    ref = nrc_oracle.encode(g, params, v, sc.mats)
    # one bfloat16 step: 2^-7 of the magnitude (8 significant bits)
    step = np.maximum(np.abs(ref), np.abs(got)) * 2.0 ** -7 + 1e-6
    bad = np.abs(got - ref) > step
    assert not bad.any(), (np.argwhere(bad)[:5], got[bad][:5], ref[bad][:5])
    assert (got == ref).mean() > 0.98
    assert np.abs(ref[:, :32]).mean() > 0.05  # the grid features are not trivially small


def test_query_matches_oracle(setup):
    cache, g, params, v, dv, sc = setup
    out = torch.empty((N, 4), dtype=torch.float32, device="cuda")
    cache.query(dv.data_ptr(), N, out.data_ptr())
    cache.ctx.sync()
    got = out.cpu().numpy()
    assert (got[:, 3] == 0).all()
    ref = nrc_oracle.query(cache.weights(), g, params, v, sc.mats)
    err = np.abs(got[:, :3] - ref) / (np.abs(ref) + 1e-2)
    assert np.median(err) < 1e-4 and np.quantile(err, 0.99) < 1e-2 and err.max() < 5e-2, \
        (np.median(err), np.quantile(err, 0.99), err.max())
    assert (ref > 0).mean() > 0.1


def test_training_gradients_match_oracle(setup):
    cache, g, params, v, dv, sc = setup
    loss, gw, gg = cache.sample_gradients(dv.data_ptr(), N)
    ref_loss, ref_w, ref_g = nrc_oracle.sample_gradients(cache.weights(), g, params, v, sc.mats)
    assert abs(loss - ref_loss) <= 1e-3 * abs(ref_loss), (loss, ref_loss)
    sw = np.abs(ref_w).max()
    assert np.abs(gw - ref_w).max() < 1e-2 * sw, (np.abs(gw - ref_w).max(), sw)
    sg = np.abs(ref_g).max()
    assert sg > 0
    assert np.abs(gg - ref_g).max() < 1e-2 * sg, (np.abs(gg - ref_g).max(), sg)
    # entries no sample reaches keep a zero gradient on the device too
    assert (gg[ref_g == 0] == 0).all()
    assert (ref_g != 0).sum() > 1000
    # a second call starts from a zeroed grid gradient again
    loss2, _, gg2 = cache.sample_gradients(dv.data_ptr(), N)
    assert np.abs(gg2 - gg).max() < 1e-3 * sg and abs(loss2 - loss) <= 1e-6 * abs(loss)
