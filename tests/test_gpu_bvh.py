"""GPU BVH build and ray casts through the C ABI against the oracle: Morton codes and radix-tree
topology bit-exact, closest hits (t, prim, u, v) bit-exact against brute force, any-hit
occlusion identical, plus size-independent properties at the full benchmark size."""
import numpy as np
import pytest
import torch

import wayland_b200 as wl
from helpers import axis_rays, degenerate_rays, geometries, random_rays
from wayland_b200 import scenes

pytestmark = pytest.mark.gpu
GEOMS = geometries()


class Geo:
    def __init__(self, V, I):
        self.V = np.ascontiguousarray(V, np.float32)
        self.I = np.ascontiguousarray(I, np.uint32)
        self.N = None
        self.tri_flags = None
        self.tri_material = np.zeros(len(self.I), np.uint32)
        self.mats = np.array([scenes.matte((0.5, 0.5, 0.5))])
        self.lights = np.zeros(0, wl._abi.LIGHT_DTYPE)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()


def cast_device(ctx, sc, rays, mode):
    d_r = dev(rays)
    d_h = torch.empty(len(rays) * 16, dtype=torch.uint8, device="cuda")
    sc.cast(d_r.data_ptr(), d_h.data_ptr(), len(rays), mode)
    ctx.sync()
    return d_h.cpu().numpy().view(wl.HIT_DTYPE)


def hits_equal(a, b):
    return np.array_equal(a.view(np.uint32).reshape(-1, 4), b.view(np.uint32).reshape(-1, 4))


@pytest.mark.parametrize("name,V,I", GEOMS, ids=[g[0] for g in GEOMS])
def test_build_topology(ctx, oracle, name, V, I):
    g = Geo(V, I)
    sc = wl.Scene(ctx, g)
    assert np.array_equal(sc.export_morton(), oracle.morton63(g.V, g.I))
    sp, left, right, parent, bounds = sc.export_binary()
    osp, ol, orr, opar, ob = oracle.lbvh(g.V, g.I)
    assert np.array_equal(sp, osp)
    assert np.array_equal(left, ol) and np.array_equal(right, orr)
    assert np.array_equal(parent, opar)
    assert np.array_equal(bounds.view(np.uint32), ob.view(np.uint32))
    info = sc.info()
    assert info["leaf_tris"] == len(g.I) and 1 <= info["wide_depth"] <= 64
    sc.close()


@pytest.mark.parametrize("name,V,I", GEOMS, ids=[g[0] for g in GEOMS])
def test_cast_bitexact(ctx, oracle, name, V, I):
    g = Geo(V, I)
    sc = wl.Scene(ctx, g)
    rays = np.concatenate([random_rays(6000, 21), axis_rays(2000, 22)])
    if name == "cornell":
        rays["org"] = np.random.default_rng(4).uniform(0.01, 0.99, (len(rays), 3))
    ref = oracle.cast_bruteforce(g.V, g.I, rays, 0)
    got = cast_device(ctx, sc, rays, wl.CAST_CLOSEST)
    assert hits_equal(got, ref)
    assert hits_equal(sc.cast_host(rays, wl.CAST_CLOSEST), ref)
    anyr = oracle.cast_bruteforce(g.V, g.I, rays, 1)
    anyg = cast_device(ctx, sc, rays, wl.CAST_ANY)
    assert np.array_equal(anyg["prim"] == wl.INVALID, anyr["prim"] == wl.INVALID)
    # any hits with a node's children visited far to near (the shadow pass's tunable order)
    ctx.set_tune(dict(wave_paths=0, extend_ctas_per_sm=0, extend_refill=12, shadow_ctas_per_sm=0,
                      shadow_refill=12, shadow_far_first=1))
    try:
        anyf = cast_device(ctx, sc, rays, wl.CAST_ANY)
    finally:
        ctx.set_tune(None)
    assert np.array_equal(anyf["prim"] == wl.INVALID, anyr["prim"] == wl.INVALID)
    sc.close()


def test_empty_scene(ctx):
    g = Geo(np.zeros((0, 3), np.float32), np.zeros((0, 3), np.uint32))
    sc = wl.Scene(ctx, g)
    h = sc.cast_host(random_rays(100, 1), wl.CAST_CLOSEST)
    assert (h["prim"] == wl.INVALID).all()
    sc.close()


@pytest.mark.parametrize("kind", [wl.BVH_LBVH, wl.BVH_SAH])
def test_degenerate_rays(ctx, oracle, kind):
    """wl_cast_rays takes device rays it cannot check on the host: NaN or zero directions,
    infinite or NaN origins and empty [tmin, tmax] end their traversal and hit nothing (closest
    and any hit, both any-hit child orders), like the brute force; valid rays in the same batch
    keep their hits bit for bit."""
    s = scenes.displaced_sphere(subdiv=24)
    sc = wl.Scene(ctx, s, bvh_kind=kind)
    bad = degenerate_rays(5)
    good = random_rays(500, 6, -3.0, 3.0)
    rays = np.concatenate([good[:250], bad, good[250:]])
    sl = slice(250, 250 + len(bad))
    ref = oracle.cast_bruteforce(s.V, s.I, rays, 0)
    got = cast_device(ctx, sc, rays, wl.CAST_CLOSEST)
    assert (got["prim"][sl] == wl.INVALID).all()
    assert hits_equal(got, ref)
    anyr = oracle.cast_bruteforce(s.V, s.I, rays, 1)
    for far in (0, 1):
        ctx.set_tune(dict(wave_paths=0, extend_ctas_per_sm=0, extend_refill=12, shadow_ctas_per_sm=0,
                          shadow_refill=12, shadow_far_first=far))
        try:
            anyg = cast_device(ctx, sc, rays, wl.CAST_ANY)
        finally:
            ctx.set_tune(None)
        assert (anyg["prim"][sl] == wl.INVALID).all()
        assert np.array_equal(anyg["prim"] == wl.INVALID, anyr["prim"] == wl.INVALID)
    sc.close()


def test_scene_validation(ctx):
    g = Geo(*scenes.random_triangles(10, 0))
    g.I = g.I.copy()
    g.I[3, 1] = 10 ** 6
    with pytest.raises(wl.WlError):
        wl.Scene(ctx, g)
    g = Geo(*scenes.random_triangles(10, 0))
    g.V = g.V.copy()
    g.V[2, 0] = np.nan
    with pytest.raises(wl.WlError):
        wl.Scene(ctx, g)


def test_cast_large_scene_vs_oracle_bvh(ctx, oracle):
    """200K-triangle displaced sphere, primary and surface-leaving rays, against the oracle's
    independent CPU BVH (equal to brute force by construction)."""
    s = scenes.displaced_sphere(subdiv=100)
    sc = wl.Scene(ctx, s)
    ob = oracle.bvh(s.V, s.I)
    prim = random_rays(40000, 31, -3.0, 3.0)
    ref = ob.cast(prim, 0)
    assert hits_equal(cast_device(ctx, sc, prim, wl.CAST_CLOSEST), ref)
    ok = ref["prim"] != wl.INVALID
    sec = random_rays(int(ok.sum()), 32)
    sec["org"] = (prim["org"][ok] + prim["dir"][ok] * ref["t"][ok][:, None]).astype(np.float32)
    assert hits_equal(cast_device(ctx, sc, sec, wl.CAST_CLOSEST), ob.cast(sec, 0))
    anyr = ob.cast(sec, 1)
    anyg = cast_device(ctx, sc, sec, wl.CAST_ANY)
    assert np.array_equal(anyg["prim"] == wl.INVALID, anyr["prim"] == wl.INVALID)
    sc.close()


def test_full_size_properties(ctx, oracle):
    """The benchmark's 2M-triangle scene: the build is a valid tree over a permutation of the
    triangles, the sorted Morton codes are non-decreasing and equal the oracle's, and a ray
    batch matches the oracle's CPU BVH bit for bit."""
    s = scenes.displaced_sphere()
    n = s.num_tris
    sc = wl.Scene(ctx, s)
    codes = sc.export_morton()
    assert np.array_equal(codes, oracle.morton63(s.V, s.I))
    sp, left, right, parent, bounds = sc.export_binary()
    assert np.array_equal(np.sort(sp), np.arange(n, dtype=np.uint32))
    assert (np.diff(codes[sp].astype(np.int64)) >= 0).all() or (np.diff(codes[sp]) >= 0).all()
    kids = np.concatenate([left, right])
    assert np.array_equal(np.sort(kids), np.arange(1, 2 * n - 1))
    assert parent[0] == -1 and (parent[1:] >= 0).all()
    info = sc.info()
    assert info["leaf_tris"] == n and info["wide_depth"] <= 64
    rays = random_rays(20000, 41, -3.0, 3.0)
    ob = oracle.bvh(s.V, s.I)
    assert hits_equal(cast_device(ctx, sc, rays, wl.CAST_CLOSEST), ob.cast(rays, 0))
    sc.close()


def check_binary_tree(sp, left, right, parent, bounds, n):
    """A valid binary BVH in the Karras layout: leaves n-1+p over a permutation of the triangles,
    every node but the root 0 the child of exactly one parent, and every internal node's box
    (and triangle count) the union (sum) of its children's."""
    assert np.array_equal(np.sort(sp), np.arange(n, dtype=np.uint32))
    if n == 1:
        return
    kids = np.concatenate([left, right])
    assert np.array_equal(np.sort(kids), np.arange(1, 2 * n - 1))
    assert parent[0] == -1
    idx = np.arange(n - 1)
    assert np.array_equal(parent[left], idx) and np.array_equal(parent[right], idx)
    b = bounds.reshape(-1, 6)
    lo = np.minimum(b[left, :3], b[right, :3])
    hi = np.maximum(b[left, 3:], b[right, 3:])
    assert np.array_equal(b[:n - 1, :3], lo) and np.array_equal(b[:n - 1, 3:], hi)


@pytest.mark.parametrize("name,V,I", GEOMS, ids=[g[0] for g in GEOMS])
def test_sah_build_and_cast(ctx, oracle, name, V, I):
    """Binned-SAH build: a valid binary tree over a permutation of the triangles (including
    coincident centroids, flat and degenerate triangles), the same Morton codes as the LBVH, and
    closest hits bit-exact against brute force with any-hit occlusion identical."""
    g = Geo(V, I)
    sc = wl.Scene(ctx, g, bvh_kind=wl.BVH_SAH)
    assert sc.info()["kind"] == wl.BVH_SAH
    assert np.array_equal(sc.export_morton(), oracle.morton63(g.V, g.I))
    check_binary_tree(*sc.export_binary(), len(g.I))
    rays = np.concatenate([random_rays(6000, 21), axis_rays(2000, 22)])
    if name == "cornell":
        rays["org"] = np.random.default_rng(4).uniform(0.01, 0.99, (len(rays), 3))
    assert hits_equal(cast_device(ctx, sc, rays, wl.CAST_CLOSEST), oracle.cast_bruteforce(g.V, g.I, rays, 0))
    anyr = oracle.cast_bruteforce(g.V, g.I, rays, 1)
    anyg = cast_device(ctx, sc, rays, wl.CAST_ANY)
    assert np.array_equal(anyg["prim"] == wl.INVALID, anyr["prim"] == wl.INVALID)
    sc.close()


@pytest.mark.parametrize("n", [2, 3, 32, 33, 34, 65, 2049, 5000])
def test_sah_sizes(ctx, oracle, n):
    """Triangle counts around the small-node limit (32) and the binning chunk (2048)."""
    V, I = scenes.random_triangles(n, 100 + n)
    g = Geo(V, I)
    sc = wl.Scene(ctx, g, bvh_kind=wl.BVH_SAH)
    check_binary_tree(*sc.export_binary(), n)
    rays = random_rays(3000, 7 + n)
    assert hits_equal(cast_device(ctx, sc, rays, wl.CAST_CLOSEST), oracle.cast_bruteforce(g.V, g.I, rays, 0))
    sc.close()


def test_sah_full_size(ctx, oracle):
    """The benchmark's 2M-triangle scene with the SAH build: a valid tree, the same tree on a
    second build (deterministic), fewer node visits than the LBVH for the same rays, and a ray
    batch bit-exact against the oracle's CPU BVH."""
    s = scenes.displaced_sphere()
    n = s.num_tris
    sc = wl.Scene(ctx, s, bvh_kind=wl.BVH_SAH)
    t1 = sc.export_binary()
    check_binary_tree(*t1, n)
    sc.build_bvh(wl.BVH_SAH)
    t2 = sc.export_binary()
    for a, b in zip(t1, t2):
        assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))
    assert sc.info()["wide_depth"] <= 64
    rays = random_rays(20000, 41, -3.0, 3.0)
    ob = oracle.bvh(s.V, s.I)
    assert hits_equal(cast_device(ctx, sc, rays, wl.CAST_CLOSEST), ob.cast(rays, 0))
    d_r = dev(rays)
    nodes_sah, _ = sc.cast_stats(d_r.data_ptr(), len(rays))
    lb = wl.Scene(ctx, s)
    nodes_lbvh, _ = lb.cast_stats(d_r.data_ptr(), len(rays))
    assert nodes_sah < nodes_lbvh
    lb.close()
    sc.close()
