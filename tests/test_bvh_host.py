"""The BVH build and traversal logic of wayland_b200/csrc/wl_bvh.cuh, compiled for the CPU by the
test harness, against the oracle: Morton codes and radix-tree topology bit-exact, closest hits
(t, prim, u, v) bit-exact against brute force, any-hit occlusion identical."""
import numpy as np
import pytest

import pyoracle as po
from helpers import axis_rays, degenerate_rays, geometries, random_rays

GEOMS = geometries()


def host_build(host_bvh, V, I):
    V = np.ascontiguousarray(V, np.float32)
    I = np.ascontiguousarray(I, np.uint32)
    return host_bvh.hb_build(V.ctypes.data, I.ctypes.data, len(I)), V, I


def host_cast(host_bvh, h, rays, mode):
    hits = np.zeros(len(rays), po.HIT_DTYPE)
    st = np.zeros(2, np.uint64)
    host_bvh.hb_cast(h, rays.ctypes.data, len(rays), mode, hits.ctypes.data, st.ctypes.data)
    return hits, st


@pytest.mark.parametrize("name,V,I", GEOMS, ids=[g[0] for g in GEOMS])
def test_topology(host_bvh, oracle, name, V, I):
    import ctypes as C
    h, V, I = host_build(host_bvh, V, I)
    n = len(I)
    mort = np.zeros(n, np.uint64)
    sp = np.zeros(n, np.uint32)
    L = np.zeros(max(n - 1, 1), np.int32)
    R = np.zeros(max(n - 1, 1), np.int32)
    host_bvh.hb_export(h, mort.ctypes.data, sp.ctypes.data, L.ctypes.data, R.ctypes.data)
    assert np.array_equal(mort, oracle.morton63(V, I))
    osp, ol, orr, _, _ = oracle.lbvh(V, I)
    assert np.array_equal(sp, osp)
    assert np.array_equal(L[:n - 1], ol) and np.array_equal(R[:n - 1], orr)
    depth = C.c_uint32()
    nodes = host_bvh.hb_info(h, C.byref(depth))
    assert nodes >= 1 and depth.value <= 64
    host_bvh.hb_destroy(h)


@pytest.mark.parametrize("name,V,I", GEOMS, ids=[g[0] for g in GEOMS])
def test_closest_hit_bitexact(host_bvh, oracle, name, V, I):
    h, V, I = host_build(host_bvh, V, I)
    rays = np.concatenate([random_rays(6000, 11), axis_rays(2000, 12)])
    if name == "cornell":
        rays["org"] = np.random.default_rng(2).uniform(0.01, 0.99, (len(rays), 3))
    got, st = host_cast(host_bvh, h, rays, 0)
    ref = oracle.cast_bruteforce(V, I, rays, 0)
    assert np.array_equal(got.view(np.uint32).reshape(-1, 4), ref.view(np.uint32).reshape(-1, 4))
    anyg, _ = host_cast(host_bvh, h, rays, 1)
    anyr = oracle.cast_bruteforce(V, I, rays, 1)
    assert np.array_equal(anyg["prim"] == po.np.uint32(0xFFFFFFFF), anyr["prim"] == 0xFFFFFFFF)
    anyf, _ = host_cast(host_bvh, h, rays, 2)  # children far to near
    assert np.array_equal(anyf["prim"] == po.np.uint32(0xFFFFFFFF), anyr["prim"] == 0xFFFFFFFF)
    host_bvh.hb_destroy(h)


def test_rays_from_surfaces(host_bvh, oracle):
    """Secondary rays starting at hit points on the surface they left (the path tracer's
    common case), in random directions."""
    from wayland_b200 import scenes
    sc = scenes.displaced_sphere(subdiv=24)
    h, V, I = host_build(host_bvh, sc.V, sc.I)
    prim = random_rays(6000, 7, -3.0, 3.0)
    hit = oracle.cast_bruteforce(V, I, prim, 0)
    ok = hit["prim"] != 0xFFFFFFFF
    assert ok.sum() > 1000
    rays = random_rays(int(ok.sum()), 8)
    p = prim[ok]
    rays["org"] = (p["org"] + p["dir"] * hit["t"][ok][:, None]).astype(np.float32)
    got, _ = host_cast(host_bvh, h, rays, 0)
    ref = oracle.cast_bruteforce(V, I, rays, 0)
    assert np.array_equal(got.view(np.uint32).reshape(-1, 4), ref.view(np.uint32).reshape(-1, 4))
    assert (ref["prim"] != 0xFFFFFFFF).mean() > 0.05
    host_bvh.hb_destroy(h)


def host_cast_batched(host_bvh, h, rays, mode, post, refill, node_steps=3):
    hits = np.zeros(len(rays), po.HIT_DTYPE)
    st = np.zeros(2, np.uint64)
    host_bvh.hb_cast_batched(h, rays.ctypes.data, len(rays), mode, post, refill, node_steps,
                             hits.ctypes.data, st.ctypes.data)
    return hits, st


@pytest.mark.parametrize("post,refill,node_steps", [(0, 4, 3), (8, 12, 3), (16, 8, 1), (24, 24, 2),
                                                    (32, 1, 3), (12, 6, 4)])
def test_batched_traversal_matches(host_bvh, oracle, post, refill, node_steps):
    """The GPU kernels' batched traversal (node and triangle phases chosen per warp, up to
    node_steps node visits per phase, postponed triangle groups, refill of idle lanes),
    simulated for one warp: closest hits bit-exact against brute force for every phase threshold,
    any-hit occlusion identical, and at least the node and triangle work of the one-lane
    traversal (the deferred triangle tests only delay culling)."""
    from wayland_b200 import scenes
    sc = scenes.displaced_sphere(subdiv=24)
    h, V, I = host_build(host_bvh, sc.V, sc.I)
    prim = random_rays(3000, 17, -3.0, 3.0)
    hit = oracle.cast_bruteforce(V, I, prim, 0)
    ok = hit["prim"] != 0xFFFFFFFF
    sec = random_rays(int(ok.sum()), 18)
    sec["org"] = (prim["org"][ok] + prim["dir"][ok] * hit["t"][ok][:, None]).astype(np.float32)
    rays = np.concatenate([prim, sec, axis_rays(500, 19)])
    ref = oracle.cast_bruteforce(V, I, rays, 0)
    got, st = host_cast_batched(host_bvh, h, rays, 0, post, refill, node_steps)
    assert np.array_equal(got.view(np.uint32).reshape(-1, 4), ref.view(np.uint32).reshape(-1, 4))
    _, st1 = host_cast(host_bvh, h, rays, 0)
    assert st[0] >= st1[0] and st[1] >= st1[1]
    anyr = oracle.cast_bruteforce(V, I, rays, 1)
    anyg, _ = host_cast_batched(host_bvh, h, rays, 1, post, refill, node_steps)
    assert np.array_equal(anyg["prim"] == 0xFFFFFFFF, anyr["prim"] == 0xFFFFFFFF)
    # any hit with children visited far to near (the shadow pass's tunable order): same answers
    anyf, _ = host_cast_batched(host_bvh, h, rays, 2, post, refill, node_steps)
    assert np.array_equal(anyf["prim"] == 0xFFFFFFFF, anyr["prim"] == 0xFFFFFFFF)
    host_bvh.hb_destroy(h)


def test_degenerate_rays_miss(host_bvh, oracle):
    """Degenerate rays (NaN or zero directions, infinite or NaN origins, empty [tmin, tmax]) end
    their traversal and hit nothing, in the single-lane and the batched warp traversal, like the
    brute force; valid rays in the same batch keep their hits."""
    from wayland_b200 import scenes
    sc = scenes.displaced_sphere(subdiv=24)
    h, V, I = host_build(host_bvh, sc.V, sc.I)
    bad = degenerate_rays(5)
    good = random_rays(500, 6, -3.0, 3.0)
    rays = np.concatenate([good[:250], bad, good[250:]])
    for mode in (0, 1):
        ref = oracle.cast_bruteforce(V, I, rays, mode)
        assert (ref["prim"][250:250 + len(bad)] == 0xFFFFFFFF).all()
        single, _ = host_cast(host_bvh, h, rays, mode)
        batched, _ = host_cast_batched(host_bvh, h, rays, mode, 8, 6, 3)
        for got in (single, batched):
            assert (got["prim"][250:250 + len(bad)] == 0xFFFFFFFF).all()
            if mode == 0:
                assert np.array_equal(got.view(np.uint32).reshape(-1, 4), ref.view(np.uint32).reshape(-1, 4))
            else:
                assert np.array_equal(got["prim"] == 0xFFFFFFFF, ref["prim"] == 0xFFFFFFFF)
    far, _ = host_cast(host_bvh, h, rays, 2)
    assert (far["prim"][250:250 + len(bad)] == 0xFFFFFFFF).all()
    host_bvh.hb_destroy(h)

