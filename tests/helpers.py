"""Shared test inputs (seeded)."""
import numpy as np

from wayland_b200 import _abi, scenes


def random_rays(n, seed, lo=-1.5, hi=1.5, tmin=1e-3, tmax=1e30):
    rng = np.random.default_rng(seed)
    r = np.zeros(n, _abi.RAY_DTYPE)
    r["org"] = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    r["dir"] = d / np.linalg.norm(d, axis=1, keepdims=True)
    r["tmin"] = tmin
    r["tmax"] = tmax
    return r


def axis_rays(n, seed, lo=-1.5, hi=1.5):
    """Rays along +-x, +-y, +-z (zero direction components)."""
    rng = np.random.default_rng(seed)
    r = np.zeros(n, _abi.RAY_DTYPE)
    r["org"] = rng.uniform(lo, hi, (n, 3))
    axis = rng.integers(0, 3, n)
    sign = rng.choice([-1.0, 1.0], n)
    d = np.zeros((n, 3))
    d[np.arange(n), axis] = sign
    r["dir"] = d
    r["tmin"] = 0.0
    r["tmax"] = 1e30
    return r


def geometries():
    """(name, V, I) triples covering a soup, the Cornell box, a displaced sphere and edge cases."""
    soup = scenes.random_triangles(3000, 1)
    cb = scenes.cornell_box()
    sph = scenes.displaced_sphere(subdiv=20)
    # many triangles with identical centroids (equal Morton codes)
    rng = np.random.default_rng(3)
    dupV = np.concatenate([np.array([[-0.5, -0.5, 0.0], [0.5, -0.5, 0.0], [0.0, 0.5, 0.0]]) * s
                           for s in rng.uniform(0.5, 1.0, 64)]).astype(np.float32)
    dupI = np.arange(len(dupV), dtype=np.uint32).reshape(-1, 3)
    # a coplanar grid (flat bounding boxes on one axis)
    g = np.linspace(-1, 1, 9)
    gv, gi = [], []
    for a in range(8):
        for b in range(8):
            k = len(gv)
            gv += [[g[a], g[b], 0.0], [g[a + 1], g[b], 0.0], [g[a + 1], g[b + 1], 0.0], [g[a], g[b + 1], 0.0]]
            gi += [[k, k + 1, k + 2], [k, k + 2, k + 3]]
    one = (np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32), np.array([[0, 1, 2]], np.uint32))
    # degenerate triangles mixed in (zero area, collinear)
    degV = np.concatenate([soup[0][:300], np.array([[0, 0, 0], [0, 0, 0], [0, 0, 0],
                                                    [0, 0, 0], [1, 1, 1], [2, 2, 2]], np.float32)])
    degI = np.arange(len(degV), dtype=np.uint32).reshape(-1, 3)
    return [("soup", *soup), ("cornell", cb.V, cb.I), ("sphere", sph.V, sph.I),
            ("dup_centroids", dupV, dupI), ("grid", np.array(gv, np.float32), np.array(gi, np.uint32)),
            ("one", *one), ("degenerate", degV, degI)]


def degenerate_rays(seed, lo=-1.5, hi=1.5):
    """Rays a caller can hand to wl_cast_rays by mistake, each kind over several origins: NaN
    directions (whole or one component), a zero direction, an infinite or NaN origin, an infinite
    direction component, tmin > tmax, tmin == tmax, and negative tmax. None may hit anything."""
    rng = np.random.default_rng(seed)
    kinds = []
    for _ in range(12):
        o = rng.uniform(lo, hi, 3)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        nan = float("nan")
        inf = float("inf")
        kinds += [
            (o, (nan, nan, nan), 1e-3, 1e30),
            (o, (d[0], nan, d[2]), 1e-3, 1e30),
            (o, (0.0, 0.0, 0.0), 1e-3, 1e30),
            ((inf, o[1], o[2]), d, 1e-3, 1e30),
            ((o[0], nan, o[2]), d, 1e-3, 1e30),
            (o, (d[0], inf, d[2]), 1e-3, 1e30),
            (o, d, 2.0, 1.0),
            (o, d, 0.5, 0.5),
            (o, d, 0.0, -1.0),
        ]
    r = np.zeros(len(kinds), _abi.RAY_DTYPE)
    for i, (o, d, t0, t1) in enumerate(kinds):
        r["org"][i] = o
        r["dir"][i] = d
        r["tmin"][i] = t0
        r["tmax"][i] = t1
    return r

