"""FP64 CPU oracle of the radiance cache (test infrastructure only; never imported by the
product path).

The cache has no counterpart in the reference renderer: this restates the project's own
published algorithms, the multiresolution hash-grid encoding of Mueller et al. 2022 ("Instant
Neural Graphics Primitives": per level a resolution floor(base * scale^l), the 8 corners of the
cell around the normalised position, dense indexing where the (res + 1)^3 corners fit the table,
else the spatial hash x ^ y * 2654435761 ^ z * 805459861 mod T, trilinear interpolation) and the
online radiance cache of Mueller et al. 2021 (relative L2 loss), as wayland_b200/csrc/wl_nrc.cuh,
nrc.cu and nrc_tc.cu implement them. Parity is therefore pinned against this restatement only.

- The MLP in numpy float64: inputs, weights and hidden activations rounded to bfloat16 (round to
  nearest even) as the device does, products and sums in float64; relative L2 loss
  sum_{s,c<3} (o - t)^2 / (o^2 + 0.01) / (3 n) and its gradient with respect to the 17408
  weights (W0..W3 64x64, W4 16x64, row = output), with the loss gradient dY and the
  pre-activation gradients dZ_l rounded to bfloat16 where the device's tensor-core backward pass
  rounds them (they are MMA operands there).
- The encoding: corner indices in float32 / uint32 exactly as the device computes them, the
  interpolation of the FP16 features in float64, the direction (real spherical harmonics of
  degree <= 3) and material features; the grid gradient as the scatter of the input gradient
  to the corners with the trilinear weights.
"""
import numpy as np

HID, OUT, MATS = 64, 16, 4
NW = MATS * HID * HID + OUT * HID


def bf16r(x):
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)
    return np.where(np.isnan(x), x, out).astype(np.float64)


def split(w):
    w = bf16r(w)
    mats = [w[l * HID * HID:(l + 1) * HID * HID].reshape(HID, HID) for l in range(MATS)]
    mats.append(w[MATS * HID * HID:].reshape(OUT, HID))
    return mats


def forward(w, x):
    """Returns (outputs n x 16, activations list a0..a4)."""
    Ws = split(w)
    a = bf16r(x)
    acts = [a]
    for l in range(MATS):
        a = bf16r(np.maximum(a @ Ws[l].T, 0.0))
        acts.append(a)
    return a @ Ws[MATS].T, acts


def gradients(w, x, t, bf16_deltas=True, return_input_grad=False):
    """Loss and dLoss/dW (float64, length 17408); with return_input_grad also dLoss/dx
    (n x 64), the gradient the hash grid receives."""
    rd = bf16r if bf16_deltas else (lambda a: a)
    Ws = split(w)
    o, acts = forward(w, x)
    n = len(x)
    o3 = o[:, :3]
    den = o3 * o3 + 0.01
    loss = float(((o3 - t[:, :3]) ** 2 / den).sum() / (3 * n))
    d = np.zeros_like(o)
    d[:, :3] = 2.0 * (o3 - t[:, :3]) / den / (3 * n)
    d = rd(d)
    grads = [None] * (MATS + 1)
    grads[MATS] = d.T @ acts[MATS]
    g = d @ Ws[MATS]
    for l in range(MATS - 1, -1, -1):
        dl = rd(g * (acts[l + 1] > 0))
        grads[l] = dl.T @ acts[l]
        g = dl @ Ws[l]
    gw = np.concatenate([gr.reshape(-1) for gr in grads])
    return (loss, gw, g) if return_input_grad else (loss, gw)


# ---------------------------------------------------------------------------------------------
# Hash-grid encoding (wayland_b200/csrc/wl_nrc.cuh): the index arithmetic in float32 / uint32
# exactly as the device computes it, the interpolation in float64 from the FP16 features the
# device gathers, every feature rounded to bfloat16 where the device rounds it.

SH_C = (0.28209479177387814, 0.48860251190291987, 1.0925484305920792, 0.94617469575755997,
        0.31539156525251999, 0.54627421529603959, 0.59004358992664352, 2.8906114426405538,
        0.45704579946446572, 0.3731763325901154, 1.4453057213202769)


def f16r(x):
    """Round to IEEE half precision (round to nearest even), returned as float64."""
    return np.asarray(x, np.float32).astype(np.float16).astype(np.float64)


class GridDesc:
    """levels, log2_table, base_resolution, per_level_scale and the normalisation box (lo,
    inv_ext, float32) of a cache's hash grid (wl_nrc_get_grid)."""

    def __init__(self, levels, log2_table, base, scale, lo, inv_ext):
        self.levels, self.log2T, self.base = int(levels), int(log2_table), int(base)
        self.scale = np.float32(scale)
        self.lo = np.asarray(lo, np.float32)
        self.inv_ext = np.asarray(inv_ext, np.float32)

    def res(self, l):
        """floor(base * scale^l), the product taken step by step in float32 (grid_res)."""
        s = np.float32(1.0)
        for _ in range(l):
            s = np.float32(s * self.scale)
        return int(np.floor(np.float32(self.base) * s))


def grid_index(g, res, x, y, z):
    """Entry of corner (x, y, z) of a level of resolution res (grid_index): dense where the
    (res + 1)^3 corners fit the table, else the spatial hash of Mueller et al. 2022."""
    T = 1 << g.log2T
    side = res + 1
    x = np.asarray(x, np.uint64)
    y = np.asarray(y, np.uint64)
    z = np.asarray(z, np.uint64)
    if side ** 3 <= T:
        return ((x + np.uint64(side) * (y + np.uint64(side) * z)) & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    m = np.uint64(0xFFFFFFFF)
    h = (x & m) ^ ((y * np.uint64(2654435761)) & m) ^ ((z * np.uint64(805459861)) & m)
    return (h & np.uint64(T - 1)).astype(np.uint32)


def grid_normalise(g, pos):
    p = np.asarray(pos, np.float32)
    return np.clip((p - g.lo[None]) * g.inv_ext[None], np.float32(0.0), np.float32(1.0)).astype(np.float32)


def grid_corners(g, pos):
    """For every position, level and corner k (bit 0: +x, bit 1: +y, bit 2: +z): the entry
    index (n, levels, 8) uint32 and the trilinear weight (n, levels, 8) float64."""
    pn = grid_normalise(g, pos)
    n = len(pn)
    idx = np.zeros((n, g.levels, 8), np.uint32)
    wts = np.zeros((n, g.levels, 8), np.float64)
    for l in range(g.levels):
        res = g.res(l)
        x = (pn * np.float32(res)).astype(np.float32)
        fl = np.floor(x).astype(np.float32)
        c = fl.astype(np.int64)
        f = (x - fl).astype(np.float32)
        over = c >= res
        c = np.where(over, res - 1, c)
        f = np.where(over, np.float32(1.0), f).astype(np.float64)
        for k in range(8):
            d = np.array([k & 1, (k >> 1) & 1, (k >> 2) & 1])
            wk = np.ones(n)
            for a in range(3):
                wk = wk * (f[:, a] if d[a] else 1.0 - f[:, a])
            wts[:, l, k] = wk
            idx[:, l, k] = grid_index(g, res, c[:, 0] + d[0], c[:, 1] + d[1], c[:, 2] + d[2])
    return idx, wts


def sh16(d):
    """Real spherical harmonics of degree <= 3 of unit directions (n, 3), float64."""
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    xx, yy, zz = x * x, y * y, z * z
    c = SH_C
    return np.stack([np.full_like(x, c[0]), -c[1] * y, c[1] * z, -c[1] * x, c[2] * x * y, -c[2] * y * z,
                     c[3] * zz - c[4], -c[2] * x * z, c[5] * (xx - yy), c[6] * y * (-3.0 * xx + yy),
                     c[7] * x * y * z, c[8] * y * (1.0 - 5.0 * zz), c[9] * z * (5.0 * zz - 3.0),
                     c[8] * x * (1.0 - 5.0 * zz), c[10] * z * (xx - yy), c[6] * x * (-xx + 3.0 * yy)], 1)


def encode(g, params, verts, mats):
    """The 64 input features of each vertex (nrc_encode), bfloat16-rounded, float64.
    params: the grid's FP32 parameters (levels, 2^log2T, 2), gathered as FP16 like the device.
    verts: structured array of wl_nrc_vertex (pos, material, wo, n, extra). mats: wl_disney."""
    n = len(verts)
    x = np.zeros((n, 64))
    idx, wts = grid_corners(g, verts["pos"])
    feat = f16r(params)
    for l in range(g.levels):
        e = feat[l][idx[:, l, :]]                  # (n, 8, 2)
        x[:, 2 * l:2 * l + 2] = (wts[:, l, :, None] * e).sum(1)
    x[:, 32:48] = sh16(np.asarray(verts["wo"], np.float64))
    m = mats[verts["material"]]
    dif = (1.0 - m["metallic"].astype(np.float64)) * (1.0 - m["trans"].astype(np.float64))
    col = m["color"].astype(np.float64)
    met = m["metallic"].astype(np.float64)[:, None]
    nrm = np.asarray(verts["n"], np.float64)
    x[:, 48:51] = nrm * 0.5 + 0.5
    x[:, 51] = m["roughness"]
    x[:, 52:55] = col * dif[:, None]
    x[:, 55:58] = 0.04 * (1.0 - met) + col * met
    x[:, 58] = m["trans"]
    x[:, 59] = 1.0
    return bf16r(x)


def query(w, g, params, verts, mats):
    """Cache prediction max(o, 0) for outputs 0..2 (the render's query path)."""
    o, _ = forward(w, encode(g, params, verts, mats))
    return np.maximum(o[:, :3], 0.0)


def sample_gradients(w, g, params, verts, mats):
    """Loss, dLoss/dW and dLoss/dparams (levels, 2^log2T, 2) of one training step on the
    vertices (targets in extra[:, :3]): the input gradient of the grid features scattered to
    the 8 corners of every level with the trilinear weights (nrc_grid_backward)."""
    x = encode(g, params, verts, mats)
    t = np.asarray(verts["extra"], np.float64)
    loss, gw, gin = gradients(w, x, t, return_input_grad=True)
    ggrid = np.zeros(params.shape, np.float64)
    idx, wts = grid_corners(g, verts["pos"])
    for l in range(g.levels):
        for f in range(2):
            np.add.at(ggrid[l, :, f], idx[:, l, :].reshape(-1),
                      (wts[:, l, :] * gin[:, 2 * l + f][:, None]).reshape(-1))
    return loss, gw, ggrid
