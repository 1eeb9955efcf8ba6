"""FP64 CPU oracle of the radiance-cache MLP (test infrastructure only).

Restates the network of wayland_b200/csrc/wl_nrc.cuh and nrc_tc.cu in numpy float64: inputs,
weights and hidden activations rounded to bfloat16 (round to nearest even) as the device does,
products and sums in float64; relative L2 loss sum_{s,c<3} (o - t)^2 / (o^2 + 0.01) / (3 n) and
its gradient with respect to the 17408 weights (W0..W3 64x64, W4 16x64, row = output), with the
loss gradient dY and the pre-activation gradients dZ_l rounded to bfloat16 where the device's
tensor-core backward pass rounds them (they are MMA operands there).
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


def gradients(w, x, t, bf16_deltas=True):
    """Loss and dLoss/dW (float64, length 17408)."""
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
    return loss, np.concatenate([gr.reshape(-1) for gr in grads])
