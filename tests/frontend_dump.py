"""Runs the reference's own frontend (oracle/_ref/wl_frontend: minipbrt + the reference's
SceneManager, driving the library through the integration guide's DeviceManager) and reads its
dump: the arrays DeviceManager::Setup handed to wl_scene_create, the camera and, when it
rendered, the linear film. Test infrastructure."""
import os
import struct
import subprocess

import numpy as np

from wayland_b200 import _abi, scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FRONTEND = os.path.join(ROOT, "oracle", "_ref", "wl_frontend")


def available():
    return os.path.exists(FRONTEND)


def run(pbrt_path, width, height, dump, frames=0, depth=25, strict=False):
    """frames = 0: parse only (no GPU)."""
    cmd = [FRONTEND, str(pbrt_path), "--width", str(width), "--height", str(height), "--dump", str(dump),
           "--depth", str(depth)]
    cmd += ["--parse-only"] if frames == 0 else ["--frames", str(frames)]
    if strict:
        cmd.append("--strict")
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=os.path.dirname(str(pbrt_path)))
    if r.returncode != 0:
        raise RuntimeError(f"wl_frontend failed ({r.returncode}): {r.stdout}{r.stderr}")
    return read(dump)


def read(path):
    """(scenes.Scene of the frontend's arrays, film (H, W, 3) float32 or None)."""
    b = open(path, "rb").read()
    assert b[:4] == b"WLFE"
    ver, nV, nT, nMat, nL, nTex, W, H, frames = struct.unpack("<9I", b[4:40])
    assert ver == 1
    off = [40]

    def take(dt, n):
        a = np.frombuffer(b, dt, n, off[0])
        off[0] += a.nbytes
        return a.copy()

    V = take(np.float32, 3 * nV).reshape(-1, 3)
    N = take(np.float32, 3 * nV).reshape(-1, 3)
    UV = take(np.float32, 2 * nV).reshape(-1, 2)
    I = take(np.uint32, 3 * nT).reshape(-1, 3)
    tri_material = take(np.uint32, nT)
    tri_flags = take(np.uint32, nT)
    mats = take(_abi.DISNEY_DTYPE, nMat)
    lights = take(_abi.LIGHT_DTYPE, nL)
    textures = []
    for _ in range(nTex):
        w, h = struct.unpack("<II", b[off[0]:off[0] + 8])
        off[0] += 8
        textures.append(take(np.uint8, 4 * w * h).reshape(h, w, 4))
    cam = take(np.float32, 12)
    film = take(np.float32, 3 * W * H).reshape(H, W, 3) if frames else None
    camera = {k: cam[3 * i:3 * i + 3] for i, k in enumerate(("pos", "look_at", "up", "right"))}
    sc = scenes.Scene("frontend", V, I, tri_material, mats, lights, N=N, tri_flags=tri_flags, camera=camera,
                      width=W, height=H, UV=UV, textures=textures)
    return sc, film
