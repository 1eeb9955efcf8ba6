"""The example program (examples/path_tracer.cpp, the equivalent of the reference's
examples/PathTracer/main.cpp over the C ABI) built with g++ and run as a separate process: the
procedural Cornell box of the benchmark's first configuration, 256x256, 16 frames of one sample,
depth 8, PCG32 seed 0, strict math. Its linear film must equal the CPU oracle's render of the same
scene and camera bit for bit, and its PNG must decode to the tone-mapped film, flipped."""
import os
import struct
import subprocess
import zlib

import numpy as np
import pytest

import pyoracle as po
import wayland_b200 as wl
from wayland_b200 import scenes

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "tests", "_build")


def read_png_rgba(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat = 8, b""
    w = h = None
    while pos < len(data):
        n, typ = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        assert zlib.crc32(typ + body) == struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]
        if typ == b"IHDR":
            w, h = struct.unpack(">II", body[:8])
            assert body[8:13] == bytes([8, 6, 0, 0, 0])
        elif typ == b"IDAT":
            idat += body
        pos += 12 + n
    raw = zlib.decompress(idat)
    rows = np.frombuffer(raw, np.uint8).reshape(h, 4 * w + 1)
    assert (rows[:, 0] == 0).all()
    return rows[:, 1:].reshape(h, w, 4)


def test_example_program_matches_oracle(oracle, tmp_path):
    os.makedirs(BUILD, exist_ok=True)
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "examples"), f"OUT={BUILD}"])
    png, raw = str(tmp_path / "cornell.png"), str(tmp_path / "film.bin")
    r = subprocess.run([os.path.join(BUILD, "path_tracer"), "--strict", "--out", png, "--raw", raw],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    blob = open(raw, "rb").read()
    assert blob[:4] == b"WLRF"
    W, H = struct.unpack("<II", blob[4:12])
    cam = np.frombuffer(blob[12:60], np.float32)
    film = np.frombuffer(blob[60:], np.float32).reshape(H, W, 3)
    assert (W, H) == (256, 256) and film.mean() > 0.01
    sc = scenes.cornell_box(256, 256)
    for k, key in enumerate(("pos", "look_at", "up", "right")):
        np.testing.assert_allclose(cam[3 * k:3 * k + 3], sc.camera[key], rtol=1e-6, atol=1e-7)
        sc.camera[key] = cam[3 * k:3 * k + 3].copy()
    p = wl.render_params(256, 256, 16, max_depth=8, rng=wl.RNG_PCG32, seed=0, math=wl.MATH_STRICT)
    ocam = po.Camera()
    for key in ("pos", "look_at", "up", "right"):
        getattr(ocam, key)[:] = [float(x) for x in sc.camera[key]]
    q = po.RenderParams()
    for key, _ in q._fields_:
        if key == "env":
            q.env[:] = list(p.env)
        else:
            setattr(q, key, getattr(p, key))
    ref, _, _ = oracle.render(sc, ocam, q)
    assert np.array_equal(film.view(np.uint32), np.ascontiguousarray(ref, np.float32).view(np.uint32))
    # the PNG: AceApprox tone mapping x 255, truncated, rows flipped (Renderer.cpp:94-105)
    img = read_png_rgba(png)[::-1]
    tm = oracle.ace(np.clip(film, 0.0, 1e30).reshape(-1, 3)).reshape(H, W, 3)
    assert np.array_equal(img[..., :3], (tm * np.float32(255.0)).astype(np.uint8))
    assert (img[..., 3] == 255).all()
