"""Generate the golden vectors in tests/golden/ from the reference's own code.

The reference (Extra-Creativity/Wayland) has no tests and no golden vectors of its own. These
fixtures are the outputs of its src/Frontend/Device/*.h functions (tea<4>, rnd, PinholeGenerateRay,
SampleDisneyBSDF, EvalDisneyBSDF, PdfDisneyBSDF, AceApprox) compiled on the host from the
reference tree by oracle/ref_build (-> oracle/_ref/libwlref.so), plus a small image rendered by
the path loop of PathTracing.cu:40-288 written over those functions, and images rendered by
the reference's PathTracing.cu, AO.cu and BDPT.cu programs themselves (compiled on the host with their OptiX
calls emulated over the oracle's CPU BVH, oracle/ref_build/ref_programs.cpp and ref_bdpt.cpp). sin/cos/log inside the
reference functions are routed to the project's own single-precision versions (see
oracle/ref_build/shim/wl_ref_math.h), so the vectors pin the oracle bit for bit.

Run in a container that holds the reference tree:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

import pyoracle as po  # noqa: E402
from wayland_b200 import scenes  # noqa: E402


def random_materials(rng, n):
    m = np.zeros(n, po.DISNEY_DTYPE)
    m["color"] = rng.uniform(0, 1, (n, 3))
    m["metallic"] = np.where(rng.uniform(size=n) < 0.2, 0.0, rng.uniform(0, 1, n))
    m["roughness"] = np.where(rng.uniform(size=n) < 0.05, 0.0, rng.uniform(0, 1, n))
    m["specular"] = rng.uniform(0, 1, n)
    m["specular_tint"] = rng.uniform(0, 1, n)
    m["eta"] = rng.uniform(1.0, 2.4, n)
    kind = rng.uniform(size=n)
    m["trans"] = np.where(kind < 0.3, rng.uniform(0, 1, n), np.where(kind < 0.6, 1.0, 0.0))
    m["subsurface"] = rng.uniform(0, 1, n)
    m["sheen"] = rng.uniform(0, 1, n)
    m["sheen_tint"] = rng.uniform(0, 1, n)
    m["clearcoat"] = rng.uniform(0, 1, n)
    m["clearcoat_gloss"] = rng.uniform(0, 1, n)
    m["texture"] = -1
    return m


def unit(rng, n):
    v = rng.normal(size=(n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def main():
    po.build_ref()
    ref = po.RefLib()
    rng = np.random.default_rng(20261203)
    out = {}
    # random streams
    pairs = rng.integers(0, 2 ** 32, (256, 2), dtype=np.uint64).astype(np.uint32)
    out["tea_in"] = pairs
    out["tea_out"] = np.array([ref.tea4(int(a), int(b)) for a, b in pairs], np.uint32)
    seeds = rng.integers(0, 2 ** 32, 16, dtype=np.uint64).astype(np.uint32)
    out["rnd_seed"] = seeds
    out["rnd_out"] = np.stack([ref.rnd_stream(int(s), 64) for s in seeds])
    # BSDF
    n = 4096
    mats = random_materials(rng, n)
    Ns, V, L = unit(rng, n), unit(rng, n), unit(rng, n)
    # geometric normals near the shading normals, some flipped (back faces / transmission)
    Ng = Ns + 0.2 * unit(rng, n)
    Ng = (Ng / np.linalg.norm(Ng, axis=1, keepdims=True)).astype(np.float32)
    tex = rng.uniform(0, 1, (n, 3)).astype(np.float32)
    s0 = rng.integers(0, 2 ** 32, n, dtype=np.uint64).astype(np.uint32)
    out.update(mats=mats, Ns=Ns, Ng=Ng, V=V, L=L, tex=tex, sample_seed=s0)
    out["eval"] = ref.disney_eval(mats, Ns, Ng, V, L, tex)
    out["pdf"] = ref.disney_pdf(mats, Ns, Ng, V, L)
    out["sample"], out["sample_seed_out"] = ref.disney_sample(mats, Ns, Ng, V, s0)
    # camera + tone map
    sc = scenes.cornell_box(256, 256)
    cam = sc.camera_struct()
    camo = po.Camera()
    for k in ("pos", "look_at", "up", "right"):
        getattr(camo, k)[:] = list(getattr(cam, k))
    px = rng.integers(0, 256, 512).astype(np.uint32)
    py = rng.integers(0, 256, 512).astype(np.uint32)
    cs = rng.integers(0, 2 ** 32, 512, dtype=np.uint64).astype(np.uint32)
    out["cam"] = np.array([list(cam.pos), list(cam.look_at), list(cam.up), list(cam.right)], np.float32)
    out.update(cam_px=px, cam_py=py, cam_seed=cs)
    out["cam_dir"], out["cam_seed_out"] = ref.camera_rays(camo, 256, 256, px, py, cs)
    rad = np.concatenate([rng.uniform(0, 4, (1000, 3)), rng.exponential(20, (24, 3))]).astype(np.float32)
    out["ace_in"] = rad
    out["ace_out"] = ref.ace(rad)
    np.savez_compressed(os.path.join(HERE, "device_math.npz"), **out)

    # a small image of the procedural Cornell box through the reference's arithmetic
    W = H = 32
    p = po.RenderParams(width=W, height=H, spp=4, first_frame=0, max_depth=25, rr_depth=5,
                        rr_prob=0.9, eps=1e-3, strategy=2, rng=0, math=1, lights=0, seed=0)
    img, segs = ref.render(sc, camo, p)
    np.savez_compressed(os.path.join(HERE, "cornell_32x32_4spp.npz"), image=img,
                        segments=np.uint64(segs), V=sc.V, I=sc.I, tri_material=sc.tri_material,
                        mats=sc.mats, lights=sc.lights, cam=out["cam"])

    # ambient occlusion (AO.cu) of the displaced sphere through the reference's arithmetic
    sph = scenes.displaced_sphere(40, 24, subdiv=12, seed=5)
    scam = po.Camera()
    for k in ("pos", "look_at", "up", "right"):
        getattr(scam, k)[:] = [float(x) for x in sph.camera[k]]
    ap = po.AoParams(width=40, height=24, spp=2, first_frame=0, camera_samples=4, ao_rays=32,
                     radius=1.0, eps=1e-3, rng=0, wave_paths=0, seed=0)
    ao_img, ao_rays = ref.render_ao(sph, scam, ap)
    np.savez_compressed(os.path.join(HERE, "ao_sphere_40x24.npz"), image=ao_img,
                        rays=np.uint64(ao_rays), V=sph.V, N=sph.N, I=sph.I,
                        tri_flags=sph.tri_flags,
                        cam=np.array([list(scam.pos), list(scam.look_at), list(scam.up),
                                      list(scam.right)], np.float32))
    # the reference's own bidirectional program (Programs/BDPT/BDPT.cu, run over the host
    # emulation of its OptiX calls): the Cornell box and a small glass sphere
    for name, bsc in (("bdpt_cornell_32x32_4spp.npz", scenes.cornell_box(32, 32)),
                      ("bdpt_glass_40x40_4spp.npz", scenes.glass_sphere(40, 40, subdiv=12))):
        bcam = po.Camera()
        for k in ("pos", "look_at", "up", "right"):
            getattr(bcam, k)[:] = [float(x) for x in bsc.camera[k]]
        rad = ref.render_bdpt(bsc, bcam, bsc.width, bsc.height, 4)
        np.savez_compressed(os.path.join(HERE, name), image=rad[..., :3].copy(), V=bsc.V, I=bsc.I,
                            N=bsc.N if bsc.N is not None else np.zeros(0, np.float32),
                            cam=np.array([list(bcam.pos), list(bcam.look_at), list(bcam.up),
                                          list(bcam.right)], np.float32))
    # the reference's own PathTracing.cu and AO.cu programs over the OptiX host emulation
    # (oracle/ref_build/ref_programs.cpp): the displaced sphere with vertex normals and four
    # lights (the programs' background is 0), and ambient occlusion in a closed room (AO.cu
    # needs every camera ray to hit: after a miss it traces from the payload's stale hit point)
    sph2 = scenes.displaced_sphere(48, 32, subdiv=24, seed=3)
    c2 = po.Camera()
    for k in ("pos", "look_at", "up", "right"):
        getattr(c2, k)[:] = [float(x) for x in sph2.camera[k]]
    rad = ref.program_pt(sph2, c2, 48, 32, 4)
    np.savez_compressed(os.path.join(HERE, "program_pt_sphere_48x32_4spp.npz"), image=rad[..., :3].copy(),
                        V=sph2.V, I=sph2.I)
    room = scenes.door_slit_room(32, 24, cells=8, slit=0.0)
    c3 = po.Camera()
    for k in ("pos", "look_at", "up", "right"):
        getattr(c3, k)[:] = [float(x) for x in room.camera[k]]
    rad = ref.program_ao(room, c3, 32, 24, 2)
    np.savez_compressed(os.path.join(HERE, "program_ao_room_32x24_2spp.npz"), image=rad[..., :3].copy(),
                        V=room.V, I=room.I)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main()
