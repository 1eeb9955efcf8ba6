"""Benchmark: plain path tracing at scale (Mpaths/s) on one or more B200s.

Workload (one step): the displaced-sphere scene - an icosphere subdivided to 1,997,120 triangles
and displaced by fBm of amplitude 0.05 over a 2-triangle ground plane, per-object Disney
parameters from seed 0, 4 quad lights and a constant environment of 0.1 - rendered at
1920 x 1080 with 64 samples per pixel and path depth 16 in FP32 (132,710,400 paths), through
wl_render in WL_MATH_FAST mode with the reference's TEA+LCG streams, uniform light selection,
MIS and Russian roulette (after depth 5, p = 0.9). Synthetic data; the BVH is built once
outside the timed region (Mpaths/s = W * H * spp / render time).

Prints one JSON line (see the keys below). `--impl reference` times the reference's own
PathTracing.cu program compiled on the host (oracle/_ref/libwlref.so, its OptiX calls emulated
over the oracle's CPU BVH) on all host cores, on a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

W, H, SPP, DEPTH = 1920, 1080, 64, 16
METRIC = "Mpaths/s"
# DRAM bytes (read + write) per extend ray of this workload, from an ncu launch list of the same
# command (dram__bytes_read.sum + dram__bytes_write.sum over the 16 extend launches of one step,
# divided by the step's extend rays); CUDA events cannot count DRAM bytes, so the bench scales
# this figure by its own rays and labels the number as taken from that capture
EXTEND_DRAM_BYTES_PER_RAY = 153.0
TRAFFIC_SOURCE = ("ncu launch list of this workload: 45.34 GB of DRAM over the 16 extend launches "
                  "of one step / 298.3 M extend rays = 153 B per ray, times this run's rays")
# The CPU legs time the same fixed pixel sample: CPU_ROWS rows of the 1920x1080 image around its
# centre, at the full 64 spp
CPU_ROWS = 32
WORKLOAD = "plain PT at scale: displaced icosphere 1,997,120 tris + ground, 4 quad lights + env 0.1, 1920x1080, 64 spp, depth 16, FP32"


# BVH build used for every scene (set from --bvh)
BVH_KIND = [1]

def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region (SM clock, throttle reasons)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.f.flush()
        rows = [l.split(",") for l in open(self.f.name).read().strip().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except (ValueError, IndexError):
                continue
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


class CpuPT:
    """The CPU path tracer on a bounded sample of the workload (pixel rows at 64 spp): the
    reference's own PathTracing.cu program run on the host cores over an emulation of its OptiX
    calls (oracle/_ref/libwlref.so, kind "reference") when it was built, else the project's CPU
    port of the same loop (oracle/_build/liboracle.so, kind "port"). Traversal in both is the
    oracle's CPU BVH (OptiX is closed); the program's background is 0 instead of 0.1."""

    def __init__(self, scene, threads):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import ctypes as C
        import pyoracle as po
        self.C = C
        self.threads = threads
        if os.path.exists(po.LIB_REF):
            self.lib, self.kind = po.RefLib(), "reference"
        else:
            self.lib, self.kind = po.Oracle(), "port"
        self.cam = po.Camera()
        for k in ("pos", "look_at", "up", "right"):
            getattr(self.cam, k)[:] = [float(x) for x in scene.camera[k]]
        self.p = po.RenderParams(width=W, height=H, spp=SPP, first_frame=0, max_depth=DEPTH,
                                 rr_depth=5, rr_prob=0.9, eps=1e-3, strategy=2, rng=0, math=1,
                                 lights=0, seed=0)
        self.p.env[:] = list(scene.env)
        self.keep, self.osc = po.make_or_scene(scene)
        self.bvh = self.lib.lib.or_bvh_create(self.osc.V, self.osc.I, self.osc.nT)
        self.film = np.zeros((H, W, 3), np.float32)
        self.film4 = np.zeros((H, W, 4), np.float32)
        if self.kind == "reference":
            f = self.lib.lib.ref_program_pt
            f.restype = C.c_uint64
            f.argtypes = [C.POINTER(po.OrScene), C.c_void_p, C.POINTER(po.Camera), C.c_uint32,
                          C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, C.c_void_p, C.c_uint32,
                          C.c_uint32]
        self.npx = None

    def run(self, lo, hi):
        C = self.C
        t = time.perf_counter()
        if self.kind == "reference":
            self.lib.lib.ref_program_pt(C.byref(self.osc), self.bvh, C.byref(self.cam), W, H, SPP, 0,
                                        self.threads, self.film4.ctypes.data, lo, hi)
        else:
            self.lib.lib.or_render(C.byref(self.osc), self.bvh, C.byref(self.cam), C.byref(self.p), 0,
                                   self.threads, self.film.ctypes.data, None, lo, hi)
        return time.perf_counter() - t

    def sample(self, rows=CPU_ROWS):
        """Times the fixed sample (rows x W pixels around the image centre at SPP samples per
        pixel); returns (Mpaths/s, seconds, description)."""
        npx = rows * W
        lo = (H // 2) * W - npx // 2
        dt = self.run(lo, lo + npx)
        desc = (f"{npx} pixels ({rows} rows around the image centre) x {SPP} spp "
                f"= {npx * SPP} paths in {dt:.2f} s on {self.threads} threads")
        if self.kind == "reference":
            desc += " (PathTracing.cu as compiled: depth cap 25, background 0)"
        return npx * SPP / dt / 1e6, dt, desc

    def close(self):
        self.lib.lib.or_bvh_destroy(self.bvh)


def reference_arm(args):
    """The reference's own CPU implementation of the path (PathTracing.cu compiled on the host
    over an emulation of its OptiX calls) on all host cores. Each step renders the same fixed
    pixel sample of the bench frame (CPU_ROWS centre rows at 64 spp, about 3.9 M paths), so
    ms_per_step is the time of the sample actually rendered, not of a full frame."""
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    from wayland_b200 import scenes
    scene = scenes.displaced_sphere(W, H, SPP, DEPTH)
    threads = os.cpu_count() or 1
    cpu = CpuPT(scene, threads)
    vals, secs, desc = [], [], ""
    for step in range(args.warmup + args.steps):
        v, dt, desc = cpu.sample()
        if step >= args.warmup:
            vals.append(v)
            secs.append(dt)
    cpu.close()
    value = float(statistics.mean(vals))
    npx = CPU_ROWS * W
    line = {"metric": METRIC, "value": round(value, 4), "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * float(statistics.mean(secs)), 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "device": "host CPU", "threads": threads,
                       "sampled": True, "sample_pixels": npx, "sample_paths": npx * SPP,
                       "sample": f"{CPU_ROWS} rows around the centre of the 1920x1080 frame, 64 spp; "
                                 "a step renders this sample, not the full frame"},
            "cpu_baseline": {"value": round(value, 4), "unit": METRIC, "cores": threads,
                             "kind": cpu.kind, "sample": desc},
            "e2e": {"value": round(value, 4), "unit": METRIC, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    if cpu.kind != "reference":
        line["note"] = "oracle/_ref/libwlref.so absent: the project's CPU port of the same loop was timed"
    print(json.dumps(line), flush=True)
    return 0


def raycast_microbench(wl, torch, ctx, sc, scene, stream, tune=None):
    """2^24 coherent primary rays (4096 x 4096 view), 2^24 cosine-distributed bounce rays from
    the primary hit points and 2^24 any-hit shadow rays from the same points to uniform points of
    random lights; Mrays/s and traversal counts. The shadow rays are also timed with the other
    any-hit child order (far to near against near to far) under `shadow_other_order`."""
    n_side = 4096
    dev = torch.device("cuda")
    cam = {k: torch.tensor(np.asarray(scene.camera[k], np.float32), device=dev) for k in scene.camera}
    # square view with the camera's vertical field of view
    right = cam["right"] / torch.linalg.norm(cam["right"]) * torch.linalg.norm(cam["up"])
    j, i = torch.meshgrid(torch.arange(n_side, device=dev), torch.arange(n_side, device=dev), indexing="ij")
    u = (2.0 * (i.float() + 0.5) / n_side - 1.0).reshape(-1, 1)
    v = (2.0 * (j.float() + 0.5) / n_side - 1.0).reshape(-1, 1)
    d = cam["look_at"][None] + right[None] * u + cam["up"][None] * v
    d = d / torch.linalg.norm(d, dim=1, keepdim=True)
    n = d.shape[0]
    rays = torch.zeros((n, 8), dtype=torch.float32, device=dev)
    rays[:, 0:3] = cam["pos"][None]
    rays[:, 3] = 1e-3
    rays[:, 4:7] = d
    rays[:, 7] = 1e30
    hits = torch.empty((n, 4), dtype=torch.float32, device=dev)

    def timed(rbuf, reps=5, mode=wl.CAST_CLOSEST):
        with torch.cuda.stream(stream):
            sc.cast(rbuf.data_ptr(), hits.data_ptr(), n, mode)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                sc.cast(rbuf.data_ptr(), hits.data_ptr(), n, mode)
            e1.record(stream)
            torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    t_primary = timed(rays)
    nodes_p, tris_p = sc.cast_stats(rays.data_ptr(), n)
    # bounce rays from the primary hits
    with torch.cuda.stream(stream):
        sc.cast(rays.data_ptr(), hits.data_ptr(), n, wl.CAST_CLOSEST)
    torch.cuda.synchronize()
    prim = hits[:, 1].view(torch.int32)
    ok = prim != -1
    V = torch.from_numpy(scene.V).to(dev)
    I = torch.from_numpy(scene.I.astype(np.int64)).to(dev)
    p = torch.where(ok, prim, torch.zeros_like(prim)).long()
    a, b, c = V[I[p, 0]], V[I[p, 1]], V[I[p, 2]]
    ng = torch.cross(b - a, c - a, dim=1)
    ng = ng / torch.linalg.norm(ng, dim=1, keepdim=True).clamp_min(1e-30)
    ng = torch.where((ng * rays[:, 4:7]).sum(1, keepdim=True) > 0, -ng, ng)
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    r1 = torch.rand(n, device=dev, generator=g)
    r2 = torch.rand(n, device=dev, generator=g)
    phi = 2 * np.pi * r1
    sx, sy, sz = torch.sqrt(r2) * torch.cos(phi), torch.sqrt(r2) * torch.sin(phi), torch.sqrt(1 - r2)
    t1 = torch.where(ng[:, 0:1].abs() > 0.9, torch.tensor([[0.0, 1.0, 0.0]], device=dev),
                     torch.tensor([[1.0, 0.0, 0.0]], device=dev))
    tx = torch.cross(ng, t1, dim=1)
    tx = tx / torch.linalg.norm(tx, dim=1, keepdim=True)
    ty = torch.cross(ng, tx, dim=1)
    bd = tx * sx[:, None] + ty * sy[:, None] + ng * sz[:, None]
    brays = torch.zeros_like(rays)
    brays[:, 0:3] = rays[:, 0:3] + rays[:, 4:7] * hits[:, 0:1]
    brays[:, 3] = 1e-3
    brays[:, 4:7] = bd
    brays[:, 7] = 1e30
    # rays whose primary missed become copies of primary rays (still 2^24 traced)
    brays = torch.where(ok[:, None], brays, rays)
    # shadow rays (any hit) from the same surface points to a uniform point of a random light
    nl = len(scene.lights)
    li = torch.randint(0, nl, (n,), device=dev, generator=g)
    first = torch.from_numpy(scene.lights["first_tri"].astype(np.int64)).to(dev)
    count = torch.from_numpy(scene.lights["tri_count"].astype(np.int64)).to(dev)
    lt = first[li] + (torch.rand(n, device=dev, generator=g) * count[li]).long().clamp_max(count[li] - 1)
    s1 = torch.sqrt(torch.rand(n, device=dev, generator=g))[:, None]
    s2 = torch.rand(n, device=dev, generator=g)[:, None]
    la, lb, lc = V[I[lt, 0]], V[I[lt, 1]], V[I[lt, 2]]
    lp = la * (1 - s1) + lb * (s1 * (1 - s2)) + lc * (s1 * s2)
    sd = lp - brays[:, 0:3]
    dist = torch.linalg.norm(sd, dim=1, keepdim=True).clamp_min(1e-6)
    srays = torch.zeros_like(rays)
    srays[:, 0:3] = brays[:, 0:3]
    srays[:, 3] = 1e-3
    srays[:, 4:7] = sd / dist
    srays[:, 7] = (dist * (1 - 1e-3))[:, 0]
    t_shadow = timed(srays, mode=wl.CAST_ANY)
    nodes_s, tris_s = sc.cast_stats(srays.data_ptr(), n, wl.CAST_ANY)
    t_bounce = timed(brays)
    nodes_b, tris_b = sc.cast_stats(brays.data_ptr(), n)
    other = None
    if tune is not None:
        flipped = dict(tune)
        flipped.pop("fixed", None)
        flipped["shadow_far_first"] = 0 if tune.get("shadow_far_first") else 1
        ctx.set_tune(flipped)
        t_o = timed(srays, mode=wl.CAST_ANY)
        n_o, tr_o = sc.cast_stats(srays.data_ptr(), n, wl.CAST_ANY)
        restore = dict(tune)
        restore.pop("fixed", None)
        ctx.set_tune(restore)
        other = {"shadow_far_first": flipped["shadow_far_first"], "ms": round(t_o, 3),
                 "mrays_s": round(n / t_o / 1e3, 1), "nodes_per_ray": round(n_o / n, 2),
                 "tris_per_ray": round(tr_o / n, 2)}
    out = {}
    for name, t, nn, tt in (("primary", t_primary, nodes_p, tris_p), ("bounce", t_bounce, nodes_b, tris_b),
                            ("shadow", t_shadow, nodes_s, tris_s)):
        nodes_per, tris_per = nn / n, tt / n
        bytes_per = 48 + 80 * nodes_per + 48 * tris_per
        out[name] = {"rays": n, "ms": round(t, 3), "mrays_s": round(n / t / 1e3, 1),
                     "nodes_per_ray": round(nodes_per, 2), "tris_per_ray": round(tris_per, 2),
                     "algorithmic_gbs": round(n * bytes_per / (t * 1e-3) / 1e9, 1)}
    out["primary_hit_fraction"] = round(float(ok.float().mean()), 4)
    if other is not None:
        out["shadow_other_order"] = other
    return out


def graph_leg(wl, torch, ctx, sc, scene, stream, repeats=24, frames=4):
    """Progressive rendering, 1 spp per call at 1920x1080 on the benchmark scene: device time per
    call with direct launches and with every wave replayed as one CUDA graph. The two modes
    alternate in blocks of `frames` calls, `repeats` blocks each; the median block time per
    frame is reported (and the spread), so that drift on a shared machine hits both modes."""
    cam = scene.camera_struct()
    modes = (("launches", 0), ("graph", wl._abi.RENDER_GRAPH))
    films = {name: wl.Film(ctx, W, H) for name, _ in modes}
    times = {name: [] for name, _ in modes}
    frame = {name: 0 for name, _ in modes}
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    for rep in range(repeats + 1):  # block 0 of each mode is warm-up (first launches, capture)
        for name, flags in modes:
            p = wl.render_params(W, H, 1, max_depth=DEPTH, env=scene.env, flags=flags)
            ctx.sync()
            e0.record(stream)
            for _ in range(frames):
                p.first_frame = frame[name]
                frame[name] += 1
                wl.render(ctx, sc, cam, p, films[name])
            e1.record(stream)
            e1.synchronize()
            if rep:
                times[name].append(e0.elapsed_time(e1) / frames)
    out = {}
    for name, _ in modes:
        t = sorted(times[name])
        out[name] = {"ms_per_frame": round(statistics.median(t), 3), "min": round(t[0], 3),
                     "max": round(t[-1], 3), "repeats": repeats, "frames_per_repeat": frames}
        films[name].close()
    out["graph_over_launches"] = round(out["graph"]["ms_per_frame"] / out["launches"]["ms_per_frame"], 4)
    return out


def cornell_leg(wl, torch, ctx, repeats=20):
    """Configuration 1: the procedural Cornell box (36 triangles), 256x256 x 16 spp, depth 8,
    NEE+MIS, PCG32 seed 0, FP32 fast math: one render of 1,048,576 paths, the case dominated by
    per-launch overhead. Median device time of `repeats` renders, with direct launches and with
    CUDA-graph replay."""
    from wayland_b200 import scenes
    sc = scenes.cornell_box(256, 256, 16, 8)
    s = wl.Scene(ctx, sc, bvh_kind=BVH_KIND[0])
    cam = sc.camera_struct()
    stream = torch.cuda.ExternalStream(ctx.stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    out = {"scene": f"Cornell box {sc.num_tris} tris, 256x256, 16 spp, depth 8, PCG32 seed 0"}
    paths = 256 * 256 * 16
    for name, flags in (("launches", 0), ("graph", wl._abi.RENDER_GRAPH)):
        film = wl.Film(ctx, 256, 256)
        t = []
        for rep in range(repeats + 2):
            p = wl.render_params(256, 256, 16, max_depth=8, rng=wl.RNG_PCG32, seed=0,
                                 first_frame=16 * rep, flags=flags)
            ctx.sync()
            e0.record(stream)
            wl.render(ctx, s, cam, p, film)
            e1.record(stream)
            e1.synchronize()
            if rep >= 2:
                t.append(e0.elapsed_time(e1))
        ms = statistics.median(t)
        out[name] = {"ms": round(ms, 3), "mpaths_s": round(paths / ms / 1e3, 1)}
        film.close()
    s.close()
    return out


def batch_leg(wl, torch, ctx, stream, jobs=64):
    """Configuration 3: 64 procedural scenes (scenes.batch_scene: triangles lognormal in [10K, 5M],
    resolution, spp, depth and 1-8 lights drawn per scene), rendered one wl_render call per scene,
    as one wl_render_batch, and as one wl_render_batch replayed as a single CUDA graph
    (WL_RENDER_GRAPH; captured on the first round, replayed on the timed second round). Device
    time; Mpaths/s = all jobs' W x H x spp / time."""
    from wayland_b200 import scenes
    datas = [scenes.batch_scene(i) for i in range(jobs)]
    objs = [wl.Scene(ctx, d, bvh_kind=BVH_KIND[0]) for d in datas]
    params = [wl.render_params(d.width, d.height, d.spp, max_depth=d.max_depth) for d in datas]
    cams = [d.camera_struct() for d in datas]
    paths = sum(d.width * d.height * d.spp for d in datas)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    out = {"jobs": jobs, "triangles": int(sum(d.num_tris for d in datas)), "paths": int(paths)}
    gparams = [wl.render_params(d.width, d.height, d.spp, max_depth=d.max_depth, flags=wl._abi.RENDER_GRAPH)
               for d in datas]
    for mode in ("separate", "batch", "batch_graph") * 2:  # second round timed
        films = [wl.Film(ctx, d.width, d.height) for d in datas]
        ctx.sync()
        e0.record(stream)
        if mode == "batch":
            wl.render_batch(ctx, objs, cams, params, films)
        elif mode == "batch_graph":
            wl.render_batch(ctx, objs, cams, gparams, films)
        else:
            for o, c, p, f in zip(objs, cams, params, films):
                wl.render(ctx, o, c, p, f)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        out[mode] = {"ms": round(ms, 1), "mpaths_s": round(paths / ms / 1e3, 1)}
        for f in films:
            f.close()
    for o in objs:
        o.close()
    out["batch_gain"] = round(out["separate"]["ms"] / out["batch"]["ms"], 3)
    out["batch_graph_gain"] = round(out["separate"]["ms"] / out["batch_graph"]["ms"], 3)
    return out


def bdpt_ao_leg(wl, torch, ctx, res=1024, spp=256, oracle_spp=2048, ao_res=(512, 256)):
    """Configuration 5: the glass-sphere caustic scene (158,420 sphere triangles + plane + a
    0.05-wide quad light), roughness 0.05. BDPT with subpaths of at most 10 vertices: samples/s
    at res x res x spp (fast math), and the relMSE of that image against an FP64 oracle: the
    reference's BDPT estimator evaluated in WL_MATH_STRICT mode (per sample bit-identical to the
    reference's own BDPT.cu compiled on the host, which the strict-mode tests check) with an FP64
    film, oracle_spp samples per pixel of disjoint seeds. The oracle is rendered in two halves;
    relMSE(half A, half B) / 4 is its own noise floor. (A plain path tracer cannot serve: its
    estimate of the caustic through the glass sphere stays dominated by rare paths that hit the
    small light, with a noise floor far above 1.) AO: 4 camera samples x 32 occlusion rays of
    radius 0.1 per pixel at ao_res (about 2^24 rays). Device time with CUDA events on the
    library's stream."""
    from wayland_b200 import scenes
    sc = scenes.glass_sphere(res, res)
    scene = wl.Scene(ctx, sc, bvh_kind=BVH_KIND[0])
    cam = sc.camera_struct()
    stream = torch.cuda.ExternalStream(ctx.stream)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    film = wl.Film(ctx, res, res, fp64=True)
    p = wl.render_params(res, res, 8, strategy=wl.STRATEGY_BDPT, max_depth=10, first_frame=10000000)
    wl.render(ctx, scene, cam, p, film)  # first launches
    ctx.sync()
    film.close()
    film = wl.Film(ctx, res, res, fp64=True)
    p = wl.render_params(res, res, spp, strategy=wl.STRATEGY_BDPT, max_depth=10)
    torch.cuda.nvtx.range_push("bdpt")  # the window a profiler can select (--nvtx-include bdpt/)
    e0.record(stream)
    wl.render(ctx, scene, cam, p, film)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.nvtx.range_pop()
    ms = e0.elapsed_time(e1)
    st = ctx.stats()
    img = film.download64()
    film.close()
    t0 = time.perf_counter()
    halves = []
    for h in range(2):
        ref = wl.Film(ctx, res, res, fp64=True)
        wl.render(ctx, scene, cam, wl.render_params(res, res, oracle_spp // 2, strategy=wl.STRATEGY_BDPT,
                                                    max_depth=10, math=wl.MATH_STRICT,
                                                    first_frame=20000000 + h * oracle_spp), ref)
        halves.append(ref.download64())
        ref.close()
    oracle_s = time.perf_counter() - t0
    r64 = 0.5 * (halves[0] + halves[1])

    def rel(a, b):
        return float(((a - b) ** 2 / (b * b + 1e-2)).mean())

    samples = res * res * spp
    out = {"scene": f"glass sphere {sc.num_tris} tris, roughness 0.05, {res}x{res}, subpaths <= 10 vertices",
           "spp": spp, "ms": round(ms, 1), "msamples_s": round(samples / ms / 1e3, 2),
           "closest_hit_rays_per_sample": round(st["segments"] / samples, 3),
           "kernels_ms": {"closest_hit": round(st["ms_extend"], 1), "vertices_and_connect": round(st["ms_shade"], 1),
                          "connection_rays": round(st["ms_shadow"], 1), "other": round(st["ms_other"], 1)},
           "connection_rays_per_sample": round(st["shadow_rays"] / samples, 3),
           "relmse_vs_fp64_oracle": rel(img, r64),
           "oracle": f"BDPT in strict math (the reference's estimator, bit-exact per sample), {oracle_spp} spp, "
                     f"FP64 film, disjoint seeds ({oracle_s:.1f} s)",
           "oracle_noise_floor": float(((halves[0] - halves[1]) ** 2 / (r64 * r64 + 1e-2)).mean()) / 4}
    # the radiance cache on the camera subpaths: BDPT over the paths of at most cache_t vertices
    # after the camera, the cache's prediction at the cache_t-th eye vertex for the longer ones;
    # trained online (path-traced training paths every frame), warm-up frames without an image
    # included in the time
    # the cache at the second eye vertex: deeper cache vertices on this scene sit mostly in the
    # glass, where the path-traced training targets of caustic light are too noisy (measured at
    # 512^2 x 64 spp against the same oracle: relMSE 0.042 at the 2nd vertex, 0.046 at the 3rd,
    # 0.52 at the 4th, 6.4 at the 5th)
    cache_t, warm = 2, 16
    cache = wl.RadianceCache(ctx, scene, query_depth=cache_t)
    cp = wl.render_params(res, res, warm, strategy=wl.STRATEGY_BDPT, max_depth=10, first_frame=30000000)
    cache.reserve(cp)
    cfilm = wl.Film(ctx, res, res, fp64=True)
    ctx.sync()
    e0.record(stream)
    wl.render_nrc(ctx, scene, cam, cp, cache, None)
    wl.render_nrc(ctx, scene, cam, wl.render_params(res, res, spp, strategy=wl.STRATEGY_BDPT, max_depth=10),
                  cache, cfilm)
    e1.record(stream)
    e1.synchronize()
    cms = e0.elapsed_time(e1)
    cimg = cfilm.download64()
    cst = cache.stats()
    cfilm.close()
    cache.close()
    out["with_cache"] = {"cache_vertex": cache_t, "warmup_frames": warm, "spp": spp, "ms": round(cms, 1),
                         "msamples_s": round(samples / cms / 1e3, 2), "relmse_vs_fp64_oracle": rel(cimg, r64),
                         "train_samples_last_frame": cst["train_samples"],
                         "note": "paths of at most cache_t vertices after the camera by BDPT, longer ones by "
                                 "the cache at the cache_t-th eye vertex; time includes the warm-up frames "
                                 "and every frame's training step"}
    # ambient occlusion, radius 0.1
    aw, ah = ao_res
    afilm = wl.Film(ctx, aw, ah)
    ap = wl.ao_params(aw, ah, 1, radius=0.1)
    wl.render_ao(ctx, scene, cam, ap, afilm)
    ctx.sync()
    e0.record(stream)
    wl.render_ao(ctx, scene, cam, wl.ao_params(aw, ah, 1, radius=0.1, first_frame=1), afilm)
    e1.record(stream)
    e1.synchronize()
    ams = e0.elapsed_time(e1)
    rays = aw * ah * 4 * (1 + 32)
    afilm.close()
    out["ao"] = {"res": f"{aw}x{ah}", "rays": rays, "ms": round(ams, 2),
                 "mrays_s": round(rays / ams / 1e3, 1),
                 "note": "rays counted as 4 camera + 128 occlusion rays per pixel"}
    scene.close()
    return out


def nrc_convergence(wl, torch, ctx, res=(1920, 1080), oracle_spp=8192, target=1e-2,
                    budget_s=60.0, chunk=4, warmup_frames=16):
    """Configuration 4: time to relMSE <= target against an FP64-accumulated high-spp render, for
    the plain path tracer and for the radiance-cache path tracer (1 spp per frame), on the
    door-slit room (about 500K triangles, mostly indirect light) at 1920x1080. relMSE = mean over
    pixels and channels of (I - R)^2 / (R^2 + 1e-2). Times are device time of the render calls
    (CUDA events on the library's stream); the cache's time includes its warm-up frames
    (training only, no image) from a fresh cache. The oracle is rendered in two halves of
    disjoint frames; relMSE(half A, half B) / 4 is its own noise floor."""
    from wayland_b200 import scenes
    W_, H_ = res
    sc = scenes.door_slit_room(W_, H_)
    scene = wl.Scene(ctx, sc, bvh_kind=BVH_KIND[0])
    cam = sc.camera_struct()
    stream = torch.cuda.ExternalStream(ctx.stream)
    # oracle: FP64 films of two halves of disjoint frames, plain path tracer, fast math
    t0 = time.perf_counter()
    halves = []
    for h in range(2):
        hf = wl.Film(ctx, W_, H_, fp64=True)
        done = 0
        while done < oracle_spp // 2:
            k = min(512, oracle_spp // 2 - done)
            wl.render(ctx, scene, cam, wl.render_params(W_, H_, k, first_frame=1000000 + h * oracle_spp + done,
                                                        max_depth=16), hf)
            done += k
        halves.append(torch.from_numpy(hf.download64()).cuda())
        hf.close()
    ref = 0.5 * (halves[0] + halves[1])
    oracle_s = time.perf_counter() - t0
    noise_floor = float(((halves[0] - halves[1]) ** 2 / (ref * ref + 1e-2)).mean()) / 4
    del halves

    def relmse(img):
        x = torch.from_numpy(img).cuda().double()
        return float(((x - ref) ** 2 / (ref * ref + 1e-2)).mean())

    # first launches of the cache's kernels (module loading) outside the timed runs
    tmp = wl.RadianceCache(ctx, scene)
    wl.render_nrc(ctx, scene, cam, wl.render_params(W_, H_, 1, max_depth=16), tmp, None)
    ctx.sync()
    tmp.close()

    def run(kind):
        film = wl.Film(ctx, W_, H_)
        cache = wl.RadianceCache(ctx, scene) if kind == "nrc" else None
        if cache is not None:
            cache.reserve(wl.render_params(W_, H_, 1, max_depth=16))
        t_dev = 0.0
        spp = 0
        curve = []
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        if cache is not None and warmup_frames:
            e0.record(stream)
            wl.render_nrc(ctx, scene, cam, wl.render_params(W_, H_, warmup_frames, first_frame=5000000,
                                                            max_depth=16), cache, None)
            e1.record(stream)
            e1.synchronize()
            t_dev += e0.elapsed_time(e1) * 1e-3
        while True:
            n = chunk
            p = wl.render_params(W_, H_, n, first_frame=spp, max_depth=16)
            e0.record(stream)
            if cache is None:
                wl.render(ctx, scene, cam, p, film)
            else:
                wl.render_nrc(ctx, scene, cam, p, cache, film)
            e1.record(stream)
            e1.synchronize()
            t_dev += e0.elapsed_time(e1) * 1e-3
            spp += n
            err = relmse(film.download())
            curve.append((spp, round(t_dev, 4), err))
            if err <= target or t_dev > budget_s:
                break
        extra = {}
        if cache is not None:
            st = cache.stats()
            mq, mt = cache.kernel_times()
            extra = {"train_samples_last_frame": st["train_samples"], "queries_last_frame": st["queries"],
                     "kernel_ms_last_frame": {"mlp_query": round(mq, 4), "train_step": round(mt, 4)}}
            cache.close()
        film.close()
        reached = curve[-1][2] <= target
        return {"reached": reached, "seconds": curve[-1][1] if reached else None, "spp": curve[-1][0],
                "ms_per_frame": round(1e3 * curve[-1][1] / (curve[-1][0] + (warmup_frames if cache is not None else 0)), 3),
                "final_relmse": curve[-1][2], "curve": curve[:: max(1, len(curve) // 12)], **extra}

    plain = run("plain")
    torch.cuda.nvtx.range_push("nrc")  # the window a profiler can select (--nvtx-include nrc/)
    nrc = run("nrc")
    torch.cuda.nvtx.range_pop()
    scene.close()
    out = {"scene": f"door-slit room {sc.num_tris} tris, {W_}x{H_}, depth 16, fast math",
           "oracle": f"{oracle_spp} spp, FP64 film, plain path tracer ({oracle_s:.1f} s)",
           "oracle_noise_floor": noise_floor,
           "cache": "hash grid 16 levels x 2^19 entries x 2 FP16 features, MLP 64-64-64-64-64-16 BF16 "
                    "(FP32 accumulation), 2^14 training paths per frame",
           "target_relmse": target, "plain": plain, "nrc": nrc}
    if plain["seconds"] and nrc["seconds"]:
        out["nrc_time_fraction"] = round(nrc["seconds"] / plain["seconds"], 4)
    return out


def nrc_kernels(wl, torch, ctx, queries=1920 * 1080, samples=1 << 16, repeats=10, in_situ=None):
    """FLOP roofline of the radiance cache's tensor-core kernels at 1080p batch sizes: the query
    MLP on `queries` rows (34,816 FLOP per row) and the fused training step on `samples` rows
    (104,448 FLOP per row), through wl_nrc_mlp_forward / wl_nrc_train_step on device buffers;
    each kernel's own device time comes from wl_nrc_kernel_times (CUDA events around the
    tensor-core launch alone; median of repeats). in_situ: (queries, samples, ms_query, ms_train)
    of the last frame of a real 1080p cache render, reported beside it. Against the measured
    sustained BF16 peak."""
    from wayland_b200 import scenes
    sc = scenes.cornell_box(16, 16)
    s = wl.Scene(ctx, sc)
    c = wl.RadianceCache(ctx, s)
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    x = torch.rand((queries, 64), device="cuda", generator=g) * 2 - 1
    out = torch.empty((queries, 4), device="cuda")
    t = torch.rand((samples, 4), device="cuda", generator=g)
    tq, tt = [], []
    for r in range(repeats + 2):
        c.forward(x.data_ptr(), out.data_ptr(), queries)
        c.lib.wl_nrc_train_step(c.handle, wl._abi.C.c_void_p(x.data_ptr()), wl._abi.C.c_void_p(t.data_ptr()),
                                samples, None)
        mq, mt = c.kernel_times()
        if r >= 2:
            tq.append(mq)
            tt.append(mt)
    c.close()
    s.close()
    pk = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = pk.get("bf16_tflops_sustained", 1400.0)
    kind = "measured sustained" if "bf16_tflops_sustained" in pk else "fallback sustained"

    def entry(rows, ms, flop_per_row):
        tf = rows * flop_per_row / (ms * 1e-3) / 1e12 if ms > 0 else 0.0
        return {"rows": int(rows), "ms": round(ms, 4), "tflops": round(tf, 1), "frac": round(tf / peak, 4)}

    outd = {"mlp_query": entry(queries, statistics.median(tq), 34816),
            "train_step": entry(samples, statistics.median(tt), 104448),
            "peak_tflops": peak, "peak_kind": kind, "bound": "tensor",
            "timing": "wl_nrc_kernel_times: CUDA events around the tensor-core kernel alone"}
    if in_situ:
        nq, ns, mq, mt = in_situ
        outd["render_last_frame"] = {"mlp_query": entry(nq, mq, 34816), "train_step": entry(ns, mt, 104448)}
    return outd


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-raycast", action="store_true")
    ap.add_argument("--math", default="fast", choices=["fast", "strict"])
    ap.add_argument("--nrc-only", action="store_true",
                    help="only the radiance-cache convergence comparison (prints its JSON)")
    ap.add_argument("--no-nrc", action="store_true")
    ap.add_argument("--no-bdpt", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="skip the progressive 1-spp launches/graph leg")
    ap.add_argument("--no-cornell", action="store_true", help="skip the Cornell-box configuration leg")
    ap.add_argument("--bdpt-only", action="store_true", help="only the BDPT + AO leg (prints its JSON)")
    ap.add_argument("--bdpt-res", type=int, default=1024, help="image side of the BDPT leg")
    ap.add_argument("--bdpt-spp", type=int, default=256, help="samples per pixel of the BDPT leg")
    ap.add_argument("--bdpt-oracle-spp", type=int, default=2048, help="samples per pixel of its oracle")
    ap.add_argument("--nrc-res", default="1920x1080", help="resolution of the radiance-cache comparison")
    ap.add_argument("--nrc-oracle-spp", type=int, default=8192)
    ap.add_argument("--nrc-budget-s", type=float, default=60.0)
    ap.add_argument("--tune", default=None,
                    help="fixed launch shape as JSON (wl_set_tune fields) instead of the autotuner")
    ap.add_argument("--bvh", default="sah", choices=["sah", "lbvh"],
                    help="BVH build of every scene: binned SAH (default) or Morton LBVH")
    ap.add_argument("--case", default="full", choices=["full", "small"],
                    help="small: the same 2M-triangle scene at 960x540 x 4 spp (for ncu captures)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    BVH_KIND[0] = 1 if args.bvh == "sah" else 0  # wl.BVH_SAH / wl.BVH_LBVH
    if args.impl == "reference":
        return reference_arm(args)
    global W, H, SPP
    if args.case == "small":
        W, H, SPP = 960, 540, 4

    import torch
    import torch.distributed as dist
    import wayland_b200 as wl
    from wayland_b200 import scenes

    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    local = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    if args.bdpt_only:
        ctx = wl.Context(local)
        print(json.dumps(bdpt_ao_leg(wl, torch, ctx, res=args.bdpt_res, spp=args.bdpt_spp,
                                     oracle_spp=args.bdpt_oracle_spp)), flush=True)
        ctx.close()
        return 0
    if args.nrc_only:
        ctx = wl.Context(local)
        w_, h_ = (int(v) for v in args.nrc_res.split("x"))
        r = nrc_convergence(wl, torch, ctx, res=(w_, h_), oracle_spp=args.nrc_oracle_spp,
                            budget_s=args.nrc_budget_s)
        n = r["nrc"]
        ins = (n["queries_last_frame"], n["train_samples_last_frame"], n["kernel_ms_last_frame"]["mlp_query"],
               n["kernel_ms_last_frame"]["train_step"]) if "kernel_ms_last_frame" in n else None
        r["kernels"] = nrc_kernels(wl, torch, ctx, in_situ=ins)
        print(json.dumps(r), flush=True)
        ctx.close()
        return 0
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    scene = scenes.displaced_sphere(W, H, SPP, DEPTH)
    if args.case == "small":
        scene.camera = scenes.pinhole((0.0, 0.6, 4.2), (0.0, -0.2, 0.0), (0, 1, 0), 40.0, W, H)
    ctx = wl.Context(local)
    sc = wl.Scene(ctx, scene, bvh_kind=BVH_KIND[0])
    info = sc.info()
    film = wl.Film(ctx, W, H)
    stream = torch.cuda.ExternalStream(ctx.stream)
    cam = scene.camera_struct()
    math_mode = wl.MATH_FAST if args.math == "fast" else wl.MATH_STRICT
    # each rank renders its own 64 samples per pixel (frames rank*64 ...): weak scaling, no
    # data-path collective
    params = wl.render_params(W, H, SPP, max_depth=DEPTH, env=scene.env, math=math_mode,
                              first_frame=rank * SPP)
    paths = W * H * SPP

    def barrier():
        if world > 1:
            dist.barrier()

    # launch shapes (paths per wave, traversal CTAs per SM and refill threshold) chosen by the
    # project's autotuner on this scene, outside the timed region
    if args.tune:
        ctx.set_tune(json.loads(args.tune))
        tune = dict(json.loads(args.tune), fixed=True)
    else:
        tune = None if args.no_autotune else ctx.autotune(sc, cam, params)
    for _ in range(args.warmup):
        wl.render(ctx, sc, cam, params, film)
    ctx.sync()
    # untimed pass with traversal counters: segments per path, node visits and triangle tests
    sp = wl.render_params(W, H, SPP, max_depth=DEPTH, env=scene.env, math=math_mode,
                          first_frame=rank * SPP, flags=wl._abi.RENDER_TRAVERSAL_STATS)
    wl.render(ctx, sc, cam, sp, film)
    tstats = ctx.stats()

    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed")  # the window a profiler can select (--nvtx-include timed/)
    e0.record(stream)
    for _ in range(args.steps):
        wl.render(ctx, sc, cam, params, film)
    e1.record(stream)
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()
    barrier()
    clk = clocks.stop()
    # per-kernel device times of the last timed render (CUDA events the library records around
    # each launch on its stream)
    st = ctx.stats()
    ext_ms, shade_ms, shadow_ms, other_ms = st["ms_extend"], st["ms_shade"], st["ms_shadow"], st["ms_other"]
    launches = st["kernel_launches"] * args.steps
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    ms_step = ms_max / args.steps
    value = world * paths * args.steps / (ms_max * 1e-3) / 1e6

    # end to end through the public API with host buffers: render + film download per step, into
    # page-locked host memory (as a caller that reads a film every frame would keep it)
    host_film = torch.empty((H, W, 3), dtype=torch.float32, pin_memory=True).numpy()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        wl.render(ctx, sc, cam, params, film)
        film.download(host_film)
    e2e_s = (time.perf_counter() - t0) / args.steps
    et = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(et, op=dist.ReduceOp.MAX)
    e2e_value = world * paths / float(et.item()) / 1e6

    line = None
    if rank == 0:
        peak, peak_kind = peaks()
        segs = tstats["segments"]
        seg_per_path = segs / paths
        nodes_per = tstats["extend_node_visits"] / max(segs, 1)
        tris_per = tstats["extend_tri_tests"] / max(segs, 1)
        b_ray = 48 + 80 * nodes_per + 48 * tris_per
        achieved = segs * b_ray / (ext_ms * 1e-3) / 1e9
        b_path = 96 + 364 * seg_per_path
        # DRAM bytes per extend launch: the profiled bytes per ray x this run's rays per extend
        # launch (a wave launches generate, a counter reset and film once, and extend, a counter
        # reset, shade and shadow per bounce)
        ext_launches = max((st["kernel_launches"] - 3 * st["waves"]) // 4, 1)
        traffic = round(EXTEND_DRAM_BYTES_PER_RAY * segs / ext_launches) if args.case == "full" else None
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": METRIC, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": WORKLOAD if args.case == "full" else "profiling case: " + WORKLOAD.replace("1920x1080, 64 spp", f"{W}x{H}, {SPP} spp"), "width": W, "height": H, "spp": SPP, "max_depth": DEPTH,
                       "triangles": scene.num_tris, "math": args.math, "rng": "tea_lcg",
                       "strategy": "mis", "parallelism": f"{world} independent sample sets (weak)",
                       "l2": "working set larger than L2 (BVH %.0f MB + path queues), no flush" % (info["bytes"] / 1e6)},
            "e2e": {"value": round(e2e_value, 2), "unit": METRIC,
                    "h2d_bytes_per_step": 128, "d2h_bytes_per_step": W * H * 12},
            "roofline": {"bound": "hbm", "kernel": "k_extend (closest-hit traversal)",
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "traffic_source": TRAFFIC_SOURCE if traffic is not None else None,
                         "peak_kind": peak_kind,
                         "bytes_per_ray": round(b_ray, 1),
                         "algorithmic_bytes_per_launch": round(segs * b_ray / ext_launches),
                         "note": "algorithmic bytes = rays x (48 + 80 N_node + 48 N_tri); BVH nodes are mostly L2 hits, so DRAM traffic is far below this"},
            "roofline_path": {"bytes_per_path": round(b_path, 1),
                              "achieved_gbs": round(b_path * value * 1e6 / world / 1e9, 1),
                              "frac": round(b_path * value * 1e6 / world / 1e9 / peak, 4)},
            "kernels_ms_per_step": {"extend": round(ext_ms, 2), "shade": round(shade_ms, 2),
                                    "shadow": round(shadow_ms, 2), "other": round(other_ms, 2)},
            "segments_per_path": round(seg_per_path, 3),
            "shadow_rays_per_path": round(tstats["shadow_rays"] / paths, 3),
            "extend_nodes_per_ray": round(nodes_per, 2), "extend_tris_per_ray": round(tris_per, 2),
            "shadow_nodes_per_ray": round(tstats["shadow_node_visits"] / max(tstats["shadow_rays"], 1), 2),
            "shadow_tris_per_ray": round(tstats["shadow_tri_tests"] / max(tstats["shadow_rays"], 1), 2),
            "bvh": {"kind": "binned SAH" if BVH_KIND[0] == 1 else "LBVH",
                    "wide_nodes": info["wide_nodes"], "depth": info["wide_depth"],
                    "build_ms": round(info["ms_build"], 1)},
            "gpu_launches": launches,
            "autotune": tune,
            "clocks": clk,
        }
        def leg(key, fn):
            # an extra leg that fails is recorded in the line instead of losing the line
            try:
                line[key] = fn()
            except Exception as e:  # noqa: BLE001
                line[key] = {"error": f"{type(e).__name__}: {e}"}

        if not args.no_raycast:
            leg("raycast", lambda: raycast_microbench(wl, torch, ctx, sc, scene, stream, tune))
        if world == 1 and not args.no_graph:
            leg("progressive_1spp", lambda: graph_leg(wl, torch, ctx, sc, scene, stream))
        if world == 1 and not args.no_cornell:
            leg("cornell_config1", lambda: cornell_leg(wl, torch, ctx))
        if world == 1 and not args.no_batch:
            leg("batch", lambda: batch_leg(wl, torch, ctx, stream))
        if world == 1 and not args.no_bdpt:
            leg("bdpt", lambda: bdpt_ao_leg(wl, torch, ctx))
        if world == 1 and not args.no_nrc:
            # the second half of the metric: time to relMSE 1e-2 vs an FP64 high-spp render,
            # radiance cache vs plain path tracing (door-slit room)
            w_, h_ = (int(v) for v in args.nrc_res.split("x"))

            def nrc_leg():
                r = nrc_convergence(wl, torch, ctx, res=(w_, h_), oracle_spp=args.nrc_oracle_spp,
                                    budget_s=args.nrc_budget_s)
                n = r["nrc"]
                ins = None
                if "kernel_ms_last_frame" in n:
                    ins = (n["queries_last_frame"], n["train_samples_last_frame"],
                           n["kernel_ms_last_frame"]["mlp_query"], n["kernel_ms_last_frame"]["train_step"])
                r["kernels"] = nrc_kernels(wl, torch, ctx, in_situ=ins)
                return r
            leg("time_to_relmse", nrc_leg)
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            cpu = CpuPT(scene, threads)
            v, _, desc = cpu.sample()
            cpu.close()
            line["cpu_baseline"] = {"value": round(v, 4), "unit": METRIC, "cores": threads,
                                    "kind": cpu.kind, "sample": desc}
    film.close()
    sc.close()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
