"""The multi-GPU film reduction's host logic with world_size 2 on CPU (gloo): each rank renders
its frame slice with the oracle into an FP64 mean, the all-reduce combines the sums, and the
result equals a single-process render of all frames."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import pyoracle as po
from wayland_b200 import multi, scenes


def test_frame_slices_cover_all_frames():
    for spp in (1, 5, 8, 64):
        for world in (1, 2, 3, 8):
            got = []
            for r in range(world):
                s, n = multi.frame_slice(spp, r, world, first_frame=10)
                got += list(range(s, s + n))
            assert got == list(range(10, 10 + spp))


def _params(spp, first):
    p = po.RenderParams(width=24, height=16, spp=spp, first_frame=first, max_depth=6, rr_depth=5,
                        rr_prob=0.9, eps=1e-3, strategy=2, rng=0, math=1, lights=0, seed=0)
    return p


def _cam(sc):
    c = po.Camera()
    for k in ("pos", "look_at", "up", "right"):
        getattr(c, k)[:] = [float(x) for x in sc.camera[k]]
    return c


def _rank(rank, world, port, spp, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sc = scenes.cornell_box(24, 16)
        start, n = multi.frame_slice(spp, rank, world)
        orc = po.Oracle()
        _, mean64, _ = orc.render(sc, _cam(sc), _params(n, start), prec=1, want64=True)
        sums = torch.from_numpy(mean64 * n)
        img = multi.allreduce_mean(sums, n)
        out[rank] = img.numpy().tobytes()
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_equals_one_render():
    spp = 5
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, spp, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs)
        imgs = [np.frombuffer(out[r], np.float64).reshape(16, 24, 3) for r in range(2)]
    sc = scenes.cornell_box(24, 16)
    _, ref, _ = po.Oracle().render(sc, _cam(sc), _params(spp, 0), prec=1, want64=True)
    assert np.array_equal(imgs[0], imgs[1])
    assert np.allclose(imgs[0], ref, rtol=1e-12, atol=1e-14)
