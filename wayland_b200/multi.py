"""One image rendered by several GPUs (one process per GPU, torch.distributed over NCCL).

Path samples are independent, so each rank renders a disjoint slice of the image's frames
(frame = sample index per pixel; the frames of all ranks together are exactly those of a
single-GPU render) into an FP64-sum film, and one all-reduce (sum) of the W x H x 3 doubles
gives every rank the mean image. The reduction is the film's only exchange; the path tracer
needs none. (The reference renders on one device: ContextManager.cpp:147-194 sets up one
OptiX context per CUDA device but the renderer uses the first.)
"""
import ctypes as C

import numpy as np

from . import _abi


def frame_slice(spp, rank, world, first_frame=0):
    """(first frame, frames) of rank's share of spp samples per pixel: contiguous slices, the
    first spp % world ranks one frame longer."""
    base, extra = divmod(spp, world)
    count = base + (1 if rank < extra else 0)
    start = first_frame + rank * base + min(rank, extra)
    return start, count


class _DeviceArray:
    """A device buffer seen by torch through the CUDA array interface."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"data": (ptr, False), "shape": shape, "typestr": typestr,
                                         "version": 3}


def film_sum_tensor(film):
    """The film's FP64 sum buffer (H, W, 3) as a torch tensor sharing the device memory."""
    import torch
    _, sum64, _ = film.device_ptrs()
    if not sum64:
        raise ValueError("the film has no FP64 sum (create it with fp64=True)")
    return torch.as_tensor(_DeviceArray(sum64, (film.height, film.width, 3), "<f8"),
                           device=f"cuda:{film.ctx.device}")


def allreduce_mean(sums, frames, group=None):
    """Sum the per-rank FP64 sums and frame counts over the process group; returns the mean
    image (sums / total frames). sums: a torch tensor (device tensor with NCCL, host with gloo),
    reduced in place."""
    import torch
    import torch.distributed as dist
    n = torch.tensor([float(frames)], dtype=torch.float64, device=sums.device)
    dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(n, op=dist.ReduceOp.SUM, group=group)
    return sums / n


def render_distributed(wl, ctx, scene, camera, params, film, rank, world, group=None):
    """Render params.spp samples per pixel of one image on `world` ranks: this rank's frame slice
    into film (an FP64-sum film, fresh), then the all-reduce. Returns the mean image as a device
    tensor (identical on every rank) and this rank's frame count."""
    p = _abi.RenderParams()
    C.memmove(C.byref(p), C.byref(params), C.sizeof(p))
    start, count = frame_slice(params.spp, rank, world, params.first_frame)
    if count:
        p.first_frame = start
        p.spp = count
        wl.render(ctx, scene, camera, p, film)
    ctx.sync()
    sums = film_sum_tensor(film).clone()
    return allreduce_mean(sums, count, group), count


def mean_image(film):
    """Host copy of a film's FP64 mean (single process)."""
    return np.asarray(film.download64())
