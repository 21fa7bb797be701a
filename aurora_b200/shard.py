"""Splitting one render over several ranks (one process per GPU).

The path has no exchange step: every (pixel, sample) is independent and each rank
holds its own copy of the scene and BVH. A rank renders a contiguous range of sample
indices of the full frame (the counter-based random numbers depend only on the pixel
and the sample index, so the union of the ranks' samples is exactly the samples of one
single-GPU render), and the films are combined once at the end with one all-reduce. The
path-replay adjoint splits the same way, and its per-material and texel gradients are
combined with one all-reduce (sum) as well.
"""
from __future__ import annotations


def sample_range(rank: int, world: int, spp: int, scaling: str = "strong") -> tuple[int, int]:
    """(first sample index, sample count) of `rank`.

    strong: the frame's `spp` samples are split over the ranks (the first spp % world
    ranks take one more). weak: every rank renders `spp` samples of its own range
    [rank * spp, (rank + 1) * spp)."""
    if world < 1 or not 0 <= rank < world or spp < 0:
        raise ValueError(f"sample_range: rank {rank} of {world}, spp {spp}")
    if scaling == "weak":
        return rank * spp, spp
    if scaling != "strong":
        raise ValueError(f"sample_range: unknown scaling {scaling!r}")
    base, extra = divmod(spp, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def combine_films(film, count: int, group=None):
    """Sample-count weighted mean of the ranks' films (RGB mean + alpha), in place.

    `film` is this rank's (H, W, 4) float32 mean over its `count` samples; after the call
    every rank holds the mean over all ranks' samples. One all-reduce of the film (FP64)
    and one of the counts."""
    import torch
    import torch.distributed as dist
    acc = film.to(torch.float64) * float(count)
    n = torch.tensor([float(count)], dtype=torch.float64, device=acc.device)
    dist.all_reduce(acc, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(n, op=dist.ReduceOp.SUM, group=group)
    film.copy_((acc / n.clamp_min(1.0)).to(film.dtype))
    return film


def max_over_ranks(value: float, group=None, device=None) -> float:
    """The largest `value` over all ranks (device timings are reported as the max)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t[0])


def render_sharded(scene, opts, out, group=None, scaling: str = "strong"):
    """Renders this rank's sample range of `opts` into `out` (a (H, W, 4) torch tensor on the
    scene's device) and combines the films: with strong scaling the result equals a
    single-GPU render of opts.spp samples, up to the rounding of the combine."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    first, count = sample_range(rank, world, opts.spp, scaling)
    if count > 0:
        o = type(opts).from_buffer_copy(opts)
        o.spp, o.sample_offset = count, opts.sample_offset + first
        scene.render(o, out=out)
    else:
        out.zero_()
    return combine_films(out, count, group)


def combine_gradients(grads, count: int, total: int, group=None, device=None):
    """Gradients of a loss on the mean film over all ranks' samples, in place.

    `grads` are this rank's float32 arrays (per-material and texel gradients) of the same loss
    on the mean film over its own `count` samples; the film over all `total` samples is the
    count-weighted mean of the ranks' films, so its gradient is the sum over ranks of
    count / total times theirs: one all-reduce (sum, FP64) of all the arrays together. `device`:
    where the reduced tensor lives (a CUDA device with NCCL, None for the CPU with gloo)."""
    import numpy as np
    import torch
    import torch.distributed as dist
    arrays = [np.asarray(g) for g in grads]
    flat = np.concatenate([a.astype(np.float64).ravel() for a in arrays]) * (float(count) / float(max(total, 1)))
    t = torch.from_numpy(flat)
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    out = t.cpu().numpy()
    k = 0
    for a in arrays:
        a[...] = out[k:k + a.size].reshape(a.shape).astype(a.dtype)
        k += a.size
    return grads


def adjoint_sharded(scene, opts, dloss_dfilm, group=None, scaling: str = "strong", device=None):
    """The path-replay adjoint of `opts` split over the ranks like render_sharded: each rank
    replays its sample range and the gradients are combined with one all-reduce. With strong
    scaling the result is the single-GPU adjoint of opts.spp samples (same random numbers),
    up to the rounding of the sum. Returns (grad_mat, grad_tex) on every rank."""
    import numpy as np
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    first, count = sample_range(rank, world, opts.spp, scaling)
    gm = np.zeros((scene.nmat, 4), np.float32)
    gt = np.zeros(max(scene.ntexel, 1), np.float32)
    if count > 0:
        o = type(opts).from_buffer_copy(opts)
        o.spp, o.sample_offset = count, opts.sample_offset + first
        scene.adjoint(o, dloss_dfilm, gm, gt)
    total = opts.spp if scaling == "strong" else world * opts.spp
    combine_gradients((gm, gt), count, total, group, device)
    return gm, gt
