"""One image across GPUs: disjoint sample ranges of the same frame, one rank a GPU, summed into rank 0's accum.

The reference renders one adapter's image one sample a dispatch (renderer/src/gpu.rs:4176-4196, `Params.size.z` the
sample index): every sample of a pixel is drawn from (pixel, sample, vertex, decision) alone, so samples
[first, first + k) rendered on another GPU are the very samples one GPU would render there, and an image split by
sample ranges is exact up to the order its sums are taken in. Each rank renders its range into its own accum
(trt_render with first_sample), copies it into a tensor on its device (trt_accum_copy) and one sum-reduce
(torch.distributed over NCCL) brings the 80-byte Pixel records together on rank 0. The scene is replicated on every
rank; nothing but the accum crosses NVLink.
"""
from __future__ import annotations


def sample_range(rank: int, world: int, spp: int) -> tuple[int, int]:
    """(first sample, samples) of rank `rank`: contiguous ranges covering [0, spp), the remainder on the first ranks."""
    if world < 1 or not 0 <= rank < world or spp < 0:
        raise ValueError("sample_range: bad rank, world or spp")
    base, extra = divmod(spp, world)
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def reduce_accum(dist, accum, dst: int = 0):
    """Sums the ranks' accum tensors (w * h * 20 float32, on each rank's device or the CPU for gloo) into rank dst's."""
    dist.reduce(accum, dst=dst, op=dist.ReduceOp.SUM)
    return accum


def render_split(scene, params, spp: int, rank: int, world: int, dist, accum, flags: int = 0):
    """Renders this rank's samples of the frame into `scene`'s accum, copies it into `accum` (a torch tensor of
    w * h * 20 float32 on this rank's device) and, given a process group (dist), sums every rank's into rank 0's.
    Returns this rank's Stats."""
    first, k = sample_range(rank, world, spp)
    _, st = scene.render_raw(params, k, first_sample=first, flags=flags, read=False)
    scene.accum_copy(accum.data_ptr(), accum.numel() * 4)
    if dist is not None and world > 1:
        reduce_accum(dist, accum)
    return st
