"""Frames rendered by several ranks, one process per GPU.

The per-sample path shards without any exchange: pixels and Sobol sample
indices are independent, and the reference already addresses work by sample
range (LaunchParameters::samplingState offset / count,
src/core/launch_parameters.h:33-37, consumed at src/kernels/pathtrace.cu:1122).
Rank r renders its own disjoint sample range of every pixel into its own FP64
accumulation buffer; the frame is the element-wise sum of the ranks' buffers
(sum X, sum Y, sum Z, sample count per pixel), formed by one all-reduce. The
result does not depend on the number of ranks except for the order of the
FP64 additions.

Two ways to split a frame:
  strong  (sample_range)      a frame of S samples per pixel split into
                              contiguous blocks, the first S % G ranks taking
                              one extra sample;
  weak    (weak_sample_range) every rank renders S samples per pixel, rank r
                              the range [base + r*S, base + (r+1)*S).
"""
from __future__ import annotations


def sample_range(spp: int, rank: int, world: int, base: int = 0) -> tuple[int, int]:
    """(offset, count) of rank `rank` when `spp` samples are split over `world` ranks."""
    if world < 1 or not (0 <= rank < world) or spp < 0 or base < 0:
        raise ValueError("bad sample split")
    q, r = divmod(spp, world)
    count = q + (1 if rank < r else 0)
    offset = base + rank * q + min(rank, r)
    return offset, count


def weak_sample_range(spp_per_rank: int, rank: int, base: int = 0) -> tuple[int, int]:
    """(offset, count) of rank `rank` when every rank renders `spp_per_rank` samples."""
    if spp_per_rank < 0 or rank < 0 or base < 0:
        raise ValueError("bad sample split")
    return base + rank * spp_per_rank, spp_per_rank


def combine(accum, group=None):
    """Sums the ranks' FP64 accumulation tensors in place (one all-reduce)."""
    import torch.distributed as dist
    dist.all_reduce(accum, op=dist.ReduceOp.SUM, group=group)
    return accum


def render_range(ri, offset: int, count: int, stream=None):
    """Renders samples [offset, offset + count) into a fresh accumulation.

    The reference restarts its accumulation only when a launch starts at
    sample 0; a rank whose range starts later clears it first, and so does a
    rank with an empty range (it launches nothing, and must contribute
    zeros rather than its previous frame to the combine)."""
    if offset != 0 or count == 0:
        ri.clear_accumulation(stream=stream)
    if count:
        ri.render(offset, count, stream=stream)


def render_frame(ri, accum, offset: int, count: int, stream=None, group=None):
    """One rank's share of a frame, then the combine.

    `accum` is this rank's device tensor of height x width x 4 float64; it
    holds the whole frame on every rank afterwards. The copy and the
    all-reduce are ordered on `stream` (a torch.cuda.Stream) after the
    render."""
    import torch
    s = None if stream is None else stream.cuda_stream
    render_range(ri, offset, count, stream=s)
    ri.copy_accumulation_async(accum.data_ptr(), stream=s)
    if stream is None:
        combine(accum, group)
    else:
        with torch.cuda.stream(stream):
            combine(accum, group)
    return accum
