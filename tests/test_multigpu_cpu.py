"""The multi-rank frame (ratbite_b200.multigpu) on CPU: sample ranges,
per-rank accumulation restart and the all-reduce combine, with world_size 2
over gloo.

Each rank renders its sample range of a small Cornell box through an adapter
that gives the oracle (the reference's own per-sample code compiled for the
host) the RenderingInterface calls the multi-rank code makes; the combined
frame must equal one render of all samples, up to the order of the FP64
additions. The GPU path differs only in the renderer behind the same calls.
"""
from __future__ import annotations

import ctypes as C
import datetime
import os
import socket

import numpy as np
import pytest

from ratbite_b200 import multigpu


# ------------------------------------------------------------ sample ranges
@pytest.mark.parametrize("spp,world", [(64, 1), (64, 2), (64, 8), (5, 2), (7, 3), (3, 8), (0, 4)])
def test_sample_ranges_partition_the_frame(spp, world):
    ranges = [multigpu.sample_range(spp, r, world, base=11) for r in range(world)]
    covered = []
    for off, cnt in ranges:
        covered += list(range(off, off + cnt))
    assert covered == list(range(11, 11 + spp))            # disjoint, contiguous, in rank order
    counts = [c for _, c in ranges]
    assert max(counts) - min(counts) <= 1


def test_weak_ranges_are_disjoint():
    ranges = [multigpu.weak_sample_range(256, r) for r in range(8)]
    assert ranges[0] == (0, 256) and ranges[7] == (7 * 256, 256)
    ends = [o + c for o, c in ranges]
    assert all(ends[i] == ranges[i + 1][0] for i in range(7))


def test_bad_splits_raise():
    with pytest.raises(ValueError):
        multigpu.sample_range(8, 2, 2)
    with pytest.raises(ValueError):
        multigpu.sample_range(8, 0, 0)
    with pytest.raises(ValueError):
        multigpu.weak_sample_range(-1, 0)


# ------------------------------------------------------------ gloo ranks
W, H = 16, 16


class OracleRenderer:
    """The RenderingInterface calls used by multigpu, served by the oracle."""

    def __init__(self, ref):
        self.ref = ref
        self.clears = 0

    def render(self, offset, count, stream=None):
        assert self.ref.lib.rbref_render(offset, count, 2) == 0

    def clear_accumulation(self, stream=None):
        self.clears += 1
        zeros = np.zeros((H, W, 4), np.float64)
        self.ref.lib.rbref_write_accum(zeros.ctypes.data)

    def copy_accumulation_async(self, dst_ptr, stream=None):
        out = np.zeros((H, W, 4), np.float64)
        self.ref.lib.rbref_read_accum(out.ctypes.data)
        C.memmove(dst_ptr, out.ctypes.data, out.nbytes)


def _scene(ref):
    from oracle_lib import load_scene_into_ref, reference_luts
    from ratbite_b200 import scenes
    cie, basis = ref.cie_xyz(), ref.basis_rgb()
    sc = scenes.cornell_box(seed=1, cie_xyz=cie, width=W, height=H, spp=8, max_depth=4)
    return load_scene_into_ref(ref, sc, reference_luts(), cie, basis)


def _rank(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import torch
    import torch.distributed as dist
    from oracle_lib import RefLib
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        ref = RefLib()
        keep = _scene(ref)
        ri = OracleRenderer(ref)
        # strong split: 5 samples over 2 ranks (3 + 2)
        accum = torch.zeros((H, W, 4), dtype=torch.float64)
        off, cnt = multigpu.sample_range(5, rank, world)
        multigpu.render_frame(ri, accum, off, cnt)
        strong = accum.numpy().copy()
        # weak split, second frame on the same renderer: 3 samples per rank
        accum.zero_()
        off, cnt = multigpu.weak_sample_range(3, rank)
        multigpu.render_frame(ri, accum, off, cnt)
        weak = accum.numpy().copy()
        # an empty frame (0 samples): every range is empty, rank 0's included,
        # and the combine must give zeros, not the previous frame
        accum.zero_()
        off, cnt = multigpu.sample_range(0, rank, world)
        multigpu.render_frame(ri, accum, off, cnt)
        empty = accum.numpy().copy()
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), strong=strong, weak=weak, empty=empty, clears=ri.clears)
        del keep
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_combine_to_the_single_render(tmp_path):
    import torch.multiprocessing as mp
    from oracle_lib import RefLib, ref_render
    mp.spawn(_rank, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    ref = RefLib()
    keep = _scene(ref)
    want5 = ref_render(ref, W, H, 0, 5, threads=2)
    want6 = ref_render(ref, W, H, 0, 6, threads=2)
    del keep
    r0, r1 = np.load(tmp_path / "rank0.npz"), np.load(tmp_path / "rank1.npz")
    for key, want in (("strong", want5), ("weak", want6)):
        for r in (r0, r1):                       # every rank holds the whole frame
            got = r[key]
            assert np.array_equal(got[..., 3], want[..., 3])      # sample counts
            np.testing.assert_allclose(got[..., :3], want[..., :3], rtol=1e-12, atol=1e-300)
    for r in (r0, r1):
        assert not r["empty"].any()
    # rank 0's non-empty ranges start at sample 0 (the renderer restarts by
    # itself); rank 1 starts later in both and clears first; both clear for
    # the empty frame
    assert int(r0["clears"]) == 1 and int(r1["clears"]) == 3
