"""Checkpoint and resume of a progressive render (rb_write_accum plus the
next sample offset; RenderingInterface.save_checkpoint / load_checkpoint).

The reference's accumulation is resumable by construction (FP64 sums and
sample counts; the sample offset selects the Sobol indices,
src/kernels/pathtrace.cu:1120-1122) but lives only in its process. A render
interrupted after some samples, checkpointed, and resumed in a new context
ends bit-identical to the uninterrupted render."""
from __future__ import annotations

import numpy as np
import pytest

from oracle_lib import RefLib, reference_luts
from ratbite_b200 import lighttree, scenes
from ratbite_b200._native import NativeError
from ratbite_b200.rendering_interface import RenderingInterface

pytestmark = pytest.mark.gpu


def _open(sc, t):
    ri = RenderingInterface(device=0)
    ri.load_scene(sc, t["luts"], t["cie"], t["basis"], light_tree=lighttree.build_for_scene(sc))
    return ri


def test_resume_from_a_checkpoint_is_exact(tmp_path):
    ref = RefLib()
    t = dict(cie=ref.cie_xyz(), basis=ref.basis_rgb(), luts=reference_luts())
    sc = scenes.scale_scene(seed=5, target_tris=60_000, n_emitters=64, width=64, height=36, spp=16, max_depth=8,
                            envmap_size=(128, 64))
    with _open(sc, t) as ri:
        ri.render(0, 7)
        ri.render(7, 9)
        want = ri.read_accumulation()
    path = tmp_path / "frame.npz"
    with _open(sc, t) as ri:
        ri.render(0, 7)
        ri.save_checkpoint(path, 7)
    with _open(sc, t) as ri:
        nxt = ri.load_checkpoint(path)
        assert nxt == 7
        ri.render(nxt, 9)
        got = ri.read_accumulation()
        assert ri.status().flags == 0
    assert np.array_equal(got, want)
    # a checkpoint of another film size is refused
    small = scenes.scale_scene(seed=5, target_tris=60_000, n_emitters=64, width=32, height=18, spp=4,
                               max_depth=8, envmap_size=(128, 64))
    with _open(small, t) as ri:
        with pytest.raises(ValueError):
            ri.load_checkpoint(path)
        with pytest.raises(ValueError):
            ri.write_accumulation(np.zeros((36, 64, 4)))


def test_write_accumulation_round_trip():
    ref = RefLib()
    t = dict(cie=ref.cie_xyz(), basis=ref.basis_rgb(), luts=reference_luts())
    sc = scenes.cornell_box(seed=1, cie_xyz=t["cie"], width=24, height=16, spp=2, max_depth=4)
    with _open(sc, t) as ri:
        a = np.random.default_rng(1).uniform(0, 5, (16, 24, 4))
        ri.write_accumulation(a)
        assert np.array_equal(ri.read_accumulation(), a)
    empty = RenderingInterface(device=0)
    from ratbite_b200._native import load
    assert load().rb_write_accum(empty.ctx, a.ctypes.data) != 0     # no film yet
    empty.cleanup()


def test_render_on_the_default_stream_is_ordered_there():
    """A caller that passes torch's default stream (handle 0) gets its work
    ordered on that stream (cudaStreamLegacy), not on the library's own
    stream: an event recorded after the call completes only after the
    render, and a device-to-device copy of the accumulation enqueued behind
    it on the same stream sees the finished samples."""
    import torch
    ref = RefLib()
    t = dict(cie=ref.cie_xyz(), basis=ref.basis_rgb(), luts=reference_luts())
    sc = scenes.scale_scene(seed=5, target_tris=60_000, n_emitters=64, width=320, height=180, spp=64, max_depth=8,
                            envmap_size=(128, 64))
    with _open(sc, t) as ri:
        ri.render(0, 4)
        torch.cuda.synchronize()
        s = torch.cuda.current_stream()
        assert s.cuda_stream == 0
        out = torch.empty((180, 320, 4), dtype=torch.float64, device="cuda")
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        ri.render(4, 60, stream=s.cuda_stream)
        ri.copy_accumulation_async(out.data_ptr(), stream=s.cuda_stream)
        b.record()
        b.synchronize()
        ms = a.elapsed_time(b)
        got = out.cpu().numpy()
        assert np.array_equal(got, ri.read_accumulation())
        assert (got[..., 3] == 64).all()
        print(f"render on the default stream: {ms:.1f} ms between the events")
        assert ms > 1.0
        # graph replay too: captured on the library's stream, launched on the caller's
        ri.render_graph(64, 8, stream=s.cuda_stream)
        ri.copy_accumulation_async(out.data_ptr(), stream=s.cuda_stream)
        s.synchronize()
        assert (out[..., 3] == 72).all().item()
