"""Batched jobs on the GPU (ratbite_b200.batch): a few small jobs rendered
together, the plain ones in one shared wavefront (rb_render_jobs), the
cached one on its own stream. Each plain job's accumulation must equal
rendering the job alone with rb_render bit for bit; the cached job's image
must be finite; every job reports a completion time.
"""
from __future__ import annotations

import numpy as np
import pytest

from ratbite_b200 import batch
from ratbite_b200.rendering_interface import RenderingInterface

pytestmark = pytest.mark.gpu


def test_batched_jobs_equal_individual_renders():
    jobs = [batch.Job(0, 11, 128, 24, 20_000, "plain"), batch.Job(1, 12, 256, 16, 40_000, "plain"),
            batch.Job(2, 13, 128, 40, 30_000, "cached"), batch.Job(3, 14, 128, 8, 20_000, "plain")]
    br = batch.BatchRenderer(jobs, threads=4)
    res = br.run(batch.Schedule(max_paths=1 << 20, grid_percent=100, streams=2, chunk=16), keep_images=True)
    print(f"4 small jobs: {res.paths_per_s / 1e6:.1f} M paths/s, p50 {res.percentile(50) * 1e3:.2f} ms, "
          f"p99 {res.percentile(99) * 1e3:.2f} ms")
    assert len(res.latencies) == 4 and all(t > 0 for t in res.latencies)
    for j in jobs:
        img = res.images[j.index]
        assert np.all(np.isfinite(img)) and np.all(img[..., 3] == j.spp)
        if j.form != "plain":
            continue
        sc, lt = br.scenes[j.index]
        ri = RenderingInterface(device=0)
        ri.load_scene(sc, br.luts, br.cie, br.basis, light_tree=lt, max_depth=sc.max_depth)
        ri.render(0, j.spp)
        want = ri.read_accumulation()
        ri.cleanup()
        assert np.array_equal(img, want), f"job {j.index}"
