"""Several render jobs in one shared wavefront (rb_render_jobs) against each
job rendered on its own (rb_render), through the C ABI.

A shared wave mixes the jobs' paths; every kernel reads each path's own
job's scene, and each pixel still accumulates its samples in sample order,
so every job's FP64 accumulation must equal its own render bit for bit,
whatever the wave capacity (jobs split across waves, or several jobs in a
wave) and whether a job starts at sample 0 or later."""
from __future__ import annotations

import numpy as np
import pytest

import cases
from oracle_lib import RefLib, reference_luts
from ratbite_b200 import lighttree, scenes
from ratbite_b200.rendering_interface import RenderingInterface, render_jobs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tables():
    ref = RefLib()
    return dict(cie=ref.cie_xyz(), basis=ref.basis_rgb(), luts=reference_luts())


def _jobs(tables):
    """Four jobs: different scenes, films, depths and light setups."""
    out = []
    for sc in (scenes.cornell_box(seed=1, cie_xyz=tables["cie"], width=48, height=40, spp=8, max_depth=8),
               cases.many_lights_scene(),
               scenes.scale_scene(seed=5, target_tris=40_000, n_emitters=64, width=64, height=36, spp=4, max_depth=12,
                                  envmap_size=(128, 64)),
               scenes.cornell_box(seed=7, cie_xyz=tables["cie"], width=17, height=9, spp=3, max_depth=3)):
        out.append((sc, lighttree.build_for_scene(sc)))
    return out


def _open(tables, sc, lt, **kw):
    ri = RenderingInterface(device=0, **kw)
    ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lt)
    return ri


@pytest.mark.parametrize("max_paths", [0, 3000])
def test_shared_wavefront_matches_each_job_alone(tables, max_paths):
    import torch
    jobs = _jobs(tables)
    offsets = [0, 0, 5, 0]
    counts = [8, 6, 4, 3]
    alone = []
    for (sc, lt), off, cnt in zip(jobs, offsets, counts):
        with _open(tables, sc, lt) as ri:
            if off:
                ri.clear_accumulation()
            ri.render(off, cnt)
            alone.append(ri.read_accumulation())
            assert ri.status().flags == 0
    ris = [_open(tables, sc, lt) for sc, lt in jobs]
    for ri, off in zip(ris, offsets):
        if off:
            ri.clear_accumulation()
    events = [torch.cuda.Event() for _ in ris]
    for e in events:
        e.record()                                  # creates the event the library records again
    render_jobs(ris, offsets, counts, max_paths=max_paths, done_events=events)
    torch.cuda.synchronize()
    for k, (ri, want) in enumerate(zip(ris, alone)):
        got = ri.read_accumulation()
        assert ri.status().flags == 0
        assert np.array_equal(got, want), k
        assert events[k].query()
    # a second call continues every job's accumulation (offsets past the first range)
    render_jobs(ris, [o + c for o, c in zip(offsets, counts)], [2, 2, 2, 2], max_paths=max_paths)
    for (sc, lt), off, cnt, ri in zip(jobs, offsets, counts, ris):
        with _open(tables, sc, lt) as solo:
            if off:
                solo.clear_accumulation()
            solo.render(off, cnt)
            solo.render(off + cnt, 2)
            assert np.array_equal(ri.read_accumulation(), solo.read_accumulation())
    for ri in ris:
        ri.cleanup()


def test_shared_wavefront_rejects_bad_jobs(tables):
    from ratbite_b200._native import NativeError
    jobs = _jobs(tables)[:2]
    ris = [_open(tables, sc, lt) for sc, lt in jobs]
    empty = RenderingInterface(device=0)             # no scene
    with pytest.raises(NativeError):
        render_jobs([ris[0], empty], [0, 0], [1, 1])
    for ri in ris + [empty]:
        ri.cleanup()


@pytest.mark.parametrize("grid_percent", [50, 200])
def test_shared_wavefront_on_a_caller_stream(tables, grid_percent):
    """The first call on fresh contexts allocates the wave and the job tables
    (zero-filled on the host context's own stream) and renders on a caller's
    stream with a large wave: the render must wait for the fills. Grids at
    half and twice the resident maximum give the same accumulations."""
    import torch
    jobs = _jobs(tables)
    counts = [5, 3, 2, 4]
    alone = []
    for (sc, lt), cnt in zip(jobs, counts):
        with _open(tables, sc, lt) as ri:
            ri.render(0, cnt)
            alone.append(ri.read_accumulation())
    ris = [_open(tables, sc, lt) for sc, lt in jobs]
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    render_jobs(ris, [0] * len(ris), counts, max_paths=12 << 20, grid_percent=grid_percent, stream=side.cuda_stream)
    side.synchronize()
    for k, (ri, want) in enumerate(zip(ris, alone)):
        assert ri.status().flags == 0
        assert np.array_equal(ri.read_accumulation(), want), k
        ri.cleanup()
