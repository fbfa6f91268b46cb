"""rb_render_graph on the GPU: the render call's waves captured once as a CUDA
graph and replayed with the call's sample offset read from device memory.
The accumulation must equal rb_render's bit for bit -- across calls that
share a graph (different offsets), calls of several wave sizes, and after a
setter changes the scene (the graph is captured again) -- and for small
launch-bound frames the replay should cost less host time per call.
"""
from __future__ import annotations

import time

import numpy as np
import pytest

from ratbite_b200 import assets, lighttree, scenes
from ratbite_b200.rendering_interface import RenderingInterface

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    cie, basis, luts = assets.cie_xyz(), assets.basis_rgb(), assets.luts()
    sc = scenes.cornell_box(seed=1, cie_xyz=cie, width=48, height=40, spp=8, max_depth=8)
    return sc, dict(luts=luts, cie=cie, basis=basis), lighttree.build_for_scene(sc)


def _ri(setup, capacity=0):
    sc, t, lt = setup
    ri = RenderingInterface(device=0, max_paths_in_flight=capacity)
    ri.load_scene(sc, t["luts"], t["cie"], t["basis"], light_tree=lt)
    return ri


def test_replayed_calls_equal_direct_calls(setup):
    ri = _ri(setup, capacity=48 * 40 * 3)        # several waves per call
    ri.render(0, 21)
    want = ri.read_accumulation()
    for off in (0, 7, 14):                        # one graph, three offsets
        ri.render_graph(off, 7)
    assert np.array_equal(ri.read_accumulation(), want)
    # two call shapes alternating (two graphs kept)
    ri.render_graph(0, 5)
    ri.render_graph(5, 16)
    assert np.array_equal(ri.read_accumulation(), want)
    ri.render(0, 5)
    ri.render(5, 16)
    assert np.array_equal(ri.read_accumulation(), want)
    assert ri.status().flags == 0
    ri.cleanup()


def test_setter_captures_again(setup):
    sc, t, lt = setup
    ri = _ri(setup)
    ri.render_graph(0, 4)
    first = ri.read_accumulation()
    mats = sc.material_records()
    mats[0].base_color[0] = 0.05                  # a different scene state
    ri.fill_model_materials(mats)
    ri.render_graph(0, 4)
    got = ri.read_accumulation()
    ri.render(0, 4)
    want = ri.read_accumulation()
    assert np.array_equal(got, want) and not np.array_equal(got, first)
    ri.cleanup()


def test_replay_costs_less_host_time_for_small_frames(setup):
    ri = _ri(setup)
    for f in (ri.render, ri.render_graph):
        f(0, 1)
    ri.synchronize()
    times = {}
    for name, f in (("rb_render", ri.render), ("rb_render_graph", ri.render_graph)):
        ri.synchronize()
        t0 = time.perf_counter()
        for k in range(200):
            f(k, 1)
        ri.synchronize()
        times[name] = (time.perf_counter() - t0) / 200 * 1e3
    print(f"48x40, depth 8, 1 spp per call: {times['rb_render']:.3f} ms per rb_render call, "
          f"{times['rb_render_graph']:.3f} ms per rb_render_graph call")
    assert times["rb_render_graph"] < times["rb_render"]
    ri.cleanup()
