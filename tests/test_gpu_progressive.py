"""Progressive rendering (rb_progressive_restart / rb_progressive_step) on the
GPU: the sub-launch schedule of the reference's render loop
(src/core/rendering_interface.cpp:1846-1872, 1980-2013), and accumulation
that equals one render of all samples bit for bit (samples are accumulated
per pixel in sample order whatever the sub-launch boundaries are).
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle_lib import RefLib, reference_luts
from ratbite_b200 import abi, lighttree, scenes
from ratbite_b200._native import load
from ratbite_b200.rendering_interface import RenderingInterface

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    ref = RefLib()
    cie, basis = ref.cie_xyz(), ref.basis_rgb()
    sc = scenes.cornell_box(seed=1, cie_xyz=cie, width=48, height=48, spp=8)
    lt = lighttree.build_for_scene(sc)
    return sc, dict(luts=reference_luts(), cie=cie, basis=basis), lt


def _ri(setup):
    sc, t, lt = setup
    ri = RenderingInterface(device=0, max_paths_in_flight=48 * 48 * 7)   # several waves per sub-launch
    ri.load_scene(sc, t["luts"], t["cie"], t["basis"], light_tree=lt)
    return ri


def _plan(total, mode):
    offs = np.zeros(256, np.uint32)
    cnts = np.zeros(256, np.uint32)
    n = load().rb_progressive_plan(total, mode, offs.ctypes.data, cnts.ctypes.data, 256)
    return list(zip(offs[:n].tolist(), cnts[:n].tolist()))


@pytest.mark.parametrize("mode", [abi.RB_MODE_GRADUAL, abi.RB_MODE_IMMEDIATE])
def test_progressive_equals_single_render(setup, mode):
    total = 40 if mode == abi.RB_MODE_GRADUAL else 6
    ri = _ri(setup)
    ri.progressive_restart(total, mode)
    launched = []
    for _ in range(100):
        p = ri.progressive_step()
        if p.launched_count == 0:
            assert p.finished
            break
        launched.append((p.launched_offset, p.launched_count))
        assert p.processed == p.launched_offset
    assert launched == _plan(total, mode)
    got = ri.read_accumulation()
    ri.render(0, total)
    want = ri.read_accumulation()
    ri.cleanup()
    assert np.all(got[..., 3] == total)
    assert np.array_equal(got, want)


def test_restart_discards_the_previous_render(setup):
    ri = _ri(setup)
    ri.progressive_restart(40, abi.RB_MODE_GRADUAL)
    ri.progressive_step()
    ri.progressive_step()                       # samples 0..5 rendered
    ri.progressive_restart(3, abi.RB_MODE_IMMEDIATE)
    while not ri.progressive_step().finished:
        pass
    got = ri.read_accumulation()
    ri.render(0, 3)
    want = ri.read_accumulation()
    ri.cleanup()
    assert np.array_equal(got, want)
