"""rb_update_instances (device refit after the instances move) against a
fresh upload of the same moved scene, through the C ABI.

A camera move in the reference re-expresses every instance transform relative
to the new camera and rebuilds the instance acceleration structure
(src/core/rendering_interface.cpp:943-1063). Here the world vertices, the
geometric normals and the BVH boxes are recomputed on the device with the
tree topology kept. Closest hits do not depend on the tree's shape, so every
trace result (all 24 payload words, t, triangle) and every rendered sample
must equal those of a context built directly with the moved transforms:
the test requires bit equality.
"""
from __future__ import annotations

import copy

import numpy as np
import pytest

from gpu_util import dev, empty, host, ptr, torch
from oracle_lib import RefLib, reference_luts
from ratbite_b200 import abi, lighttree, scenes
from ratbite_b200._native import check, load
from ratbite_b200.rendering_interface import RenderingInterface

pytestmark = pytest.mark.gpu


def _moved(sc, delta):
    """The scene as seen from a camera moved by `delta`: every transform's
    translation minus delta, in float32 as the reference forms them."""
    m = copy.copy(sc)
    d = np.asarray(delta, np.float32)
    m.instances = []
    for mesh, xf in sc.instances:
        x = np.array(xf, np.float32).reshape(3, 4).copy()
        x[:, 3] = x[:, 3] - d
        m.instances.append((mesh, x))
    m.emissive = []
    for e in sc.emissive:
        e2 = dict(e)
        x = np.array(e["transform"], np.float32).reshape(3, 4).copy()
        x[:, 3] = x[:, 3] - d
        e2["transform"] = x
        m.emissive.append(e2)
    m._keep = []
    return m


def _context(sc, tables, lt):
    ri = RenderingInterface(device=0)
    ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lt)
    return ri


def _trace(ri, rays):
    """rays: (n, 6) float32, origin and direction per row."""
    assert rays.ndim == 2 and rays.shape[1] == 6 and rays.dtype == np.float32
    n = rays.shape[0]
    tr = dev(rays)
    pl, t, tri = empty(n * 24, torch().int32), empty(n, torch().float32), empty(n, torch().int32)
    check(load().rb_k_trace(ri.ctx, n, ptr(tr), ptr(pl), ptr(t), ptr(tri), None), ri.ctx, "trace")
    return host(pl).view(np.uint32), host(t), host(tri)


@pytest.mark.parametrize("delta", [(0.37, -0.21, 1.3), (-25.0, 3.5, 60.0)])
def test_refit_equals_fresh_upload(delta):
    ref = RefLib()
    tables = dict(cie=ref.cie_xyz(), basis=ref.basis_rgb(), luts=reference_luts())
    sc = scenes.scale_scene(seed=5, target_tris=60_000, n_emitters=48, width=64, height=36, spp=4, max_depth=6,
                            envmap_size=(64, 32))
    lt = lighttree.build_for_scene(sc)
    moved = _moved(sc, delta)
    a = _context(sc, tables, lt)
    a.update_instances(np.stack([x for _, x in moved.instances]),
                       np.stack([e["transform"] for e in moved.emissive]) if moved.emissive else None)
    b = _context(moved, tables, lt)
    # camera rays: from the original camera (at -delta in the moved frame)
    # into the view frustum around -z, plus random rays from near it
    rng = np.random.default_rng(7)
    n = 20000
    o = np.tile(-np.asarray(delta, np.float64), (n, 1))
    o[n // 2:] += rng.normal(0.0, 1.0, (n - n // 2, 3))
    d = np.stack([rng.uniform(-0.7, 0.7, n), rng.uniform(-0.4, 0.4, n), -np.ones(n)], axis=1)
    d[n // 2:] = rng.normal(0.0, 1.0, (n - n // 2, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.ascontiguousarray(np.concatenate([o, d], axis=1), np.float32)
    pa, ta, ia = _trace(a, rays)
    pb, tb, ib = _trace(b, rays)
    print(f"refit: hits {np.mean(ia >= 0):.2%} of {len(ia)} rays")
    assert len(ia) == n
    assert np.mean(ia >= 0) > 0.2
    assert np.array_equal(ia, ib)
    assert np.array_equal(ta.view(np.uint32), tb.view(np.uint32))
    assert np.array_equal(pa, pb)
    a.render(0, 4)
    b.render(0, 4)
    ga, gb = a.read_accumulation(), b.read_accumulation()
    assert np.array_equal(ga, gb)
    for ri in (a, b):
        st = ri.status()
        assert st.flags == 0
        ri.cleanup()


@pytest.mark.parametrize("delta", [(0.37, -0.21, 1.3), (-25.0, 3.5, 60.0)])
def test_camera_move_on_device_equals_host_refresh(delta):
    """The whole camera-move refresh on the device -- rb_update_instances for
    the transforms and rb_set_light_origin for the light data -- against a
    fresh context given the moved transforms and the light records refreshed
    on the host as the reference does (fillLightDataBuffer /
    fillLightTreeDataBuffers: float32 world value - camera position): the
    renders must be bit-identical."""
    ref = RefLib()
    tables = dict(cie=ref.cie_xyz(), basis=ref.basis_rgb(), luts=reference_luts())
    sc = scenes.scale_scene(seed=5, target_tris=60_000, n_emitters=48, width=64, height=36, spp=4, max_depth=6,
                            envmap_size=(64, 32))
    lt = lighttree.build_for_scene(sc)
    moved = _moved(sc, delta)
    a = _context(sc, tables, lt)
    a.update_instances(np.stack([x for _, x in moved.instances]),
                       np.stack([e["transform"] for e in moved.emissive]) if moved.emissive else None)
    a.set_light_origin(delta)
    tris, nodes, ptrs, masks = lt._arrays
    cam = np.asarray(delta, np.float32)
    t2, n2 = tris.copy(), nodes.copy()
    t2["vertices"] = (t2["vertices"].reshape(-1, 3, 3) - cam).reshape(-1, 9)
    n2["mean"] = n2["mean"] - cam
    b = _context(moved, tables, lighttree.record(t2, n2, ptrs.copy(), masks.copy()))
    a.render(0, 4)
    b.render(0, 4)
    ga, gb = a.read_accumulation(), b.read_accumulation()
    assert ga[..., :3].sum() > 0
    assert np.array_equal(ga, gb)
    # and back: origin 0 restores the light data as loaded
    a.set_light_origin((0.0, 0.0, 0.0))
    a.update_instances(np.stack([x for _, x in sc.instances]),
                       np.stack([e["transform"] for e in sc.emissive]) if sc.emissive else None)
    c = _context(sc, tables, lt)
    a.render(0, 4)
    c.render(0, 4)
    assert np.array_equal(a.read_accumulation(), c.read_accumulation())
    for ri in (a, b, c):
        assert ri.status().flags == 0
        ri.cleanup()


def test_refit_rejects_bad_transforms():
    ref = RefLib()
    tables = dict(cie=ref.cie_xyz(), basis=ref.basis_rgb(), luts=reference_luts())
    sc = scenes.cornell_box(seed=1, cie_xyz=tables["cie"], width=16, height=16, spp=1)
    ri = _context(sc, tables, lighttree.build_for_scene(sc))
    xf = np.stack([x for _, x in sc.instances]).astype(np.float32)
    sub = np.stack([e["transform"] for e in sc.emissive]).astype(np.float32)
    bad = xf.copy()
    bad[0, 0, 0] = np.nan
    assert load().rb_update_instances(ri.ctx, bad.ctypes.data, sub.ctypes.data, None) == abi.RB_ERR_INVALID
    assert load().rb_update_instances(ri.ctx, None, sub.ctypes.data, None) == abi.RB_ERR_INVALID
    ri.update_instances(xf, sub)                         # the same transforms: a no-op move
    ri.cleanup()
