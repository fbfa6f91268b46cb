"""The two-level acceleration structure (rb_config.acceleration =
RB_ACCEL_INSTANCED: one BVH per unique mesh and per emissive subset, a top
level over the instances, as the reference's GAS per mesh and IAS,
src/core/rendering_interface.cpp:733-848, 943-1064) against the flat one.

Rays enter object space only for the box tests; triangles are intersected in
world space after the flat upload's own transform, so every hit, payload word
and image is bit-identical to the flat structure's, and so to the oracle's
(test_gpu_parity.py pins the flat structure's payloads to it). Memory scales
with the unique triangles, and an instance update rebuilds only the top level.
"""
from __future__ import annotations

import copy
import time

import numpy as np
import pytest

import cases
from gpu_util import dev, empty, host, ptr, torch
from oracle_lib import RefLib, reference_luts
from ratbite_b200 import abi, lighttree, scenes
from ratbite_b200._native import NativeError, check, load
from ratbite_b200.rendering_interface import RenderingInterface, render_jobs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tables():
    ref = RefLib()
    return dict(cie=ref.cie_xyz(), basis=ref.basis_rgb(), luts=reference_luts())


def _open(tables, sc, accel, lt=None):
    ri = RenderingInterface(device=0, acceleration=accel)
    ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"],
                  light_tree=lt if lt is not None else lighttree.build_for_scene(sc))
    return ri


def _scenes(tables):
    return [("cornell", scenes.cornell_box(seed=1, cie_xyz=tables["cie"], width=48, height=40, spp=8, max_depth=8)),
            ("many lights", cases.many_lights_scene()),
            ("scale", scenes.scale_scene(seed=5, target_tris=300_000, n_emitters=256, width=96, height=54, spp=8,
                                         max_depth=12, envmap_size=(128, 64))),
            ("textured", scenes.textured_cornell(seed=3, cie_xyz=tables["cie"], width=48, height=48, spp=8))]


def test_instanced_renders_bit_identically(tables):
    for name, sc in _scenes(tables):
        lt = lighttree.build_for_scene(sc)
        out = []
        for accel in (abi.RB_ACCEL_FLAT, abi.RB_ACCEL_INSTANCED):
            with _open(tables, sc, accel, lt) as ri:
                ri.render(0, 8)
                out.append(ri.read_accumulation())
                assert ri.status().flags == 0
        print(f"{name}: flat and instanced accumulations bit-identical: {np.array_equal(out[0], out[1])}")
        assert np.array_equal(out[0], out[1]), name


def _trace(ri, rays):
    n = len(rays)
    gpl, gt, gtri = empty(n * 24, torch().int32), empty(n, torch().float32), empty(n, torch().int32)
    tr = dev(rays)
    check(load().rb_k_trace(ri.ctx, n, ptr(tr), ptr(gpl), ptr(gt), ptr(gtri), None), ri.ctx, "trace")
    return host(gtri), host(gt).view(np.uint32), host(gpl).view(np.uint32).reshape(n, 24)


def _occluded(ri, rays, tmax):
    n = len(rays)
    out = empty(n, torch().int32)
    check(load().rb_k_occluded(ri.ctx, n, ptr(dev(rays)), ptr(dev(tmax)), ptr(out), None), ri.ctx, "occluded")
    return host(out).view(np.uint32)


def test_instanced_trace_and_occlusion_match_flat(tables):
    """Every payload word of the closest hit (world vertices, encoded normal,
    primitive, barycentrics, material, light pointer, normal matrix),
    the distance and the canonical triangle id, and the any-hit results."""
    sc = scenes.scale_scene(seed=5, target_tris=300_000, n_emitters=256, width=96, height=54, spp=8,
                            max_depth=12, envmap_size=(128, 64))
    rng = np.random.default_rng(7)
    n = 1 << 16
    o = np.stack([rng.uniform(-14, 14, n), rng.uniform(-3, 5, n), rng.uniform(-40, 0, n)], 1)
    o[: n // 4] = 0.0
    d = cases.unit_vectors(rng, n)
    rays = np.concatenate([o, d], 1).astype(np.float32)
    tmax = rng.uniform(0.1, 30.0, n).astype(np.float32)
    res = []
    for accel in (abi.RB_ACCEL_FLAT, abi.RB_ACCEL_INSTANCED):
        with _open(tables, sc, accel) as ri:
            res.append(_trace(ri, rays) + (_occluded(ri, rays, tmax),))
    (ft, fd, fp, fo), (it, idd, ip, io) = res
    hit = ft >= 0
    print(f"rays {n}: hits {hit.mean():.1%}, occluded {fo.mean():.1%}")
    assert hit.mean() > 0.2
    assert np.array_equal(ft, it)
    assert np.array_equal(fd[hit], idd[hit])
    assert np.array_equal(fp[hit], ip[hit])
    assert np.array_equal(fp[~hit][:, 8], ip[~hit][:, 8])
    assert np.array_equal(fo, io)


def test_instanced_update_matches_a_fresh_upload(tables):
    """Moving every instance (rb_update_instances: the top level rebuilt on
    the host) renders what a fresh upload of the moved scene renders, and
    what the flat structure's device refit renders."""
    sc = scenes.scale_scene(seed=5, target_tris=200_000, n_emitters=128, width=64, height=36, spp=4,
                            max_depth=8, envmap_size=(128, 64))
    rng = np.random.default_rng(3)
    moved = []
    for m, xf in sc.instances:
        x = np.asarray(xf, np.float32).copy()
        x[:, 3] += rng.uniform(-0.5, 0.5, 3).astype(np.float32)
        moved.append(x)
    subsets = [np.asarray(e["transform"], np.float32) for e in sc.emissive]
    lt = lighttree.build_for_scene(sc)
    imgs = []
    for accel in (abi.RB_ACCEL_FLAT, abi.RB_ACCEL_INSTANCED):
        with _open(tables, sc, accel, lt) as ri:
            ri.update_instances(np.stack(moved), np.stack(subsets) if subsets else None)
            ri.render(0, 4)
            imgs.append(ri.read_accumulation())
    fresh = copy.copy(sc)                                # keeps the environment map
    fresh.instances = [(m, x) for (m, _), x in zip(sc.instances, moved)]
    fresh._keep = []
    with _open(tables, fresh, abi.RB_ACCEL_INSTANCED, lt) as ri:
        ri.render(0, 4)
        imgs.append(ri.read_accumulation())
    assert not np.array_equal(imgs[0], _render_static(tables, sc, lt))
    assert np.array_equal(imgs[1], imgs[2])
    assert np.array_equal(imgs[0], imgs[1])


def _render_static(tables, sc, lt):
    with _open(tables, sc, abi.RB_ACCEL_INSTANCED, lt) as ri:
        ri.render(0, 4)
        return ri.read_accumulation()


def test_instanced_memory_time_and_update_cost(tables):
    """The at-scale scene (2.03M instanced triangles of 12 unique meshes):
    geometry memory, frame time and instance-update time of both structures."""
    import torch as T
    sc = scenes.scale_scene(seed=3, width=480, height=270, spp=4)
    lt = lighttree.build_for_scene(sc)
    moved = np.stack([np.asarray(x, np.float32) for _, x in sc.instances])
    subsets = np.stack([np.asarray(e["transform"], np.float32) for e in sc.emissive])
    stats = {}
    for accel, name in ((abi.RB_ACCEL_FLAT, "flat"), (abi.RB_ACCEL_INSTANCED, "instanced")):
        # geometry memory: one rb_set_geometry on a fresh context
        with RenderingInterface(device=0, acceleration=accel) as probe:
            g = sc.geometry_record()
            T.cuda.synchronize()
            free0 = T.cuda.mem_get_info()[0]
            probe.load_geometry(g)
            T.cuda.synchronize()
            used = free0 - T.cuda.mem_get_info()[0]
        with _open(tables, sc, accel, lt) as ri:
            ri.render(0, 1)                              # warm-up (wave buffers)
            T.cuda.synchronize()
            t0 = time.perf_counter()
            ri.render(1, 4)
            T.cuda.synchronize()
            frame = (time.perf_counter() - t0) / 4
            t0 = time.perf_counter()
            for _ in range(3):
                ri.update_instances(moved, subsets)
            T.cuda.synchronize()
            upd = (time.perf_counter() - t0) / 3
            assert ri.status().flags == 0
        stats[name] = (used, frame, upd)
        print(f"{name}: geometry {used / 2**20:.1f} MiB, {frame * 1e3:.1f} ms per 480x270 sample, "
              f"instance update {upd * 1e3:.2f} ms")
    assert stats["instanced"][0] < 0.5 * stats["flat"][0]


def test_shared_wavefront_rejects_instanced_contexts(tables):
    sc = scenes.cornell_box(seed=1, cie_xyz=tables["cie"], width=16, height=16, spp=1, max_depth=4)
    a = _open(tables, sc, abi.RB_ACCEL_INSTANCED)
    b = _open(tables, sc, abi.RB_ACCEL_FLAT)
    with pytest.raises(NativeError):
        render_jobs([a, b], [0, 0], [1, 1])
    a.cleanup()
    b.cleanup()


def test_instanced_cached_form_and_graphs(tables):
    """The two-level structure under the cached form (paths that never stop
    at the cache give the plain image bit for bit; with queries and training
    the status stays clean) and under graph replay (rb_render_graph equals
    rb_render)."""
    from ratbite_b200.nrc import RadianceCache
    sc = scenes.scale_scene(seed=5, target_tris=100_000, n_emitters=64, width=64, height=36, spp=8, max_depth=8,
                            envmap_size=(128, 64))
    lt = lighttree.build_for_scene(sc)
    with _open(tables, sc, abi.RB_ACCEL_FLAT, lt) as ri:
        ri.render(0, 8)
        want = ri.read_accumulation()
    with _open(tables, sc, abi.RB_ACCEL_INSTANCED, lt) as ri:
        cache = RadianceCache(seed=1)
        ri.attach_radiance_cache(cache, spread_threshold=1e30, frozen=True, samples_per_wave=8)
        ri.render(0, 8)
        assert np.array_equal(ri.read_accumulation(), want)
        ri.attach_radiance_cache(cache, samples_per_wave=8)
        ri.render(0, 16)
        st = ri.cache_stats()
        assert ri.status().flags == 0 and st.queries > 0 and np.isfinite(st.last_loss)
        ri.attach_radiance_cache(None)
        cache.close()
        ri.render_graph(0, 8)
        assert np.array_equal(ri.read_accumulation(), want)
