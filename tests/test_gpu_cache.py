"""The cached form of rb_render on the GPU (include/ratbite_b200_nrc.h):
paths that terminate into the radiance cache, training paths that record
their vertices, and the optimiser steps the wave feeds.

1. The cache machinery leaves the plain estimator alone: with a threshold no
   path reaches, or with every path a training path, no path terminates and
   the accumulation equals the plain render bit for bit.
2. What the trained network gains: on the Cornell box (the plain method's
   small workload, depth 12) the trained cache's image at 16 samples per
   pixel is closer to a 2048-spp plain reference than the plain tracer's at
   16 spp, and an untrained cache (same termination, no training) is worse
   than the trained one: the gain comes from what the network learned.
3. The cached form is close to unbiased against the plain estimator: after
   training, the mean of the image matches the reference's within 5 %
   (measured +0.5 % with the drop and radiance corrections, -0.2 % to
   -2.8 % before them; the training's float atomics make each run's
   trajectory differ). An untrained cache is +43 % off, and a cache that
   ignored the reference's dropped samples was +7 % off.
4. The corrections measured on the training rows at the would-be query
   vertex are in use after training: a finite drop-probability correction
   per class and a radiance scale within its [0.5, 2] clamp.
"""
from __future__ import annotations

import numpy as np
import pytest

from ratbite_b200 import assets, lighttree, scenes
from ratbite_b200.nrc import RadianceCache
from ratbite_b200.rendering_interface import RenderingInterface

pytestmark = pytest.mark.gpu

W = H = 128


@pytest.fixture(scope="module")
def setup():
    cie, basis, luts = assets.cie_xyz(), assets.basis_rgb(), assets.luts()
    sc = scenes.cornell_box(seed=1, cie_xyz=cie, width=W, height=H, spp=4, max_depth=12)
    return sc, dict(luts=luts, cie=cie, basis=basis), lighttree.build_for_scene(sc)


def _ri(setup):
    sc, t, lt = setup
    ri = RenderingInterface(device=0)
    ri.load_scene(sc, t["luts"], t["cie"], t["basis"], light_tree=lt)
    return ri


def _mean(acc):
    return acc[..., :3] / np.maximum(acc[..., 3:4], 1.0)


def _rel_rmse(img, ref):
    return float(np.sqrt(np.mean((img - ref) ** 2)) / np.mean(ref))


def test_paths_that_never_terminate_match_the_plain_render(setup):
    ri = _ri(setup)
    ri.render(0, 8)
    want = ri.read_accumulation()
    cache = RadianceCache(seed=1)
    ri.attach_radiance_cache(cache, spread_threshold=1e30, frozen=True, samples_per_wave=8)
    ri.render(0, 8)
    assert np.array_equal(ri.read_accumulation(), want)
    st = ri.cache_stats()
    assert st.queries == 0 and st.records == 0 and st.steps == 0
    # every path a training path: vertices are recorded and trained on, the image is the plain one
    ri.attach_radiance_cache(cache, train_one_in=1, targets_per_sample=4096, batch=16384, samples_per_wave=8)
    ri.render(0, 8)
    assert np.array_equal(ri.read_accumulation(), want)
    st = ri.cache_stats()
    assert st.queries == 0 and st.records > 8 * W * H and st.steps == 2 and np.isfinite(st.last_loss)
    assert ri.status().flags == 0
    ri.attach_radiance_cache(None)
    ri.render(0, 8)
    assert np.array_equal(ri.read_accumulation(), want)
    ri.cleanup()
    cache.close()


def test_trained_cache_reduces_error_at_equal_samples(setup):
    spp = 16
    ri = _ri(setup)
    ri.render(1 << 16, 2048)            # reference: independent samples
    ref = _mean(ri.read_accumulation())
    ri.render(0, spp)
    plain = _rel_rmse(_mean(ri.read_accumulation()), ref)

    untrained = RadianceCache(seed=2)
    ri.attach_radiance_cache(untrained, frozen=True)
    ri.render(0, spp)
    cold_img = _mean(ri.read_accumulation())
    cold = _rel_rmse(cold_img, ref)
    st = ri.cache_stats()
    assert st.queries > 0 and st.steps == 0

    cache = RadianceCache(seed=2)
    ri.attach_radiance_cache(cache, targets_per_sample=16384, batch=16384)
    ri.render(1 << 20, 256)             # training frames
    warm = ri.cache_stats()
    ri.render(0, spp)
    img = _mean(ri.read_accumulation())
    cached = _rel_rmse(img, ref)
    st = ri.cache_stats()
    bias = float(img[..., 1].mean() / ref[..., 1].mean() - 1.0)
    cold_bias = float(cold_img[..., 1].mean() / ref[..., 1].mean() - 1.0)
    print(f"cached form, {W}x{H} Cornell box depth 12, {spp} spp: relative RMSE plain {plain:.4f}, "
          f"untrained cache {cold:.4f}, trained cache {cached:.4f}; mean bias trained {bias:+.4f}, "
          f"untrained {cold_bias:+.4f}; per frame {st.queries / spp:.0f} queries, {st.records / spp:.0f} records; "
          f"loss {warm.last_loss:.4f} after {warm.steps} steps")
    assert np.all(np.isfinite(img)) and ri.status().flags == 0
    assert warm.steps == 256 and st.steps == spp and st.queries > W * H
    assert np.isfinite(st.drop_bias) and np.isfinite(st.drop_bias_other) and abs(st.drop_bias_other) < 0.5
    assert 0.5 <= st.radiance_scale <= 2.0 and st.radiance_scale != 1.0
    assert cached < 0.9 * plain
    assert cached < cold
    assert abs(bias) < 0.05
    ri.cleanup()
    cache.close()
    untrained.close()
