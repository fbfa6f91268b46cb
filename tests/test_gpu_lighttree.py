"""The light tree built on the device (rb_k_build_light_tree,
rb_build_lights) through the C ABI.

It is not a byte copy of the host builder's tree (the reference's
LightTree::Builder, src/core/light_tree.cpp:47-418, which
rb_build_light_tree restates), so it is judged by what any valid tree must
satisfy in the reference's layouts: the structure (every light in exactly one
leaf of at most 8, depth-first node order, path masks, flux sums), the pdfs
of all lights summing to one at any shading point when the reference's own
sampling code (run by the oracle) walks it, the product's light sampling on
it matching the oracle's at 1e-5, and images rendered with it matching images
rendered with the host-built tree up to sampling noise. It must also be
faster than the host build at the at-scale workload's 4,096 emitters.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np
import pytest

import cases
from gpu_util import run_light
from oracle_lib import RefLib, light_tree_record, load_scene_into_ref, reference_luts
from ratbite_b200 import abi, lighttree, scenes
from ratbite_b200.rendering_interface import RenderingInterface

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    return RefLib()


@pytest.fixture(scope="module")
def tables(ref):
    return dict(cie=ref.cie_xyz(), basis=ref.basis_rgb(), luts=reference_luts())


def _check_structure(n, flux, tris, nodes, ptrs, masks):
    assert 1 <= len(nodes) <= 2 * n - 1
    seen = np.zeros(n, np.int64)
    flux_of = {}

    def walk(i, depth, mask):
        core = int(nodes["core"][i])
        if core >> 31:
            cnt, off = (core >> 27) & 0xF, core & ((1 << 27) - 1)
            assert 1 <= cnt <= 8 and off + cnt <= n
            s = 0.0
            for k in range(off, off + cnt):
                assert int(ptrs[k]) >> 30 == abi.LIGHT_TRIANGLE
                li = int(ptrs[k]) & ((1 << 30) - 1)
                seen[li] += 1
                assert int(masks[li]) == mask, (li, hex(int(masks[li])), hex(mask))
                s += float(flux[li])
            flux_of[i] = s
            return i + 1
        right = core
        assert i + 1 < right < len(nodes)
        end_left = walk(i + 1, depth + 1, mask)
        assert end_left == right                          # depth-first: the right subtree follows the left one
        end = walk(right, depth + 1, mask | (1 << depth))
        flux_of[i] = flux_of[i + 1] + flux_of[right]
        return end

    assert walk(0, 0, 0) == len(nodes)
    assert (seen == 1).all()                              # every light in exactly one leaf
    got = nodes["flux"].astype(np.float64)
    want = np.array([flux_of[i] for i in range(len(nodes))])
    assert np.allclose(got, want, rtol=1e-5)


@pytest.mark.parametrize("which", ["many_lights", "scale", "tiny", "nine", "coincident"])
def test_device_tree_structure(which):
    if which == "many_lights":
        world, flux, mat, prim = cases.many_lights_scene().emissive_arrays()
    elif which == "scale":
        world, flux, mat, prim = scenes.scale_scene(seed=3, width=64, height=36, spp=4).emissive_arrays()
    else:
        rng = np.random.default_rng(11)
        n = {"tiny": 1, "nine": 9, "coincident": 100}[which]
        base = rng.uniform(-1, 1, (n, 9)).astype(np.float32)
        if which == "coincident":
            base[:] = base[0]                              # 100 copies of one triangle: no plane separates them
        world, flux = base, rng.uniform(0.5, 2.0, n).astype(np.float32)
        mat, prim = np.zeros(n, np.uint32), np.arange(n, dtype=np.uint32)
    uvs = np.random.default_rng(4).uniform(-2, 3, (len(flux), 6)).astype(np.float32)
    tris, nodes, ptrs, masks = lighttree.build_on_device(world, flux, mat, prim, camera=(0.25, -0.5, 1.0), uvs=uvs)
    n = len(flux)
    _check_structure(n, flux, tris, nodes, ptrs, masks)
    assert np.array_equal(tris["uvs"].reshape(n, 6), uvs)        # emission-texture coordinates, in input order
    # triangles are the inputs, camera-relative, with their material and primitive
    v = tris["vertices"].reshape(n, 3, 3).astype(np.float64)
    assert np.allclose(v + np.array([0.25, -0.5, 1.0]), np.asarray(world, np.float64).reshape(n, 3, 3), atol=1e-5)
    assert np.array_equal(tris["material"], mat) and np.array_equal(tris["prim"], prim)
    # deterministic: a second build gives the same bytes
    again = lighttree.build_on_device(world, flux, mat, prim, camera=(0.25, -0.5, 1.0), uvs=uvs)
    for a, b in zip((tris, nodes, ptrs, masks), again):
        assert a.tobytes() == b.tobytes()


def _device_tree_into_ref(ref, sc, tables):
    keep = load_scene_into_ref(ref, sc, tables["luts"], tables["cie"], tables["basis"])
    world, flux, mat, prim = sc.emissive_arrays()
    tris, nodes, ptrs, masks = lighttree.build_on_device(world, flux, mat, prim)
    lt = light_tree_record(tris, nodes, ptrs, masks, keep)
    assert ref.lib.rbref_set_lights(C.byref(lt)) == 0
    return keep, lt, len(flux)


def test_device_tree_pdfs_normalise(ref, tables):
    """The reference's own traversal (traverseLightTree) of the device-built
    tree: the pdfs of all lights sum to one at any shading point, and the
    sampling pdf equals the pdf replayed from the light's mask."""
    sc = cases.many_lights_scene()
    keep, lt, n = _device_tree_into_ref(ref, sc, tables)
    rng = np.random.default_rng(3)
    for trial in range(8):
        p = np.array([rng.uniform(-0.9, 0.9), rng.uniform(-0.9, 0.5), rng.uniform(-4.0, -2.4)], np.float32)
        nrm = cases.unit_vectors(rng, 1)[0]
        cs = (abi.rb_light_case * n)()
        for i in range(n):
            cs[i].position = abi.F3(*p); cs[i].normal = abi.F3(*nrm)
            cs[i].rand = float((i + 0.5) / n)
            cs[i].q_type = abi.LIGHT_TRIANGLE; cs[i].q_index = i
        ref.lib.rbref_light_tree(n, C.cast(cs, C.c_void_p))
        q = np.array([c.q_pdf for c in cs], np.float64)
        assert abs(q.sum() - 1.0) < 1e-4, q.sum()
        for c in cs:
            if c.type == abi.LIGHT_TRIANGLE:
                assert abs(c.pdf - q[c.index]) <= 1e-5 * max(q[c.index], 1e-12) + 1e-9


def test_device_tree_sampling_matches_oracle(ref, tables):
    """sampleLightTree on the device-built tree, product against the oracle
    on the same records: identical picks, pdfs within 1e-5 relative."""
    sc = cases.many_lights_scene()
    keep, lt, n = _device_tree_into_ref(ref, sc, tables)
    cs = cases.light_cases()
    want = (abi.rb_light_case * len(cs)).from_buffer_copy(bytes(cs))
    ref.lib.rbref_light_tree(len(cs), C.cast(want, C.c_void_p))
    with RenderingInterface(device=0) as ri:
        ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lt)
        got = run_light(ri, cs)
    same = np.array([(a.type, a.index) == (b.type, b.index) for a, b in zip(got, want)])
    gp = np.array([c.pdf for c in got]); wp = np.array([c.pdf for c in want])
    rel = np.abs(gp - wp) / np.maximum(np.abs(wp), 1e-30)
    print(f"device tree: picks identical {same.mean():.4%}, pdf within 1e-5 {np.mean(rel[same] <= 1e-5):.4%}, "
          f"max rel {rel[same].max():.2e}")
    assert same.mean() >= 0.995
    assert np.mean(rel[same] <= 1e-5) >= 0.995
    assert rel[same].max() < 2e-4


def _render(tables, sc, W, H, spp, device_tree):
    with RenderingInterface(device=0) as ri:
        if device_tree:
            ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=None)
            ri.build_lights(*sc.emissive_arrays())
        else:
            ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lighttree.build_for_scene(sc))
        ri.render(0, spp)
        acc = ri.read_accumulation()
        assert ri.status().flags == 0
    return acc


def test_device_tree_renders_like_the_host_tree(tables):
    """Both trees give unbiased light sampling, so the images agree up to
    noise: the image means within 1 %, and per pixel no further apart than
    sampling noise allows (the difference of the two images has a mean near
    zero against its own spread)."""
    sc = scenes.scale_scene(seed=5, target_tris=60_000, n_emitters=126, width=64, height=36, spp=64, max_depth=6,
                            envmap_size=(64, 32))
    W, H, spp = 64, 36, 256
    a = _render(tables, sc, W, H, spp, False)
    b = _render(tables, sc, W, H, spp, True)
    ma, mb = a[..., :3] / a[..., 3:4], b[..., :3] / b[..., 3:4]
    rel = abs(mb.sum() - ma.sum()) / ma.sum()
    d = (mb - ma)[..., 1].ravel()
    z = d.mean() / (d.std() / np.sqrt(d.size))
    print(f"device vs host tree: image mean rel diff {rel:.3e}, per-pixel difference z {z:.2f}")
    assert rel < 1e-2
    assert abs(z) < 5.0


def test_device_build_beats_the_host_build():
    """4,096 emitters (the at-scale workload): device build time (CUDA
    events) against the host builder (wall time, the reference's algorithm
    restated)."""
    world, flux, mat, prim = scenes.scale_scene(seed=3, width=64, height=36, spp=4).emissive_arrays()
    assert len(flux) == 4096
    times = []
    for _ in range(5):
        lighttree.build_on_device(world, flux, mat, prim, timing=times)
    t0 = time.perf_counter()
    for _ in range(5):
        lighttree.build(world, flux, mat, prim)
    host_ms = (time.perf_counter() - t0) / 5 * 1e3
    dev_ms = float(np.median(times[1:]))
    print(f"light tree, 4096 emitters: device {dev_ms:.3f} ms, host {host_ms:.3f} ms")
    assert dev_ms < host_ms
