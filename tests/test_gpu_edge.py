"""Edge cases of the rendering path on the GPU, through the C ABI: scenes
without geometry, lights or environment; a one-pixel film; depth 1;
degenerate triangles; and the host-side rejections that keep invalid input
away from the kernels (every rejected call returns a status and leaves the
context usable). Renders that have an oracle counterpart are compared with
it like the other render tests."""
from __future__ import annotations

import copy
import ctypes as C

import numpy as np
import pytest

from oracle_lib import RefLib, light_tree_record, load_scene_into_ref, ref_render, reference_luts
from ratbite_b200 import abi, lighttree, scenes
from ratbite_b200._native import load
from ratbite_b200.rendering_interface import RenderingInterface

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tables():
    ref = RefLib()
    return dict(ref=ref, cie=ref.cie_xyz(), basis=ref.basis_rgb(), luts=reference_luts())


def _compare(tables, sc, W, H, spp, depth=None):
    ref = tables["ref"]
    keep = load_scene_into_ref(ref, sc, tables["luts"], tables["cie"], tables["basis"], width=W, height=H,
                               max_depth=depth)
    world, flux, mat, prim = sc.emissive_arrays()
    lt = None
    if len(flux):
        tris, nodes, ptrs, masks = ref.build_light_tree(world, flux, mat, prim)
        lt = light_tree_record(tris, nodes, ptrs, masks, keep)
    want = ref_render(ref, W, H, 0, spp)
    with RenderingInterface(device=0) as ri:
        ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lt, width=W, height=H,
                      max_depth=depth)
        ri.render(0, spp)
        got = ri.read_accumulation()
        st = ri.status()
    assert st.flags == 0
    assert np.array_equal(got[..., 3], want[..., 3])
    g = got[..., :3] / np.maximum(got[..., 3:4], 1)
    w = want[..., :3] / np.maximum(want[..., 3:4], 1)
    denom = max(np.abs(w).sum(), 1e-30)
    return g, w, np.abs(g - w).sum() / denom


def _no_geometry_scene(with_env=True):
    sc = scenes.cornell_box(seed=1, width=16, height=16, spp=2)
    sc.meshes, sc.instances, sc.emissive, sc.materials = [], [], [], [scenes.Material()]
    if with_env:
        sc.envmap = scenes.sky_envmap(64, 32, seed=2)
    return sc


def test_environment_only_scene(tables):
    g, w, l1 = _compare(tables, _no_geometry_scene(), 16, 16, 2)
    assert w.sum() > 0 and l1 < 1e-5


def test_dark_scene_without_lights(tables):
    sc = scenes.cornell_box(seed=1, width=16, height=16, spp=2)
    # drop the emitter: no light tree, no environment, nothing emits
    sc.emissive = []
    for m in sc.materials:
        m.emissive = None
    with RenderingInterface(device=0) as ri:
        ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"])
        ri.render(0, 3)
        got = ri.read_accumulation()
        assert ri.status().flags == 0
    assert np.all(got[..., :3] == 0.0) and np.all(got[..., 3] == 3.0)


def test_one_pixel_film_and_depth_one(tables):
    sc = scenes.cornell_box(seed=1, width=1, height=1, spp=16)
    g, w, l1 = _compare(tables, sc, 1, 1, 16)
    assert l1 < 1e-4
    sc = scenes.cornell_box(seed=1, width=24, height=24, spp=4, max_depth=1)
    g, w, l1 = _compare(tables, sc, 24, 24, 4, depth=1)
    assert l1 < 1e-4


@pytest.mark.parametrize("W,H", [(13, 9), (7, 3), (17, 2), (9, 5)])
def test_films_that_are_not_whole_tiles(tables, W, H):
    # path slots run over 8 x 4 pixel tiles; at sizes that are not multiples
    # of the tile every pixel still gets its own samples (the oracle's per
    # pixel counts and values)
    sc = scenes.cornell_box(seed=1, width=W, height=H, spp=4)
    g, w, l1 = _compare(tables, sc, W, H, 4)
    assert l1 < 5e-2                # the Cornell parity bound (rare light-tree pick flips)


def test_degenerate_triangles_are_skipped(tables):
    sc = scenes.cornell_box(seed=1, width=24, height=24, spp=4)
    sc = copy.copy(sc)
    sm = sc.meshes[0][0]
    v = np.concatenate([sm.vertices, sm.vertices[:1], sm.vertices[:1]]).astype(np.float32)
    n = len(sm.vertices)
    idx = np.concatenate([sm.indices, np.array([[0, n, n + 1], [1, 1, 2]], sm.indices.dtype)])
    sc.meshes = [list(m) for m in sc.meshes]
    sc.meshes[0][0] = scenes.Submesh(v, idx, sm.material, sm.normals, list(sm.discarded))
    sc._keep = []
    g, w, l1 = _compare(tables, sc, 24, 24, 4)
    assert l1 < 1e-4


# ------------------------------------------------------ host-side rejections
def _context(tables):
    sc = scenes.cornell_box(seed=1, width=16, height=16, spp=1)
    ri = RenderingInterface(device=0)
    ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lighttree.build_for_scene(sc))
    return sc, ri


def test_rejections_leave_the_context_usable(tables):
    lib = load()
    sc, ri = _context(tables)
    ctx = ri.ctx
    # render before anything is set
    empty = C.c_void_p()
    assert lib.rb_create(None, C.byref(empty)) == 0
    assert lib.rb_render(empty, 0, 1, None) == abi.RB_ERR_NO_SCENE
    assert lib.rb_resolve(empty, np.zeros(9, np.float32).ctypes.data, 1.0, None) == abi.RB_ERR_NO_SCENE
    lib.rb_destroy(empty)
    # launch parameters: empty film, depth above 64
    bad = sc.launch_record()
    bad.width = 0
    assert lib.rb_set_launch(ctx, C.byref(bad)) == abi.RB_ERR_INVALID
    bad = sc.launch_record()
    bad.max_path_depth = 65
    assert lib.rb_set_launch(ctx, C.byref(bad)) == abi.RB_ERR_INVALID
    # material table smaller than the geometry's references: rb_render refuses
    mats = sc.material_records()
    assert lib.rb_set_materials(ctx, C.cast(mats, C.c_void_p), 2) == 0
    assert lib.rb_render(ctx, 0, 1, None) == abi.RB_ERR_INVALID
    assert lib.rb_set_materials(ctx, C.cast(mats, C.c_void_p), len(mats)) == 0
    # a texture index beyond the (empty) texture table, an unknown texture slot, unknown BxDF
    m1 = (abi.rb_material * 1).from_buffer_copy(bytes(mats)[:C.sizeof(abi.rb_material)])
    m1[0].textures = 1
    assert lib.rb_set_materials(ctx, C.cast(m1, C.c_void_p), 1) == abi.RB_ERR_INVALID
    m1[0].textures = 1 << abi.RB_TEXTURE_SLOTS
    assert lib.rb_set_materials(ctx, C.cast(m1, C.c_void_p), 1) == abi.RB_ERR_INVALID
    m1[0].textures = 0
    m1[0].bxdf = 7
    assert lib.rb_set_materials(ctx, C.cast(m1, C.c_void_p), 1) == abi.RB_ERR_INVALID
    # vertex attributes off the 8-byte grid, or outside the vertex
    m1[0].bxdf = mats[0].bxdf
    attr = np.zeros(64, np.float32)
    m1[0].attribute_data, m1[0].vertex_count = attr.ctypes.data, 4
    for bits, stride, offs in ((abi.RB_ATTR_FRAME, 20, (0, 0, 0)), (abi.RB_ATTR_NORMAL, 16, (12, 0, 0)),
                               (abi.RB_ATTR_FRAME, 16, (8, 0, 0)), (abi.RB_ATTR_TEX_COORD_1, 8, (0, 4, 0))):
        m1[0].attributes, m1[0].attribute_stride = bits, stride
        m1[0].frame_offset = m1[0].normal_offset = offs[0]
        m1[0].texcoord1_offset = offs[1]
        assert lib.rb_set_materials(ctx, C.cast(m1, C.c_void_p), 1) == abi.RB_ERR_INVALID, (bits, stride, offs)
    # light tree whose child index points outside the node array
    world, flux, mat, prim = sc.emissive_arrays()
    tris, nodes, ptrs, masks = lighttree.build(world, flux, mat, prim)
    keep = []
    nodes = nodes.copy()
    if len(nodes) > 1:
        nodes["core"][0] = len(nodes) + 5
    else:
        nodes["core"][0] = (1 << 31) | (15 << 27)
    lt = light_tree_record(tris, nodes, ptrs, masks, keep)
    assert lib.rb_set_lights(ctx, C.byref(lt)) == abi.RB_ERR_INVALID
    # non-finite vertex
    g = copy.copy(sc)
    sm = g.meshes[0][0]
    v = sm.vertices.copy()
    v[0, 0] = np.inf
    g.meshes = [list(m) for m in g.meshes]
    g.meshes[0][0] = scenes.Submesh(v, sm.indices, sm.material, sm.normals, list(sm.discarded))
    g._keep = []
    assert lib.rb_set_geometry(ctx, C.byref(g.geometry_record())) == abi.RB_ERR_INVALID
    # environment map sizes
    img = np.ones((6, 6, 4), np.float32)
    assert lib.rb_set_envmap(ctx, img.ctypes.data, 6, 6) == abi.RB_ERR_INVALID
    # the context still renders the original scene
    ri.render(0, 2)
    acc = ri.read_accumulation()
    assert np.all(acc[..., 3] == 2.0) and acc[..., :3].sum() > 0
    assert ri.status().flags == 0
    ri.cleanup()


# ------------------------------------------------ failure detection (host-side injection)
def _cornell(tables, W=24, H=24, spp=4):
    sc = scenes.cornell_box(seed=1, cie_xyz=tables["cie"], width=W, height=H, spp=spp)
    return sc, lighttree.build_for_scene(sc)


def _render(tables, sc, lt, spp, **kw):
    with RenderingInterface(device=0, **kw) as ri:
        ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lt)
        ri.render(0, spp)
        return ri.read_accumulation(), ri.status().flags


def test_small_wavefront_capacity_renders_identically(tables):
    """A wavefront of 1,000 paths (the frame's 18,432 paths then take 19
    waves) gives the accumulation of the default capacity, bit for bit."""
    sc, lt = _cornell(tables, 48, 48, 8)
    want, f0 = _render(tables, sc, lt, 8)
    got, f1 = _render(tables, sc, lt, 8, max_paths_in_flight=1000)
    assert f0 == 0 and f1 == 0
    assert np.array_equal(got, want)


def test_injected_queue_limit_sets_the_overflow_flag(tables):
    """Queues that accept only 64 entries per bounce: appends beyond drop
    their entry and raise RB_DEV_QUEUE_OVERFLOW; nothing is written out of
    bounds, every pixel still counts its samples, and the context renders
    again."""
    sc, lt = _cornell(tables)
    with RenderingInterface(device=0, inject={"queue_limit": 64}) as ri:
        ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lt)
        ri.render(0, 4)
        acc = ri.read_accumulation()
        flags = ri.status().flags
        assert flags & abi.RB_DEV_QUEUE_OVERFLOW
        assert np.isfinite(acc).all() and (acc[..., 3] == 4).all()
        ri.render(0, 1)
        assert np.isfinite(ri.read_accumulation()).all()


def test_injected_stack_limit_sets_the_overflow_flag(tables):
    """A traversal stack of one entry cannot hold the children a ray owes at
    an 8-wide node: RB_DEV_STACK_OVERFLOW is raised, the render completes."""
    sc, lt = _cornell(tables)
    acc, flags = _render(tables, sc, lt, 4, inject={"stack_limit": 1})
    assert flags & abi.RB_DEV_STACK_OVERFLOW
    assert np.isfinite(acc).all()


def test_non_finite_radiance_sets_its_flag(tables):
    """An emitter of 3e38 (finite, but its samples overflow to infinity in
    the radiance estimate) raises RB_DEV_NAN_RADIANCE."""
    sc, lt = _cornell(tables)
    for m in sc.materials:
        if m.emissive:
            m.emissive = (3e38, 3e38, 3e38)
    _, flags = _render(tables, sc, lt, 2)
    assert flags & abi.RB_DEV_NAN_RADIANCE


def test_injected_allocation_failure_leaves_the_context_usable(tables):
    """The n-th device allocation of a context fails once, for every n up to
    the allocations of a whole load-and-render: the failing call returns an
    error (out of memory) with a message and changes nothing, and repeating
    the load and the render then gives the clean accumulation bit for bit."""
    from ratbite_b200._native import NativeError
    sc, lt = _cornell(tables)
    want, _ = _render(tables, sc, lt, 4)
    failures = 0
    for n in range(1, 80):
        try:
            ri = RenderingInterface(device=0, inject={"alloc_failure": n})
        except NativeError as e:
            assert e.code == abi.RB_ERR_OOM
            failures += 1
            continue
        with ri:
            try:
                ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lt)
                ri.render(0, 4)
                failed = False
            except NativeError as e:
                assert e.code in (abi.RB_ERR_OOM, abi.RB_ERR_CUDA)
                assert str(e).strip()
                failed = True
                failures += 1
                ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lt)
                ri.render(0, 4)
            got = ri.read_accumulation()
            assert np.array_equal(got, want), n
            assert ri.status().flags == 0
        if not failed and n > 2:
            break                       # n is past the last allocation
    assert failures >= 10
