"""Material textures (rb_set_textures; the reference's tex2D reads of
base colour, alpha, normal, metal-roughness, transmission, sheen colour and
roughness, and emission: src/kernels/pathtrace.cu:1217-1228, 1437-1560,
1640-1650) against the oracle, which runs the reference's own shading code
with its texture objects backed by the same texels.

The scene exercises sRGB decoding, nearest and bilinear filtering, wrap /
mirror / clamp addressing with coordinates beyond [0, 1], an alpha cutout,
texture coordinate set 2, a one-channel texture and a textured emitter hit
by camera rays and picked by light sampling."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gpu_util import assert_image_parity
from oracle_lib import RefLib, light_tree_record, load_scene_into_ref, ref_render, reference_luts
from ratbite_b200 import abi, lighttree, scenes
from ratbite_b200._native import NativeError
from ratbite_b200.rendering_interface import RenderingInterface, render_jobs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    return RefLib()


@pytest.fixture(scope="module")
def tables(ref):
    return dict(cie=ref.cie_xyz(), basis=ref.basis_rgb(), luts=reference_luts())


def test_textured_render_matches_oracle(ref, tables):
    sc = scenes.textured_cornell(seed=3, cie_xyz=tables["cie"], width=64, height=64, spp=16, max_depth=8)
    W, H, spp = 64, 64, 16
    keep = load_scene_into_ref(ref, sc, tables["luts"], tables["cie"], tables["basis"])
    want = ref_render(ref, W, H, 0, spp)
    lt = lighttree.build_for_scene(sc)
    with RenderingInterface(device=0) as ri:
        ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lt)
        ri.render(0, spp)
        got = ri.read_accumulation()
        assert ri.status().flags == 0
    assert (got[..., 3] == spp).all()
    assert_image_parity(f"textured cornell {W}x{H}x{spp}", got, want)
    # the textures are seen: the same scene without them renders a different image
    plain = scenes.textured_cornell(seed=3, cie_xyz=tables["cie"], width=64, height=64, spp=16, max_depth=8)
    for m in plain.materials:
        m.textures = {}
    with RenderingInterface(device=0) as ri:
        ri.load_scene(plain, tables["luts"], tables["cie"], tables["basis"], light_tree=lighttree.build_for_scene(plain))
        ri.render(0, spp)
        other = ri.read_accumulation()
    assert np.mean(np.abs(other[..., :3] - got[..., :3])) > 1e-2 * np.mean(np.abs(got[..., :3]))


def test_textured_render_other_sample_range(ref, tables):
    """Another Sobol range and a second seed's textures (other colours)."""
    sc = scenes.textured_cornell(seed=8, cie_xyz=tables["cie"], width=48, height=40, spp=8, max_depth=6)
    keep = load_scene_into_ref(ref, sc, tables["luts"], tables["cie"], tables["basis"])
    launch = sc.launch_record()
    assert ref.lib.rbref_set_launch(C.byref(launch)) == 0
    want = ref_render(ref, 48, 40, 1000, 8)
    with RenderingInterface(device=0) as ri:
        ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lighttree.build_for_scene(sc))
        ri.clear_accumulation()
        ri.render(1000, 8)
        got = ri.read_accumulation()
        assert ri.status().flags == 0
    assert_image_parity("textured cornell 48x40, samples [1000, 1008)", got, want)


def test_texture_tables_are_checked(tables):
    sc = scenes.textured_cornell(seed=3, width=16, height=16, spp=1)
    with RenderingInterface(device=0) as ri:
        # a material that names a texture beyond the table
        ri.load_textures((abi.rb_texture * 0)())
        with pytest.raises(NativeError):
            ri.fill_model_materials(sc.material_records())
        # malformed textures
        bad = (abi.rb_texture * 1)()
        img = np.zeros((4, 4, 4), np.uint8)
        bad[0].width, bad[0].height, bad[0].format, bad[0].data = 4, 4, 7, img.ctypes.data
        with pytest.raises(NativeError):
            ri.load_textures(bad)
        bad[0].format, bad[0].address_u = abi.RB_TEXFMT_RGBA8, 9
        with pytest.raises(NativeError):
            ri.load_textures(bad)
        bad[0].address_u, bad[0].filter = 0, 4
        with pytest.raises(NativeError):
            ri.load_textures(bad)
        # a valid table, then materials that use it, then a smaller table: the render refuses
        ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lighttree.build_for_scene(sc))
        ri.load_textures((abi.rb_texture * 0)())
        with pytest.raises(NativeError):
            ri.render(0, 1)


def test_device_tree_samples_the_emission_texture(tables):
    """The light tree built on the device carries the emitters' texture
    coordinates (rb_build_lights' uvs): its image matches the host-built
    tree's (bit for bit when both builders make the same tree, as for this
    scene's two emitters; else up to sampling noise), and a tree built
    without them, which reads the emission texture at (0, 0) in light
    sampling, renders a different image."""
    sc = scenes.textured_cornell(seed=3, cie_xyz=tables["cie"], width=48, height=48, spp=64, max_depth=4)
    out = []
    for mode in ("host", "device", "device without uvs"):
        with RenderingInterface(device=0) as ri:
            if mode == "host":
                ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lighttree.build_for_scene(sc))
            else:
                ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=None)
                ri.build_lights(*sc.emissive_arrays(), uvs=sc.emissive_uvs() if mode == "device" else None)
            ri.render(0, 256)
            out.append(ri.read_accumulation())
            assert ri.status().flags == 0
    a, b, c = (o[..., :3] / o[..., 3:4] for o in out)
    d = (b - a)[..., 1].ravel()
    rel = abs(b.sum() - a.sum()) / a.sum()
    z = 0.0 if d.std() == 0 else d.mean() / (d.std() / np.sqrt(d.size))
    print(f"textured emitters, device vs host tree: image mean rel diff {rel:.3e}, per-pixel difference z {z:.2f}; "
          f"without uvs: image mean rel diff {abs(c.sum() - a.sum()) / a.sum():.3e}")
    assert rel < 1e-2 and abs(z) < 5.0
    assert np.abs(c - a).sum() > 1e-3 * np.abs(a).sum()


def test_textured_jobs_in_a_shared_wavefront(tables):
    """The textured kernels of the shared wavefront (rb_render_jobs): a
    textured job and an untextured one in one wave, each bit-identical to
    its own render."""
    scs = [scenes.textured_cornell(seed=3, cie_xyz=tables["cie"], width=40, height=32, spp=6, max_depth=6),
           scenes.cornell_box(seed=2, cie_xyz=tables["cie"], width=24, height=20, spp=6, max_depth=6)]
    alone = []
    for sc in scs:
        with RenderingInterface(device=0) as ri:
            ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lighttree.build_for_scene(sc))
            ri.render(0, 6)
            alone.append(ri.read_accumulation())
    ris = []
    for sc in scs:
        ri = RenderingInterface(device=0)
        ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lighttree.build_for_scene(sc))
        ris.append(ri)
    render_jobs(ris, [0, 0], [6, 6])
    for ri, want in zip(ris, alone):
        assert ri.status().flags == 0
        assert np.array_equal(ri.read_accumulation(), want)
        ri.cleanup()


def test_textured_scene_in_the_cached_form(tables):
    """The cached form on a textured scene: with paths that never stop at
    the cache it renders the plain image bit for bit (the textured shading
    kernels under the cache's record and query bookkeeping), and with
    training on it keeps a finite loss and clean status."""
    from ratbite_b200.nrc import RadianceCache
    sc = scenes.textured_cornell(seed=3, cie_xyz=tables["cie"], width=48, height=40, spp=8, max_depth=8)
    with RenderingInterface(device=0) as ri:
        ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lighttree.build_for_scene(sc))
        ri.render(0, 8)
        want = ri.read_accumulation()
        cache = RadianceCache(seed=1)
        ri.attach_radiance_cache(cache, spread_threshold=1e30, frozen=True, samples_per_wave=8)
        ri.render(0, 8)
        assert np.array_equal(ri.read_accumulation(), want)
        ri.attach_radiance_cache(cache, samples_per_wave=8)
        ri.render(0, 16)
        st = ri.cache_stats()
        assert ri.status().flags == 0 and np.isfinite(st.last_loss) and st.queries > 0
        ri.attach_radiance_cache(None)
        cache.close()


def test_failed_samples_kept_or_dropped(tables):
    """rb_config.failed_sample_mode on a scene whose normal map makes BxDF
    samples fail: RB_FAILED_DROP (the reference's behaviour, the image the
    parity tests compare) drops a failed sample's radiance, RB_FAILED_KEEP
    keeps what the path gathered before the failure. Same sample sequence,
    so per pixel the kept image is at least the dropped one, and larger
    somewhere."""
    sc = scenes.textured_cornell(seed=3, cie_xyz=tables["cie"], width=48, height=48, spp=16, max_depth=8)
    out = []
    for mode in (abi.RB_FAILED_DROP, abi.RB_FAILED_KEEP):
        with RenderingInterface(device=0, failed_sample_mode=mode) as ri:
            ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lighttree.build_for_scene(sc))
            ri.render(0, 16)
            out.append(ri.read_accumulation())
            assert ri.status().flags == 0
    drop, keep = out
    assert np.array_equal(drop[..., 3], keep[..., 3])
    d = keep[..., :3] - drop[..., :3]
    print(f"failed samples: kept image {d.sum() / drop[..., :3].sum():.3%} brighter, pixels changed {np.mean(np.any(d != 0, -1)):.1%}")
    assert d.min() >= -1e-9 * np.abs(drop[..., :3]).max()
    assert d.sum() > 0.0


def test_software_sampler_matches_the_texture_unit(tables):
    """The shading kernels' software sampler against the texture unit the
    reference samples with (a CUDA texture object from the same texels and
    sampler settings, rb_k_texture_sample): nearest filtering returns the
    same texel except where a coordinate rounds across a texel edge,
    bilinear filtering differs only by the unit's 8-bit fixed-point weights
    (at most a few 1e-3), and the unit's sRGB decode is an approximation of
    the curve within a few 1e-3 (measured on B200: bilinear RGBA8 max
    5.4e-3, mean 1.2e-3; sRGB nearest max 3.8e-3, mean 1.1e-3); for every
    address mode, RGBA8 and R8 (whose sRGB flag the unit applies to its one
    channel)."""
    import torch
    from ratbite_b200._native import check, load
    rng = np.random.default_rng(12)
    texs = [
        scenes.Texture(rng.integers(0, 256, (13, 17, 4)).astype(np.uint8), srgb=False,
                       address=(abi.RB_TEXADDR_WRAP, abi.RB_TEXADDR_WRAP), filter=abi.RB_TEXFILTER_LINEAR),
        scenes.Texture(rng.integers(0, 256, (9, 11, 4)).astype(np.uint8), srgb=True,
                       address=(abi.RB_TEXADDR_MIRROR, abi.RB_TEXADDR_CLAMP), filter=abi.RB_TEXFILTER_NEAREST),
        scenes.Texture(rng.integers(0, 256, (8, 6, 4)).astype(np.uint8), srgb=True,
                       address=(abi.RB_TEXADDR_MIRROR, abi.RB_TEXADDR_WRAP), filter=abi.RB_TEXFILTER_LINEAR),
        scenes.Texture(rng.integers(0, 256, (7, 10)).astype(np.uint8), srgb=False,
                       address=(abi.RB_TEXADDR_CLAMP, abi.RB_TEXADDR_MIRROR), filter=abi.RB_TEXFILTER_LINEAR),
        scenes.Texture(rng.integers(0, 256, (12, 5)).astype(np.uint8), srgb=True,
                       address=(abi.RB_TEXADDR_WRAP, abi.RB_TEXADDR_CLAMP), filter=abi.RB_TEXFILTER_NEAREST),
        scenes.Texture(rng.integers(0, 256, (6, 6)).astype(np.uint8), srgb=True,
                       address=(abi.RB_TEXADDR_WRAP, abi.RB_TEXADDR_WRAP), filter=abi.RB_TEXFILTER_LINEAR),
    ]
    sc = scenes.cornell_box(seed=1, cie_xyz=tables["cie"], width=8, height=8, spp=1, max_depth=2)
    sc.textures = texs
    n = 20000
    uv = rng.uniform(-2.3, 3.1, (n, 2)).astype(np.float32)
    with RenderingInterface(device=0) as ri:
        ri.load_scene(sc, tables["luts"], tables["cie"], tables["basis"], light_tree=lighttree.build_for_scene(sc))
        d_uv = torch.from_numpy(uv).cuda()
        for k, t in enumerate(texs):
            soft = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
            hw = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
            check(load().rb_k_texture_sample(ri.ctx, k, n, C.c_void_p(d_uv.data_ptr()), C.c_void_p(soft.data_ptr()),
                                             C.c_void_p(hw.data_ptr()), None), ri.ctx, "texture sample")
            s_, h_ = soft.cpu().numpy(), hw.cpu().numpy()
            d = np.abs(s_ - h_).max(axis=1)
            kind = ("R8" if t.data.ndim == 2 else "RGBA8") + (" sRGB" if t.srgb else "") + \
                (" nearest" if t.filter == abi.RB_TEXFILTER_NEAREST else " bilinear")
            print(f"texture {k} ({kind}): max |soft - hw| {d.max():.2e}, mean {d.mean():.2e}, exact {np.mean(d == 0):.2%}; "
                  f"per channel mean {np.round(np.abs(s_ - h_).mean(axis=0), 4)}; hw[0] {np.round(h_[0], 4)} soft[0] {np.round(s_[0], 4)}")
            if t.filter == abi.RB_TEXFILTER_NEAREST and not t.srgb:
                assert np.mean(d < 1e-6) >= 0.99, k
            elif t.filter == abi.RB_TEXFILTER_NEAREST:
                # the unit's sRGB decode approximates the curve (the sampler
                # here evaluates it exactly, in double precision)
                assert np.mean(d < 5e-3) >= 0.99 and d.mean() < 2e-3, k
            else:
                assert d.max() < 1.5e-2 and d.mean() < 3e-3, k
