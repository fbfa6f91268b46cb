"""CPU checks (no GPU): the C ABI library builds and exports every declared
symbol, the ctypes records match the C layouts, the oracle's C restatements
agree with the reference compiled host-side, and the oracle itself behaves
(light-tree pdfs normalise, progressive sample ranges compose)."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import cases
from oracle_lib import REF_DIR, RefLib, load_scene_into_ref, light_tree_record, ref_render, reference_luts, _np_ptr
from ratbite_b200 import abi, scenes
from ratbite_b200 import _native

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        for m in re.finditer(r"^\s*(?:int|size_t|const char\*|void)\s+(rb_\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    assert _native.LIB_PATH.exists(), "build the library first (__graft_entry__.build())"
    out = subprocess.run(["nm", "-D", "--defined-only", str(_native.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    declared = declared_symbols()
    assert len(declared) >= 30
    missing = declared - exported
    assert not missing, missing
    # and the Python loader binds exactly those
    assert declared == set(_native.SIGNATURES)


def test_library_loads_without_gpu():
    lib = _native.load()
    assert lib.rb_abi_version() == abi.RB_ABI_VERSION
    # creating a context needs a device: without one it must fail cleanly
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a device is present")
    except Exception:
        pass
    h = C.c_void_p()
    rc = lib.rb_create(None, C.byref(h))
    assert rc != 0 and not h.value


def test_abi_record_sizes(tmp_path):
    # sizes of the C records (x86-64 SysV): computed by the C compiler
    src = tmp_path / "abi_sizes.c"
    src.write_text('#include <stdio.h>\n#include "ratbite_b200_kernels.h"\nint main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n",'
                   'sizeof(rb_config),sizeof(rb_material),sizeof(rb_submesh),sizeof(rb_mesh),sizeof(rb_instance),'
                   'sizeof(rb_emissive_subset),sizeof(rb_geometry),sizeof(rb_light_tree),sizeof(rb_launch),'
                   'sizeof(rb_bxdf_case),sizeof(rb_light_case),sizeof(rb_device_status),sizeof(rb_render_stats));}\n')
    exe = src.with_suffix("")
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    sizes = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    ours = [C.sizeof(t) for t in (abi.rb_config, abi.rb_material, abi.rb_submesh, abi.rb_mesh, abi.rb_instance,
                                  abi.rb_emissive_subset, abi.rb_geometry, abi.rb_light_tree, abi.rb_launch,
                                  abi.rb_bxdf_case, abi.rb_light_case, abi.rb_device_status,
                                  abi.rb_render_stats)]
    assert sizes == ours


def test_abi_cache_record_layouts(tmp_path):
    # the radiance-cache records: sizes and the offsets of the fields added last
    src = tmp_path / "abi_nrc.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "ratbite_b200.h"\n#include "ratbite_b200_nrc.h"\n'
                   'int main(){printf("%zu %zu %zu %zu %zu %zu %zu\\n",sizeof(rb_progress),sizeof(rb_nrc_config),'
                   'sizeof(rb_cache_params),sizeof(rb_cache_stats),offsetof(rb_cache_stats,drop_bias),'
                   'offsetof(rb_cache_stats,drop_bias_other),offsetof(rb_cache_stats,radiance_scale));}\n')
    exe = src.with_suffix("")
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    sizes = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    ours = [C.sizeof(abi.rb_progress), C.sizeof(abi.rb_nrc_config), C.sizeof(abi.rb_cache_params),
            C.sizeof(abi.rb_cache_stats), abi.rb_cache_stats.drop_bias.offset, abi.rb_cache_stats.drop_bias_other.offset,
            abi.rb_cache_stats.radiance_scale.offset]
    assert sizes == ours


# --------------------------------------------------------------- oracle
@pytest.fixture(scope="module")
def ref():
    return RefLib()


@pytest.fixture(scope="module")
def restate():
    lib = C.CDLL(str(REF_DIR / "liboracle_restate.so"))
    lib.orc_sobol.argtypes = [C.c_uint32, C.c_uint32] + [C.c_void_p] * 5
    lib.orc_pixel_hash.restype = C.c_uint32
    lib.orc_pixel_hash.argtypes = [C.c_uint32, C.c_uint32]
    lib.orc_envmap_cdf.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    return lib


def test_oracle_tables(ref):
    assert ref.lib.rbref_sizeof_material_data() == 200
    assert ref.lib.rbref_sizeof_launch_parameters() == 312
    cie = ref.cie_xyz()
    # CIE Y integral over 1 nm bins (SpectralSettings::K_CIE_Y_Integral)
    assert abs(cie[1].sum() - 106.856895) < 1e-3
    luts = reference_luts()
    assert luts["conductor"].size == 1024 and luts["sheen"].size == 4096


@pytest.mark.parametrize("dims", [1, 2, 3])
def test_sobol_restatement_matches_reference(ref, restate, dims):
    s, h, b, d = cases.sobol_inputs()
    n = len(s)
    want = np.zeros(n * dims, np.float32)
    got = np.zeros(n * dims, np.float32)
    ref.lib.rbref_sobol(n, dims, _np_ptr(s), _np_ptr(h), _np_ptr(b), _np_ptr(d), _np_ptr(want))
    restate.orc_sobol(n, dims, _np_ptr(s), _np_ptr(h), _np_ptr(b), _np_ptr(d), _np_ptr(got))
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert ((got >= 0) & (got < 1)).all()


def test_sobol_golden_vectors(restate):
    """Committed golden values produced by the reference compiled host-side
    (tests/golden/make_golden.py)."""
    g = np.load(ROOT / "tests" / "golden" / "sobol.npz")
    for dims in (1, 2, 3):
        got = np.zeros(len(g["sample"]) * dims, np.float32)
        restate.orc_sobol(len(g["sample"]), dims, _np_ptr(g["sample"]), _np_ptr(g["hash"]), _np_ptr(g["bounce"]),
                          _np_ptr(g["dim"]), _np_ptr(got))
        assert np.array_equal(got.view(np.uint32), g[f"out{dims}"].view(np.uint32))


def _sky(w, h, seed=0):
    rng = np.random.default_rng(seed)
    img = np.zeros((h, w, 4), np.float32)
    th = (np.arange(h) + 0.5) / h * np.pi
    img[..., 0] = (0.2 + 0.8 * np.cos(th)[:, None] ** 2)
    img[..., 1] = img[..., 0] * 0.9
    img[..., 2] = img[..., 0] * 1.2
    img[..., :3] += rng.random((h, w, 3)).astype(np.float32) * 0.05
    img[h // 5, w // 3, :3] = 1e4          # a sun texel: 1e4 dynamic range
    img[..., 3] = 1.0
    return img


@pytest.mark.parametrize("w,h", [(64, 32), (1024, 512), (4100 // 4 * 4, 8)])
def test_envmap_cdf_restatement_properties(restate, w, h):
    img = _sky(w, h)
    for mode in (0, 1):
        cond = np.zeros(w * h, np.uint16)
        marg = np.zeros(h, np.uint16)
        integ = np.zeros(1, np.float32)
        assert restate.orc_envmap_cdf(w, h, _np_ptr(img), mode, _np_ptr(cond), _np_ptr(marg), _np_ptr(integ)) == 0
        cond = cond.reshape(h, w)
        assert (cond >= 1).all() and (cond <= w - 1).all()
        assert (np.diff(cond.astype(np.int64), axis=1) >= 0).all()      # monotone inversion
        assert (np.diff(marg.astype(np.int64)) >= 0).all()
        # integral = sum(power * sin) / (w*h)
        p = np.maximum(img[..., :3].astype(np.float64).mean(-1), 0)
        s = np.sin(np.pi * (np.arange(h) + 0.5) / h)
        want = (p.sum(1) * s).sum() / (w * h)
        assert abs(integ[0] - want) / want < (1e-4 if mode == 0 else 1e-6)


def test_envmap_cdf_rejects_bad_sizes(restate):
    img = np.zeros((6, 6, 4), np.float32)
    out = np.zeros(64, np.uint16)
    integ = np.zeros(1, np.float32)
    assert restate.orc_envmap_cdf(6, 6, _np_ptr(img), 0, _np_ptr(out), _np_ptr(out), _np_ptr(integ)) != 0


def test_light_tree_pdfs_normalise(ref):
    """Sampling pdf equals the pdf replayed from the light's bitmask, and the
    pdfs of all lights sum to one at any shading point."""
    sc = cases.many_lights_scene()
    tables = dict(cie=ref.cie_xyz(), basis=ref.basis_rgb(), luts=reference_luts())
    keep = load_scene_into_ref(ref, sc, tables["luts"], tables["cie"], tables["basis"])
    n_lights = sum(len(e["prim"]) for e in sc.emissive)
    rng = np.random.default_rng(3)
    for trial in range(8):
        p = np.array([rng.uniform(-0.9, 0.9), rng.uniform(-0.9, 0.5), rng.uniform(-4.0, -2.4)], np.float32)
        nrm = cases.unit_vectors(rng, 1)[0]
        cs = (abi.rb_light_case * n_lights)()
        for i in range(n_lights):
            cs[i].position = abi.F3(*p); cs[i].normal = abi.F3(*nrm)
            cs[i].rand = float((i + 0.5) / n_lights)
            cs[i].q_type = abi.LIGHT_TRIANGLE; cs[i].q_index = i
        ref.lib.rbref_light_tree(n_lights, C.cast(cs, C.c_void_p))
        q = np.array([c.q_pdf for c in cs], np.float64)
        assert abs(q.sum() - 1.0) < 1e-4
        for c in cs:
            if c.type == abi.LIGHT_TRIANGLE:
                assert abs(c.pdf - q[c.index]) <= 1e-5 * max(q[c.index], 1e-12) + 1e-9


def test_oracle_render_progressive(ref):
    tables = dict(cie=ref.cie_xyz(), basis=ref.basis_rgb(), luts=reference_luts())
    sc = scenes.cornell_box(seed=2, cie_xyz=tables["cie"], width=16, height=16, spp=6)
    keep = load_scene_into_ref(ref, sc, tables["luts"], tables["cie"], tables["basis"])
    full = ref_render(ref, 16, 16, 0, 6)
    ref.lib.rbref_render(0, 2, 0)
    ref.lib.rbref_render(2, 4, 0)
    part = np.zeros_like(full)
    ref.lib.rbref_read_accum(_np_ptr(part))
    assert np.array_equal(full, part)
    assert np.isfinite(full).all() and (full[..., 3] == 6).all()
    assert full[..., 1].sum() > 0


# ------------------------------------------------------ light-tree builder
def _random_emitters(seed, n, planar=False):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-5, 5, (n, 3))
    if planar:
        c[:, 1] = 2.0
    e1 = rng.normal(size=(n, 3)) * 0.2
    e2 = rng.normal(size=(n, 3)) * 0.2
    if planar:
        e1[:, 1] = 0.0
        e2[:, 1] = 0.0
    world = np.concatenate([c, c + e1, c + e2], 1).astype(np.float32)
    area = 0.5 * np.linalg.norm(np.cross(e1, e2), axis=1)
    flux = (np.exp(rng.normal(0, 1.5, n)) * area * np.pi).astype(np.float32)
    return world, flux, rng.integers(0, 7, n).astype(np.uint32), np.arange(n, dtype=np.uint32)


@pytest.mark.parametrize("seed,n,planar,camera", [
    (1, 2, False, (0.0, 0.0, 0.0)),
    (2, 9, False, (0.0, 0.0, 0.0)),
    (3, 96, True, (0.0, 0.0, 0.0)),
    (4, 1000, False, (1.25, -0.5, 3.0)),
    (5, 4096, False, (0.0, 0.0, 0.0)),
])
def test_light_tree_builder_matches_reference(ref, seed, n, planar, camera):
    """The library's builder reproduces the reference builder byte for byte:
    nodes, light pointers, path bitmasks and light records."""
    from ratbite_b200 import lighttree
    world, flux, mat, prim = _random_emitters(seed, n, planar)
    want = ref.build_light_tree(world, flux, mat, prim, camera)
    got = lighttree.build(world, flux, mat, prim, camera)
    for name, w, g in zip(("triangles", "nodes", "pointers", "bitmasks"), want, got):
        assert w.shape == g.shape, name
        assert w.tobytes() == g.tobytes(), name


def test_light_tree_builder_rejects_bad_input():
    from ratbite_b200 import lighttree
    from ratbite_b200._native import NativeError
    world, flux, mat, prim = _random_emitters(9, 4)
    world[0, 0] = np.nan
    with pytest.raises(NativeError):
        lighttree.build(world, flux, mat, prim)
    world, flux, mat, prim = _random_emitters(9, 4)
    flux[1] = 0.0
    with pytest.raises(NativeError):
        lighttree.build(world, flux, mat, prim)


# --------------------------------------------------------------- resolve
@pytest.mark.parametrize("cs,name", [(0, "sRGB"), (1, "DCI_P3"), (2, "Rec2020")])
def test_colorspace_matrix_matches_reference(ref, cs, name):
    from ratbite_b200 import color
    want = np.zeros(9, np.float32)
    ref.lib.rbref_colorspace_matrix(cs, want.ctypes.data)
    # with the reference's white point (from its D65 spectrum) the restatement agrees to float rounding
    got = color.colorspace_matrix(name, white_xyz=color.white_of(want))
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-6)
    # the default white point (CIE D65 chromaticity) is within 2e-3
    np.testing.assert_allclose(color.colorspace_matrix(name), want, rtol=2e-3, atol=2e-3)


def test_png_round_trip(tmp_path):
    from ratbite_b200 import image_io
    img = (np.random.default_rng(3).random((9, 13, 4)) * 256).astype(np.uint8)
    image_io.write_png(tmp_path / "x.png", img)
    assert np.array_equal(image_io.read_png(tmp_path / "x.png"), img)
    with pytest.raises(ValueError):
        image_io.write_png(tmp_path / "y.png", img[..., :3])


# ------------------------------------------------------- progressive schedule
def _reference_schedule(total, gradual):
    """updateSamplingState (src/core/rendering_interface.cpp:1859-1872) after a
    restart (offset 0, count 1, :1830-1839), restated."""
    out, offset, count = [], 0, (1 if total else 0)
    while count:
        out.append((offset, count))
        offset += count
        size = min(int(max(3, count) ** 1.5), 64) if gradual else 1
        count = min(max(0, total - offset), size)
    return out


@pytest.mark.parametrize("total", [0, 1, 2, 3, 5, 64, 100, 1000, 4096])
@pytest.mark.parametrize("mode", [0, 1])
def test_progressive_plan_matches_reference_schedule(total, mode):
    lib = _native.load()
    offs = np.zeros(5000, np.uint32)
    cnts = np.zeros(5000, np.uint32)
    n = lib.rb_progressive_plan(total, mode, offs.ctypes.data, cnts.ctypes.data, 5000)
    want = _reference_schedule(total, mode == 1)
    assert n == len(want)
    assert list(zip(offs[:n].tolist(), cnts[:n].tolist())) == want
    assert int(cnts[:n].sum()) == total


def test_progressive_plan_rejects_bad_input():
    lib = _native.load()
    assert lib.rb_progressive_plan(10, 2, None, None, 0) < 0
    assert lib.rb_progressive_plan(10, 1, None, None, 4) < 0
    assert lib.rb_progressive_plan(10, 1, None, None, 0) == len(_reference_schedule(10, True))


def test_oracle_libm_jitter_is_off_by_default_and_reversible(ref):
    """The libm jitter of the oracle (oracle/shim/libm_jitter.cpp) that the
    GPU parity tests use to measure the reference's own sensitivity: off, the
    light-tree pdfs are exactly the plain oracle's; on, some move by a few
    ulps (the wrapped libm calls really go through it); off again, exact."""
    sc = cases.many_lights_scene()
    cie, basis = ref.cie_xyz(), ref.basis_rgb()
    keep = load_scene_into_ref(ref, sc, reference_luts(), cie, basis)
    cs = cases.light_cases(n=512)
    n = len(cs)

    def run():
        out = (abi.rb_light_case * n).from_buffer_copy(bytes(cs))
        ref.lib.rbref_light_tree(n, C.cast(out, C.c_void_p))
        return np.array([c.pdf for c in out], np.float64)

    base = run()
    assert np.array_equal(run(), base)
    ref.lib.rbref_set_libm_jitter(1, 7)
    try:
        moved = run()
    finally:
        ref.lib.rbref_set_libm_jitter(0, 0)
    rel = np.abs(moved - base) / np.maximum(np.abs(base), 1e-30)
    assert (rel > 0).mean() > 0.5
    assert np.median(rel[rel > 0]) < 1e-5
    assert np.array_equal(run(), base)
    del keep
