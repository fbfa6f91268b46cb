"""Test-side access to the oracle (oracle/_ref, built by oracle/Makefile).

The oracle is the reference's own per-sample path compiled host-side
(libratbite_ref.so), the reference's GPU CDF kernels compiled for sm_100a
(libratbite_ref_cdf.so) and the project's C restatements
(liboracle_restate.so). Only tests, the smoke check and the CPU baseline of
bench.py use it.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from ratbite_b200 import abi

ROOT = Path(__file__).resolve().parents[1]
REF_DIR = ROOT / "oracle" / "_ref"

_P = C.c_void_p
_U32 = C.c_uint32


def _np_ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class RefLib:
    """ctypes wrapper of libratbite_ref.so (oracle/ref_harness.cpp)."""

    def __init__(self, path: Path | None = None):
        path = path or REF_DIR / "libratbite_ref.so"
        if not path.exists():
            raise FileNotFoundError(f"oracle library missing: {path} (run make -C oracle)")
        self.lib = C.CDLL(str(path))
        L = self.lib
        for name, res, args in [
            ("rbref_abi_version", C.c_int, []),
            ("rbref_reset", None, []),
            ("rbref_set_texture_weight_mode", None, [C.c_int]),
            ("rbref_cie_xyz", None, [_P]),
            ("rbref_basis_rgb", None, [_P]),
            ("rbref_named_spectrum", C.c_int, [C.c_int, _P]),
            ("rbref_set_spectra", C.c_int, [_P, _P, _P, _U32]),
            ("rbref_set_luts", C.c_int, [_P] * 6),
            ("rbref_set_materials", C.c_int, [_P, _U32]),
            ("rbref_set_textures", C.c_int, [_P, _U32]),
            ("rbref_set_geometry", C.c_int, [_P]),
            ("rbref_set_lights", C.c_int, [_P]),
            ("rbref_set_envmap", C.c_int, [_P, _U32, _U32, _P, _P, C.c_float]),
            ("rbref_clear_envmap", None, []),
            ("rbref_set_launch", C.c_int, [_P]),
            ("rbref_render", C.c_int, [_U32, _U32, C.c_int]),
            ("rbref_render_rows", C.c_int, [_U32, _U32, C.c_int, _U32, _U32]),
            ("rbref_render_strided", C.c_int64, [_U32, _U32, C.c_int, _U32, _U32]),
            ("rbref_read_accum", None, [_P]),
            ("rbref_write_accum", None, [_P]),
            ("rbref_sobol", None, [_U32, _U32, _P, _P, _P, _P, _P]),
            ("rbref_pixel_hash", None, [_U32, _P, _P, _P]),
            ("rbref_wavelengths", None, [_U32, _P, _P, _P]),
            ("rbref_camera_ray", None, [_U32, _P, _P, _P, _P]),
            ("rbref_bxdf", None, [_U32, _P]),
            ("rbref_light_tree", None, [_U32, _P]),
            ("rbref_offset_point", None, [_U32, _P, _P, _P]),
            ("rbref_oct_encode", None, [_U32, _P, _P]),
            ("rbref_oct_decode", None, [_U32, _P, _P]),
            ("rbref_trace", None, [_U32, _P, _P, _P, _P]),
            ("rbref_occluded", None, [_U32, _P, _P, _P]),
            ("rbref_build_light_tree", C.c_int, [_U32, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
            ("rbref_colorspace_matrix", None, [C.c_int, _P]),
            ("rbref_sizeof_material_data", _U32, []),
            ("rbref_set_libm_jitter", None, [C.c_int, C.c_uint64]),
            ("rbref_sizeof_launch_parameters", _U32, []),
        ]:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args

    # ---- data tables -----------------------------------------------------
    def cie_xyz(self) -> np.ndarray:
        out = np.zeros((3, abi.RB_SPECTRUM_BINS), np.float32)
        self.lib.rbref_cie_xyz(_np_ptr(out))
        return out

    def basis_rgb(self) -> np.ndarray:
        out = np.zeros((3, abi.RB_SPECTRUM_BINS), np.float32)
        self.lib.rbref_basis_rgb(_np_ptr(out))
        return out

    def named_spectrum(self, t: int) -> np.ndarray:
        out = np.zeros(abi.RB_SPECTRUM_BINS, np.float32)
        assert self.lib.rbref_named_spectrum(t, _np_ptr(out)) == 0
        return out

    # ---- light tree builder (the reference's LightTree::Builder) -----------
    def build_light_tree(self, world, flux, material, prim, camera=(0.0, 0.0, 0.0)):
        n = len(flux)
        tris = np.zeros(n, abi.emissive_triangle_dtype())
        nodes = np.zeros(max(2 * n, 1), abi.packed_node_dtype())
        ptrs = np.zeros(n, np.uint32)
        masks = np.zeros(n, np.uint64)
        cam = np.asarray(camera, np.float64)
        world = np.ascontiguousarray(world, np.float32)
        flux = np.ascontiguousarray(flux, np.float32)
        material = np.ascontiguousarray(material, np.uint32)
        prim = np.ascontiguousarray(prim, np.uint32)
        cnt = self.lib.rbref_build_light_tree(n, _np_ptr(world), _np_ptr(flux), _np_ptr(material),
                                              _np_ptr(prim), _np_ptr(cam), _np_ptr(tris),
                                              _np_ptr(nodes), _np_ptr(ptrs), _np_ptr(masks))
        return tris, nodes[:cnt].copy(), ptrs, masks


def reference_luts() -> dict:
    """The reference's six LUT files (bin/*.bin), staged into oracle/_ref/bin
    by the oracle build. Layouts: 32x32 float, 4 x 32^3 float, 32x32 float4."""
    d = REF_DIR / "bin"
    rd = lambda n: np.fromfile(d / n, dtype=np.float32)
    return dict(
        conductor=rd("albedoConductorLUT.bin"),
        dielectric_outer=rd("albedoDielectricOuterLUT.bin"),
        dielectric_inner=rd("albedoDielectricInnerLUT.bin"),
        reflective_outer=rd("albedoDielectricReflectiveOuterLUT.bin"),
        reflective_inner=rd("albedoDielectricReflectiveInnerLUT.bin"),
        sheen=rd("sheenLUT.bin"),
    )


def light_tree_record(tris, nodes, ptrs, masks, keep: list):
    lt = abi.rb_light_tree()
    for a in (tris, nodes, ptrs, masks):
        keep.append(a)
    lt.triangle_count = len(tris)
    lt.triangles = tris.ctypes.data
    lt.node_count = len(nodes)
    lt.nodes = nodes.ctypes.data if len(nodes) else None
    lt.pointer_count = len(ptrs)
    lt.pointers = ptrs.ctypes.data
    lt.bitmasks = masks.ctypes.data
    keep.append(lt)
    return lt


def load_scene_into_ref(ref: RefLib, scene, luts: dict, cie, basis, extra=None, width=None,
                        height=None, max_depth=None):
    """Uploads `scene` into the oracle exactly as the product is fed."""
    keep = []
    L = ref.lib
    L.rbref_reset()
    extra = np.zeros((1, abi.RB_SPECTRUM_BINS), np.float32) if extra is None else extra
    for a in (cie, basis, extra):
        keep.append(a)
    L.rbref_set_spectra(_np_ptr(cie), _np_ptr(basis), _np_ptr(extra), len(extra))
    lut_arrays = [np.ascontiguousarray(luts[k], np.float32) for k in
                  ("conductor", "dielectric_outer", "dielectric_inner", "reflective_outer",
                   "reflective_inner", "sheen")]
    keep += lut_arrays
    L.rbref_set_luts(*[_np_ptr(a) for a in lut_arrays])
    texs = scene.texture_records()
    keep.append(texs)
    assert L.rbref_set_textures(C.cast(texs, C.c_void_p), len(texs)) == 0
    mats = scene.material_records()
    assert L.rbref_set_materials(C.cast(mats, C.c_void_p), len(mats)) == 0
    g = scene.geometry_record()
    assert L.rbref_set_geometry(C.byref(g)) == 0
    world, flux, mat, prim = scene.emissive_arrays()
    if len(flux):
        tris, nodes, ptrs, masks = ref.build_light_tree(world, flux, mat, prim)
        tris["uvs"] = scene.emissive_uvs()
        lt = light_tree_record(tris, nodes, ptrs, masks, keep)
        L.rbref_set_lights(C.byref(lt))
    env = getattr(scene, "envmap", None)
    if env is not None:
        keep += set_envmap_into_ref(ref, env)
    launch = scene.launch_record(width, height, max_depth)
    keep.append(launch)
    L.rbref_set_launch(C.byref(launch))
    return keep


def restate_lib():
    lib = C.CDLL(str(REF_DIR / "liboracle_restate.so"))
    lib.orc_envmap_cdf.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.orc_envmap_cdf.restype = C.c_int
    return lib


def set_envmap_into_ref(ref: RefLib, rgba: np.ndarray, mode: int = 0):
    """Environment map for the oracle with CDF tables from the C restatement
    (mode 0: the reference kernels' float order)."""
    img = np.ascontiguousarray(rgba, np.float32)
    h, w = img.shape[:2]
    cond = np.zeros(w * h, np.uint16)
    marg = np.zeros(h, np.uint16)
    integ = np.zeros(1, np.float32)
    assert restate_lib().orc_envmap_cdf(w, h, _np_ptr(img), mode, _np_ptr(cond), _np_ptr(marg), _np_ptr(integ)) == 0
    assert ref.lib.rbref_set_envmap(_np_ptr(img), w, h, _np_ptr(cond), _np_ptr(marg), float(integ[0])) == 0
    return [img, cond, marg]


def ref_render(ref: RefLib, width: int, height: int, offset: int, count: int, threads: int = 0):
    assert ref.lib.rbref_render(offset, count, threads) == 0
    out = np.zeros((height, width, 4), np.float64)
    ref.lib.rbref_read_accum(_np_ptr(out))
    return out


class RefImageGpu:
    """The reference's resolve kernel (src/kernels/image.cu) on the GPU,
    through oracle/ref_image_harness.cpp (checker only)."""

    def __init__(self):
        self.cubin = str(REF_DIR / "image.cubin").encode()
        self.lib = C.CDLL(str(REF_DIR / "libratbite_ref_image.so"))
        self.lib.rbrefgpu_resolve.argtypes = [C.c_char_p, _U32, _U32, _P, C.c_float, _P, _P]
        self.lib.rbrefgpu_resolve.restype = C.c_int

    def resolve(self, width: int, height: int, colorspace: np.ndarray, exposure_scale: float, d_render: int):
        out = np.zeros((height, width, 4), np.uint8)
        cs = np.ascontiguousarray(colorspace, np.float32)
        rc = self.lib.rbrefgpu_resolve(self.cubin, width, height, _np_ptr(cs), exposure_scale, d_render,
                                       _np_ptr(out))
        assert rc == 0, rc
        return out
