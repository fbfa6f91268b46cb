"""Loader of the native library (ratbite_b200/_lib/libratbite_b200.so).

The library is the product: every render and every per-function evaluation
runs in its sm_100a kernels. There is no Python or CPU fallback; if the
library is missing or the device is not usable the calls fail loudly.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

from . import abi

LIB_DIR = Path(__file__).resolve().parent / "_lib"
LIB_PATH = LIB_DIR / "libratbite_b200.so"

_P = C.c_void_p
_U32 = C.c_uint32

# name -> (restype, argtypes); every symbol declared in include/*.h.
SIGNATURES = {
    "rb_abi_version": (C.c_int, []),
    "rb_create": (C.c_int, [C.POINTER(abi.rb_config), C.POINTER(_P)]),
    "rb_destroy": (C.c_int, [_P]),
    "rb_last_error": (C.c_char_p, [_P]),
    "rb_set_luts": (C.c_int, [_P] * 7),
    "rb_set_spectra": (C.c_int, [_P, _P, _P, _P, _U32]),
    "rb_set_materials": (C.c_int, [_P, _P, _U32]),
    "rb_set_textures": (C.c_int, [_P, _P, _U32]),
    "rb_set_geometry": (C.c_int, [_P, _P]),
    "rb_set_lights": (C.c_int, [_P, _P]),
    "rb_set_light_origin": (C.c_int, [_P, _P, _P]),
    "rb_build_lights": (C.c_int, [_P, _U32, _P, _P, _P, _P, _P, _P]),
    "rb_update_instances": (C.c_int, [_P, _P, _P, _P]),
    "rb_build_light_tree": (C.c_int, [_U32, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "rb_set_envmap": (C.c_int, [_P, _P, _U32, _U32]),
    "rb_clear_envmap": (C.c_int, [_P]),
    "rb_rebuild_envmap_cdf": (C.c_int, [_P, _P]),
    "rb_set_launch": (C.c_int, [_P, _P]),
    "rb_render": (C.c_int, [_P, _U32, _U32, _P]),
    "rb_render_graph": (C.c_int, [_P, _U32, _U32, _P]),
    "rb_render_jobs": (C.c_int, [_P, _U32, _P, _P, _P, _P]),
    "rb_read_accum": (C.c_int, [_P, _P]),
    "rb_write_accum": (C.c_int, [_P, _P]),
    "rb_accum_device_ptr": (C.c_int, [_P, C.POINTER(_P)]),
    "rb_copy_accum_async": (C.c_int, [_P, _P, _P]),
    "rb_clear_accum": (C.c_int, [_P, _P]),
    "rb_progressive_restart": (C.c_int, [_P, _U32, C.c_int]),
    "rb_progressive_step": (C.c_int, [_P, _P, C.POINTER(abi.rb_progress)]),
    "rb_progressive_plan": (C.c_int, [_U32, C.c_int, _P, _P, _U32]),
    "rb_resolve": (C.c_int, [_P, _P, C.c_float, _P]),
    "rb_read_image": (C.c_int, [_P, _P]),
    "rb_image_device_ptr": (C.c_int, [_P, C.POINTER(_P)]),
    "rb_status": (C.c_int, [_P, C.POINTER(abi.rb_device_status)]),
    "rb_clear_status": (C.c_int, [_P]),
    "rb_synchronize": (C.c_int, [_P]),
    "rb_set_stats": (C.c_int, [_P, _U32]),
    "rb_get_stats": (C.c_int, [_P, C.POINTER(abi.rb_render_stats)]),
    "rb_k_sobol": (C.c_int, [_U32, _U32, _P, _P, _P, _P, _P, _P]),
    "rb_k_pixel_hash": (C.c_int, [_U32, _P, _P, _P, _P]),
    "rb_k_wavelengths": (C.c_int, [_U32, _P, _P, _P, _P]),
    "rb_k_texture_sample": (C.c_int, [_P, _U32, _U32, _P, _P, _P, _P]),
    "rb_k_camera_ray": (C.c_int, [_P, _U32, _P, _P, _P, _P, _P]),
    "rb_k_bxdf": (C.c_int, [_P, _U32, _P, _P]),
    "rb_k_light_tree": (C.c_int, [_P, _U32, _P, _P]),
    "rb_k_offset_point": (C.c_int, [_U32, _P, _P, _P, _P]),
    "rb_k_oct_encode": (C.c_int, [_U32, _P, _P, _P]),
    "rb_k_oct_decode": (C.c_int, [_U32, _P, _P, _P]),
    "rb_k_trace": (C.c_int, [_P, _U32, _P, _P, _P, _P, _P]),
    "rb_k_occluded": (C.c_int, [_P, _U32, _P, _P, _P, _P]),
    "rb_k_resolve": (C.c_int, [_U32, _U32, _P, C.c_float, _P, _P, _P]),
    "rb_k_generate_sheen_lut": (C.c_int, [_U32, _P, _P]),
    "rb_k_generate_luts": (C.c_int, [_U32, _P, _P, _P, _P, _P, _P]),
    "rb_envmap_cdf_scratch_bytes": (C.c_size_t, [_U32, _U32]),
    "rb_envmap_cdf": (C.c_int, [_U32, _U32, _P, C.c_int, _P, _P, _P, _P, _P]),
    "rb_envmap_cdf_noalloc": (C.c_int, [_U32, _U32, _P, C.c_int, _P, _P, _P, _P]),
    "rb_nrc_create": (C.c_int, [C.POINTER(abi.rb_nrc_config), C.POINTER(_P)]),
    "rb_nrc_destroy": (C.c_int, [_P]),
    "rb_nrc_grid_size": (C.c_size_t, []),
    "rb_nrc_weight_count": (C.c_size_t, []),
    "rb_nrc_set_parameters": (C.c_int, [_P, _P, _P]),
    "rb_nrc_get_parameters": (C.c_int, [_P, _P, _P]),
    "rb_nrc_infer": (C.c_int, [_P, _U32, _P, _P, _P]),
    "rb_nrc_train": (C.c_int, [_P, _U32, _P, _P, _P, _P]),
    "rb_nrc_gradients": (C.c_int, [_P, _U32, _P, _P, _P, _P]),
    "rb_nrc_status": (C.c_int, [_P, _P]),
    "rb_k_build_light_tree_scratch_bytes": (C.c_size_t, [_U32]),
    "rb_k_build_light_tree": (C.c_int, [_U32] + [_P] * 12 + [_P]),
    "rb_attach_radiance_cache": (C.c_int, [_P, _P, C.POINTER(abi.rb_cache_params)]),
    "rb_get_cache_stats": (C.c_int, [_P, C.POINTER(abi.rb_cache_stats)]),
}

_lib = None


class NativeError(RuntimeError):
    """A library call failed; `code` is its RB_ERR_* status (None when the
    library itself could not be loaded)."""

    def __init__(self, msg: str, code: int | None = None):
        super().__init__(msg)
        self.code = code


def load() -> C.CDLL:
    """Loads the library once (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise NativeError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                          "(or make -C ratbite_b200/csrc)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.rb_abi_version() != abi.RB_ABI_VERSION:
        raise NativeError("ABI version mismatch between include/ratbite_b200.h and the built library")
    _lib = lib
    return lib


# cudaStreamLegacy: the legacy default stream as an explicit handle.
CUDA_STREAM_LEGACY = 0x1


def stream_arg(stream):
    """The ctypes stream argument of the context calls (rb_render and the
    rest): None keeps the library's own stream (the C ABI's NULL); a handle
    of 0, which is what torch reports for the default stream, is passed as
    cudaStreamLegacy so that the work is ordered on that stream as the
    caller means, not on the library's."""
    if stream is None:
        return None
    return C.c_void_p(int(stream) if int(stream) else CUDA_STREAM_LEGACY)


def check(rc: int, ctx=None, what: str = ""):
    if rc != 0:
        msg = ""
        if ctx is not None:
            m = load().rb_last_error(ctx)
            msg = m.decode() if m else ""
        raise NativeError(f"{what} failed with status {rc}: {msg}", rc)
