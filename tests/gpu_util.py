"""GPU-side helpers for the parity tests: device buffers come from torch
(plumbing only); every evaluation goes through the C ABI of
libratbite_b200.so."""
from __future__ import annotations

import ctypes as C

import numpy as np

from ratbite_b200 import abi
from ratbite_b200._native import check, load


def torch():
    import torch as t
    return t


def dev(a: np.ndarray):
    t = torch()
    return t.from_numpy(np.ascontiguousarray(a)).cuda()


def ptr(t):
    return C.c_void_p(t.data_ptr())


def host(t) -> np.ndarray:
    torch().cuda.synchronize()
    return t.cpu().numpy()


def empty(shape, dtype):
    t = torch()
    return t.zeros(shape, dtype=dtype, device="cuda")


def struct_array_to_device(arr):
    """ctypes structure array -> device byte tensor (same layout)."""
    t = torch()
    raw = np.frombuffer(bytes(arr), dtype=np.uint8).copy()
    return t.from_numpy(raw).cuda()


def device_to_struct_array(tensor, ctype, n):
    raw = host(tensor).tobytes()
    return (ctype * n).from_buffer_copy(raw)


def run_bxdf(ri, cases):
    lib = load()
    d = struct_array_to_device(cases)
    check(lib.rb_k_bxdf(ri.ctx, len(cases), ptr(d), None), ri.ctx, "rb_k_bxdf")
    return device_to_struct_array(d, abi.rb_bxdf_case, len(cases))


def run_light(ri, cases):
    lib = load()
    d = struct_array_to_device(cases)
    check(lib.rb_k_light_tree(ri.ctx, len(cases), ptr(d), None), ri.ctx, "rb_k_light_tree")
    return device_to_struct_array(d, abi.rb_light_case, len(cases))


# Image parity bounds. With identical sample sequences a path differs from
# the oracle's only after a branch flip (see test_bxdf_parity) or a
# light-tree child flip; every other path gives the same radiance up to libm
# ulps. Measured on B200 (Cornell box, 32 emitters, instanced geometry with an
# env map): image means within 1e-8 relative and per-pixel L1 within 3e-7.
IMG_MEAN_TOL = 1e-6
IMG_L1_TOL = 1e-5


def _image_stats(got, want):
    """Image-mean relative difference and per-pixel L1 (sum |g - w| over
    sum |w|) of the per-pixel XYZ means."""
    g = got[..., :3] / np.maximum(got[..., 3:4], 1)
    w = want[..., :3] / np.maximum(want[..., 3:4], 1)
    rel_mean = abs(g.sum() - w.sum()) / abs(w.sum())
    l1 = np.abs(g - w).sum() / np.abs(w).sum()
    return rel_mean, l1


def assert_image_parity(name, got, want):
    assert np.array_equal(got[..., 3], want[..., 3])
    rel_mean, l1 = _image_stats(got, want)
    same = np.mean(np.all(got[..., :3] == want[..., :3], axis=-1))
    print(f"{name}: image-mean rel diff {rel_mean:.3e}, per-pixel L1 {l1:.3e}, pixels bit-identical {same:.2%}")
    assert rel_mean <= IMG_MEAN_TOL
    assert l1 <= IMG_L1_TOL
