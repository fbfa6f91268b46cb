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
