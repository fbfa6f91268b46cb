"""Light-tree construction through the C ABI (rb_build_light_tree): the
host restatement of ratbite's LightTree::Builder, producing the records
rb_set_lights uploads."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from ._native import NativeError, load


def build(world: np.ndarray, flux: np.ndarray, material: np.ndarray, primitive: np.ndarray,
          camera=(0.0, 0.0, 0.0)):
    """Returns (triangles, nodes, pointers, bitmasks) numpy arrays."""
    n = len(flux)
    world = np.ascontiguousarray(world, np.float32).reshape(n, 9)
    flux = np.ascontiguousarray(flux, np.float32)
    material = np.ascontiguousarray(material, np.uint32)
    primitive = np.ascontiguousarray(primitive, np.uint32)
    cam = np.ascontiguousarray(camera, np.float64)
    tris = np.zeros(n, abi.emissive_triangle_dtype())
    nodes = np.zeros(max(2 * n, 1), abi.packed_node_dtype())
    ptrs = np.zeros(n, np.uint32)
    masks = np.zeros(n, np.uint64)
    count = C.c_uint32(0)
    p = lambda a: C.c_void_p(a.ctypes.data)
    rc = load().rb_build_light_tree(n, p(world), p(flux), p(material), p(primitive), p(cam), p(tris), p(nodes),
                                    p(ptrs), p(masks), C.byref(count))
    if rc != 0:
        raise NativeError(f"rb_build_light_tree failed with status {rc}")
    return tris, nodes[:count.value].copy(), ptrs, masks


def record(tris, nodes, ptrs, masks) -> abi.rb_light_tree:
    """rb_light_tree record pointing into the arrays (kept alive on it)."""
    lt = abi.rb_light_tree()
    lt.triangle_count = len(tris)
    lt.triangles = tris.ctypes.data
    lt.node_count = len(nodes)
    lt.nodes = nodes.ctypes.data if len(nodes) else None
    lt.pointer_count = len(ptrs)
    lt.pointers = ptrs.ctypes.data
    lt.bitmasks = masks.ctypes.data
    lt._arrays = (tris, nodes, ptrs, masks)
    return lt


def build_for_scene(scene, camera=(0.0, 0.0, 0.0)) -> abi.rb_light_tree | None:
    world, flux, mat, prim = scene.emissive_arrays()
    if len(flux) == 0:
        return None
    tris, nodes, ptrs, masks = build(world, flux, mat, prim, camera)
    tris["uvs"] = scene.emissive_uvs()          # the triangles keep the input order
    return record(tris, nodes, ptrs, masks)


def build_on_device(world: np.ndarray, flux: np.ndarray, material: np.ndarray, primitive: np.ndarray,
                    camera=(0.0, 0.0, 0.0), stream=None, timing: list | None = None, uvs=None):
    """The same records built on the device (rb_k_build_light_tree), copied
    back: (triangles, nodes, pointers, bitmasks). Inputs are uploaded from
    host arrays; with `timing`, the device milliseconds of the build (CUDA
    events around the launch) are appended to it."""
    import torch
    n = len(flux)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    w = dev(np.asarray(world, np.float32).reshape(n, 9))
    f = dev(np.asarray(flux, np.float32))
    m = dev(np.asarray(material, np.uint32).view(np.int32))
    pr = dev(np.asarray(primitive, np.uint32).view(np.int32))
    uv = None if uvs is None else dev(np.asarray(uvs, np.float32).reshape(n, 6))
    lib = load()
    scratch = torch.empty(max(int(lib.rb_k_build_light_tree_scratch_bytes(n)), 1), dtype=torch.uint8, device="cuda")
    tris = torch.zeros(max(n, 1) * 68, dtype=torch.uint8, device="cuda")
    nodes = torch.zeros(max(2 * n, 1) * 32, dtype=torch.uint8, device="cuda")
    ptrs = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
    masks = torch.zeros(max(n, 1), dtype=torch.int64, device="cuda")
    count = torch.zeros(1, dtype=torch.int32, device="cuda")
    cam = np.ascontiguousarray(camera, np.float64)
    p = lambda t: C.c_void_p(t.data_ptr())
    s = torch.cuda.current_stream() if stream is None else stream
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    rc = lib.rb_k_build_light_tree(n, p(w), p(f), p(m), p(pr), None if uv is None else p(uv),
                                   C.c_void_p(cam.ctypes.data), p(scratch), p(tris),
                                   p(nodes), p(ptrs), p(masks), p(count), C.c_void_p(s.cuda_stream))
    b.record(s)
    if rc != 0:
        raise NativeError(f"rb_k_build_light_tree failed with status {rc}", rc)
    b.synchronize()
    if timing is not None:
        timing.append(a.elapsed_time(b))
    k = int(count.item())
    out_tris = np.frombuffer(tris.cpu().numpy().tobytes(), abi.emissive_triangle_dtype())[:n].copy()
    out_nodes = np.frombuffer(nodes.cpu().numpy().tobytes(), abi.packed_node_dtype())[:k].copy()
    return out_tris, out_nodes, ptrs.cpu().numpy().view(np.uint32)[:n].copy(), masks.cpu().numpy().view(np.uint64)[:n].copy()
