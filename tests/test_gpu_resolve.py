"""GPU parity of the resolve (rb_k_resolve, rb_resolve) against the
reference's own renderResolve + AgX kernel (src/kernels/image.cu) compiled for
sm_100a and run by the oracle harness on the same device data.

Tolerance: none. Both kernels evaluate the same float expressions with the
compiler's default multiply-add contraction, and the bytes are identical
(measured on B200 for every case below, including empty pixels, negative sums
and overflowing values).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gpu_util import dev, torch
from oracle_lib import RefImageGpu, RefLib, reference_luts
from ratbite_b200 import image_io, lighttree, scenes
from ratbite_b200._native import check, load
from ratbite_b200.rendering_interface import RenderingInterface

pytestmark = pytest.mark.gpu


def _compare(got, want):
    d = np.abs(got.astype(np.int16) - want.astype(np.int16))
    print(f"resolve: {got.size} bytes, identical {np.mean(d == 0):.6%}, max diff {d.max()}")
    assert d.max() == 0


def _render_data(w, h, seed):
    """Accumulation-like data: sums of up to 1024 samples over a wide dynamic
    range, with empty pixels (count 0), negative sums and huge values."""
    rng = np.random.default_rng(seed)
    n = rng.integers(0, 1025, (h, w)).astype(np.float64)
    xyz = np.exp(rng.normal(-1.0, 3.0, (h, w, 3))) * n[..., None]
    xyz[rng.random((h, w)) < 0.01] *= -1.0
    xyz[rng.random((h, w)) < 0.001] = 1e30
    data = np.concatenate([xyz, n[..., None]], axis=2)
    data[0, 0] = (0.0, 0.0, 0.0, 0.0)
    data[0, 1] = (1.0, 1.0, 1.0, 1.0)
    return np.ascontiguousarray(data)


@pytest.mark.parametrize("w,h,exposure", [(256, 256, 0.0), (1920, 1080, 2.5), (33, 7, -3.0)])
def test_k_resolve_matches_reference_kernel(w, h, exposure):
    ref = RefLib()
    cs = np.zeros(9, np.float32)
    ref.lib.rbref_colorspace_matrix(0, cs.ctypes.data)
    data = dev(_render_data(w, h, w + h))
    scale = float(2.0 ** (exposure - 7.0))
    want = RefImageGpu().resolve(w, h, cs, scale, data.data_ptr())
    out = torch().zeros((h, w, 4), dtype=torch().uint8, device="cuda")
    check(load().rb_k_resolve(w, h, cs.ctypes.data, scale, C.c_void_p(data.data_ptr()),
                              C.c_void_p(out.data_ptr()), None), None, "rb_k_resolve")
    torch().cuda.synchronize()
    _compare(out.cpu().numpy(), want)


def test_rendered_frame_resolves_like_reference(tmp_path):
    ref = RefLib()
    cie, basis = ref.cie_xyz(), ref.basis_rgb()
    sc = scenes.cornell_box(seed=1, cie_xyz=cie, width=64, height=64, spp=16)
    ri = RenderingInterface(device=0)
    ri.load_scene(sc, reference_luts(), cie, basis, light_tree=lighttree.build_for_scene(sc))
    ri.render(0, 16)
    cs = np.zeros(9, np.float32)
    ref.lib.rbref_colorspace_matrix(0, cs.ctypes.data)
    ri.resolve(exposure=6.0, colorspace=cs)
    got = ri.read_image()
    want = RefImageGpu().resolve(64, 64, cs, float(2.0 ** (6.0 - 7.0)), ri.accumulation_device_ptr())
    ri.cleanup()
    _compare(got, want)
    assert got[..., :3].mean() > 5.0                  # the box is lit, not black
    image_io.write_png(tmp_path / "cornell.png", got)
    assert np.array_equal(image_io.read_png(tmp_path / "cornell.png"), got)
