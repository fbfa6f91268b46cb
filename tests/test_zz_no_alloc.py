"""The no-allocation CDF entry point (rb_envmap_cdf_noalloc) against the
regular one (rb_envmap_cdf), through the C ABI.

rb_envmap_cdf_noalloc serves callers that may not allocate device memory
while they run (a host that owns a fixed device-memory budget, or a
per-frame loop that cannot afford the device-wide synchronisation cudaMalloc
and cudaFree may cause). Its scratch is a static device array inside the
library, so the results must be identical to the regular entry point's, call
after call, even though every call reuses that same array. This file is
collected last, and it also passes on its own in a fresh process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _image(w, h, seed):
    rng = np.random.default_rng(seed)
    img = rng.random((h, w, 4)).astype(np.float32)
    img[h // 3, w // 4, :3] = 5e3
    return img


def _run(fn_name, img, mode, scratch=None):
    import torch
    from ratbite_b200._native import load
    lib = load()
    h, w = img.shape[:2]
    d = torch.from_numpy(img).cuda()
    cond = torch.zeros(w * h, dtype=torch.int16, device="cuda")
    marg = torch.zeros(h, dtype=torch.int16, device="cuda")
    integ = torch.zeros(1, dtype=torch.float32, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())
    if fn_name == "rb_envmap_cdf":
        rc = lib.rb_envmap_cdf(w, h, p(d), mode, p(scratch), p(cond), p(marg), p(integ), None)
    else:
        rc = lib.rb_envmap_cdf_noalloc(w, h, p(d), mode, p(cond), p(marg), p(integ), None)
    assert rc == 0, rc
    torch.cuda.synchronize()
    return (cond.cpu().numpy().view(np.uint16).copy(), marg.cpu().numpy().view(np.uint16).copy(),
            float(integ.cpu().numpy()[0]))


@pytest.mark.parametrize("mode", [0, 1])
def test_noalloc_matches_regular_entry_point_twice(mode):
    import torch
    from ratbite_b200._native import load
    # two different images, back to back: the shared scratch keeps the last
    # call's contents, which must not leak into the next result
    for seed, (w, h) in ((1, (512, 256)), (2, (1024, 512))):
        img = _image(w, h, seed)
        scratch = torch.zeros(int(load().rb_envmap_cdf_scratch_bytes(w, h)), dtype=torch.uint8, device="cuda")
        want = _run("rb_envmap_cdf", img, mode, scratch)
        got = _run("rb_envmap_cdf_noalloc", img, mode)
        assert np.array_equal(got[0], want[0])
        assert np.array_equal(got[1], want[1])
        assert got[2] == want[2]


@pytest.mark.parametrize("mode", [0, 1])
def test_noalloc_at_its_maximum_height(mode):
    """An image exactly as tall as the static scratch was sized for (8192
    rows), against the regular entry point given scratch filled with 0xFF
    bytes (its contents on entry must not matter)."""
    import torch
    from ratbite_b200._native import load
    w, h = 8, 8192
    img = _image(w, h, 7)
    scratch = torch.full((int(load().rb_envmap_cdf_scratch_bytes(w, h)),), 0xFF, dtype=torch.uint8, device="cuda")
    want = _run("rb_envmap_cdf", img, mode, scratch)
    got = _run("rb_envmap_cdf_noalloc", img, mode)
    assert np.array_equal(got[0], want[0])
    assert np.array_equal(got[1], want[1])
    assert got[2] == want[2]


def test_noalloc_rejects_images_taller_than_its_scratch():
    import torch
    from ratbite_b200 import abi
    from ratbite_b200._native import load
    x = torch.zeros(16, dtype=torch.uint8, device="cuda")
    p = C.c_void_p(x.data_ptr())
    assert load().rb_envmap_cdf_noalloc(8, 8192 + 4, p, 0, p, p, p, None) == abi.RB_ERR_TOO_LARGE
