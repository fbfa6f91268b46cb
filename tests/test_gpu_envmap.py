"""Environment-map CDF on the GPU.

mode 0 (float32, reference order) must give index tables bit-identical to the
reference's own kernels (src/kernels/cdf.cu, compiled for sm_100a and run on
the same device by oracle/_ref/libratbite_ref_cdf.so); mode 1 (float64 sums)
must equal the C restatement of that mode. Sizes cover the reference's four
block-size/chunk regimes and a non-square ragged case.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from gpu_util import dev, empty, host, ptr, torch
from oracle_lib import REF_DIR, _np_ptr
from ratbite_b200._native import load
from test_cpu import _sky

pytestmark = pytest.mark.gpu

SIZES = [(64, 32), (1024, 512), (2048, 64), (4096, 16), (8192, 8), (1028, 12)]


@pytest.fixture(scope="module")
def refcdf():
    lib = C.CDLL(str(REF_DIR / "libratbite_ref_cdf.so"))
    lib.rbrefgpu_envmap_cdf.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.rbrefgpu_envmap_cdf.restype = C.c_int
    return lib


@pytest.fixture(scope="module")
def restate():
    lib = C.CDLL(str(REF_DIR / "liboracle_restate.so"))
    lib.orc_envmap_cdf.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    return lib


def ours(img, mode):
    h, w = img.shape[:2]
    lib = load()
    d = dev(img)
    scratch = empty(int(lib.rb_envmap_cdf_scratch_bytes(w, h)), torch().uint8)
    cond = empty(w * h, torch().int16)
    marg = empty(h, torch().int16)
    integ = empty(1, torch().float32)
    rc = lib.rb_envmap_cdf(w, h, ptr(d), mode, ptr(scratch), ptr(cond), ptr(marg), ptr(integ), None)
    assert rc == 0
    return host(cond).view(np.uint16).reshape(h, w), host(marg).view(np.uint16), float(host(integ)[0]), scratch


@pytest.mark.parametrize("w,h", SIZES)
def test_mode0_bit_exact_vs_reference_kernels(refcdf, w, h):
    img = _sky(w, h, seed=w + h)
    d = dev(img)
    cond = empty(w * h, torch().int16)
    marg = empty(h, torch().int16)
    integ = np.zeros(1, np.float32)
    rc = refcdf.rbrefgpu_envmap_cdf(str(REF_DIR / "cdf.cubin").encode(), w, h, ptr(d), ptr(cond), ptr(marg), _np_ptr(integ))
    assert rc == 0
    want_c = host(cond).view(np.uint16).reshape(h, w)
    want_m = host(marg).view(np.uint16)
    got_c, got_m, got_i, _ = ours(img, 0)
    assert np.array_equal(got_c, want_c)
    assert np.array_equal(got_m, want_m)
    assert np.float32(got_i).view(np.uint32) == integ.view(np.uint32)[0]


@pytest.mark.parametrize("w,h", SIZES)
def test_mode1_matches_restatement(restate, w, h):
    img = _sky(w, h, seed=3 * w + h)
    cond = np.zeros(w * h, np.uint16)
    marg = np.zeros(h, np.uint16)
    integ = np.zeros(1, np.float32)
    assert restate.orc_envmap_cdf(w, h, _np_ptr(img), 1, _np_ptr(cond), _np_ptr(marg), _np_ptr(integ)) == 0
    got_c, got_m, got_i, _ = ours(img, 1)
    # float64 sums: identical operation order; sin in double may differ in its
    # last bit between CUDA and libm, so the marginal may move by one index
    assert np.array_equal(got_c, cond.reshape(h, w))
    assert np.abs(got_m.astype(np.int64) - marg.astype(np.int64)).max() <= 1
    assert (got_m == marg).mean() > 0.99
    assert abs(got_i - integ[0]) <= 1e-6 * abs(integ[0])


def test_repeated_builds_reuse_scratch():
    img = _sky(256, 128, seed=5)
    a = ours(img, 0)
    # the same scratch must be reusable: the completion ticket resets itself
    lib = load()
    h, w = img.shape[:2]
    d = dev(img)
    cond = empty(w * h, torch().int16)
    marg = empty(h, torch().int16)
    integ = empty(1, torch().float32)
    for _ in range(3):
        assert lib.rb_envmap_cdf(w, h, ptr(d), 0, ptr(a[3]), ptr(cond), ptr(marg), ptr(integ), None) == 0
    assert np.array_equal(host(cond).view(np.uint16).reshape(h, w), a[0])
    assert np.array_equal(host(marg).view(np.uint16), a[1])


def test_scratch_contents_on_entry_do_not_matter():
    """Scratch straight from an allocator holds anything: 0xFF bytes in the
    completion counter must not stop the marginal from being built."""
    img = _sky(512, 256, seed=9)
    want_c, want_m, want_i, _ = ours(img, 0)
    lib = load()
    h, w = img.shape[:2]
    d = dev(img)
    scratch = torch().full((int(lib.rb_envmap_cdf_scratch_bytes(w, h)),), 0xFF, dtype=torch().uint8, device="cuda")
    cond = empty(w * h, torch().int16)
    marg = empty(h, torch().int16)
    integ = empty(1, torch().float32)
    assert lib.rb_envmap_cdf(w, h, ptr(d), 0, ptr(scratch), ptr(cond), ptr(marg), ptr(integ), None) == 0
    assert np.array_equal(host(cond).view(np.uint16).reshape(h, w), want_c)
    assert np.array_equal(host(marg).view(np.uint16), want_m)
    assert float(host(integ)[0]) == want_i


def test_rejects_bad_sizes():
    lib = load()
    x = empty(64, torch().uint8)
    assert lib.rb_envmap_cdf(6, 8, ptr(x), 0, ptr(x), ptr(x), ptr(x), ptr(x), None) != 0
    assert lib.rb_envmap_cdf(8, 8, ptr(x), 2, ptr(x), ptr(x), ptr(x), ptr(x), None) != 0
