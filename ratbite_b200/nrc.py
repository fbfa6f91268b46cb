"""Python handle of the neural radiance cache (include/ratbite_b200_nrc.h)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from ._native import check, load


class RadianceCache:
    """Hash-grid + 4 x 64 MLP radiance cache on the GPU. Inputs and outputs
    of infer/train are device pointers (e.g. torch tensors' data_ptr())."""

    def __init__(self, device: int = 0, seed: int = 1, learning_rate: float = 1e-2):
        self.lib = load()
        cfg = abi.rb_nrc_config()
        cfg.device, cfg.seed, cfg.learning_rate = device, seed, learning_rate
        h = C.c_void_p()
        check(self.lib.rb_nrc_create(C.byref(cfg), C.byref(h)), None, "rb_nrc_create")
        self.h = h
        self.grid_size = int(self.lib.rb_nrc_grid_size())
        self.weight_count = int(self.lib.rb_nrc_weight_count())

    def close(self):
        if self.h:
            self.lib.rb_nrc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def parameters(self):
        g = np.zeros(self.grid_size, np.float32)
        w = np.zeros(self.weight_count, np.float32)
        check(self.lib.rb_nrc_get_parameters(self.h, g.ctypes.data, w.ctypes.data), None, "rb_nrc_get_parameters")
        return g, w

    def set_parameters(self, grid, weights):
        g = np.ascontiguousarray(grid, np.float32)
        w = np.ascontiguousarray(weights, np.float32)
        check(self.lib.rb_nrc_set_parameters(self.h, g.ctypes.data, w.ctypes.data), None, "rb_nrc_set_parameters")

    def infer(self, n: int, inputs_ptr: int, outputs_ptr: int, stream=None):
        s = None if stream is None else C.c_void_p(stream)
        check(self.lib.rb_nrc_infer(self.h, n, C.c_void_p(inputs_ptr), C.c_void_p(outputs_ptr), s), None,
              "rb_nrc_infer")

    def train(self, n: int, inputs_ptr: int, targets_ptr: int, loss_ptr: int | None = None, stream=None):
        s = None if stream is None else C.c_void_p(stream)
        check(self.lib.rb_nrc_train(self.h, n, C.c_void_p(inputs_ptr), C.c_void_p(targets_ptr),
                                    None if loss_ptr is None else C.c_void_p(loss_ptr), s), None, "rb_nrc_train")

    def status(self) -> int:
        """RB_DEV_* bits raised by the network's kernels (synchronizes)."""
        f = C.c_uint32()
        check(self.lib.rb_nrc_status(self.h, C.byref(f)), None, "rb_nrc_status")
        return int(f.value)

    def gradients(self, n: int, inputs_ptr: int, targets_ptr: int):
        """(grid gradient, weight gradient) of the batch's mean loss, host arrays."""
        g = np.zeros(self.grid_size, np.float32)
        w = np.zeros(self.weight_count, np.float32)
        check(self.lib.rb_nrc_gradients(self.h, n, C.c_void_p(inputs_ptr), C.c_void_p(targets_ptr), g.ctypes.data,
                                         w.ctypes.data), None, "rb_nrc_gradients")
        return g, w
