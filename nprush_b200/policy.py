"""Learned ADC policy: the 16 -> 64 -> 64 -> 3 MLP over libnprush_cuda.

The network maps a Gaussian's 16-float ADC feature vector to logits for
(clone, split, prune) against a fixed 0 logit for keep.  Inference, the
training forward / backward and the Adam updates run in the library
(tensor-core kernels, bf16 operands, fp32 accumulation); this class holds the
handle and moves parameters and samples.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import call

FEATURES = 16
CLASSES = ("keep", "clone", "split", "prune")


class AdcPolicy:
    def __init__(self, device: int = 0, seed: int | None = 0, params=None):
        self._ctx = _lib.context(device)
        self.device = device
        h = ctypes.c_void_p()
        call("nps_mlp_create", self._ctx, ctypes.byref(h))
        self._h = h.value
        self.num_params = _lib.load().nps_mlp_num_params()
        if params is not None:
            self.set_params(params)
        elif seed is not None:
            call("nps_mlp_init", self._h, int(seed))

    def set_params(self, params):
        p = np.ascontiguousarray(params, np.float32).reshape(-1)
        assert p.size == self.num_params
        call("nps_mlp_set_params", self._h, p.ctypes.data)

    def params(self) -> np.ndarray:
        p = np.empty(self.num_params, np.float32)
        call("nps_mlp_get_params", self._h, p.ctypes.data)
        return p

    @staticmethod
    def _dev(a, dtype):
        import torch
        t = a if isinstance(a, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(a))
        t = t.to(device="cuda", dtype=dtype).contiguous()
        torch.cuda.current_stream().synchronize()
        return t

    def logits(self, features):
        """features [n, 16] (numpy or torch) -> logits [n, 3] torch CUDA."""
        import torch
        x = self._dev(features, torch.float32)
        out = torch.empty((x.shape[0], 3), device=x.device, dtype=torch.float32)
        call("nps_mlp_forward", self._h, x.data_ptr(), x.shape[0], out.data_ptr())
        return out

    def grads(self, features, labels, class_w=None):
        import torch
        x = self._dev(features, torch.float32)
        y = self._dev(labels, torch.uint8)
        g = np.empty(self.num_params, np.float32)
        loss = np.zeros(1, np.float32)
        cw = None if class_w is None else np.ascontiguousarray(class_w, np.float32)
        call("nps_mlp_grads", self._h, x.data_ptr(), y.data_ptr(), x.shape[0],
             None if cw is None else cw.ctypes.data, g.ctypes.data, loss.ctypes.data)
        return g, float(loss[0])

    def train(self, features, labels, epochs: int = 10, batch: int = 8192, lr: float = 1e-3, seed: int = 0,
              class_w=None):
        """Returns (per-epoch loss, per-epoch accuracy)."""
        import torch
        x = self._dev(features, torch.float32)
        y = self._dev(labels, torch.uint8)
        lc = np.zeros(epochs, np.float32)
        ac = np.zeros(epochs, np.float32)
        cw = None if class_w is None else np.ascontiguousarray(class_w, np.float32)
        call("nps_mlp_train", self._h, x.data_ptr(), y.data_ptr(), x.shape[0], None if cw is None else cw.ctypes.data,
             epochs, batch, float(lr), int(seed), lc.ctypes.data, ac.ctypes.data)
        return lc, ac

    def close(self):
        if getattr(self, "_h", None):
            call("nps_mlp_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
