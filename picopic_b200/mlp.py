"""The per-cell collision MLP (13 -> 128 -> 128 -> 6) on the tensor cores.

A thin host wrapper of the pcg_mlp_* C ABI: the network lives on the GPU,
its forward and backward passes and the Adam updates are the library's own
BF16/FP32 kernels.  Parameters are FP32, row-major [in][out] per layer, in
the order W1, b1, W2, b2, W3, b3.
"""
from __future__ import annotations

import ctypes

import numpy as np

from ._ffi import PcgError, load

INPUTS, HIDDEN, OUTPUTS = 13, 128, 6
SHAPES = [("w1", (INPUTS, HIDDEN)), ("b1", (HIDDEN,)), ("w2", (HIDDEN, HIDDEN)), ("b2", (HIDDEN,)),
          ("w3", (HIDDEN, OUTPUTS)), ("b3", (OUTPUTS,))]
PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)

_PF = ctypes.POINTER(ctypes.c_float)


def _fp(a):
    return a.ctypes.data_as(_PF)


def unpack(p: np.ndarray) -> dict:
    """Split a flat parameter vector into named arrays (views)."""
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    return out


class Mlp:
    def __init__(self, device: int = 0, seed: int = 0):
        self.lib = load()
        h = ctypes.c_void_p()
        rc = self.lib.pcg_mlp_create(int(device), int(seed), ctypes.byref(h))
        if rc != 0:
            raise PcgError(rc, "pcg_mlp_create", "")
        self.h = h

    def _check(self, rc, where):
        if rc != 0:
            raise PcgError(rc, where, "")

    def close(self):
        if getattr(self, "h", None):
            self.lib.pcg_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(PARAMS, dtype=np.float32)
        self._check(self.lib.pcg_mlp_get_params(self.h, _fp(p)), "pcg_mlp_get_params")
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != PARAMS:
            raise ValueError(f"{p.size} parameters, the network has {PARAMS}")
        self._check(self.lib.pcg_mlp_set_params(self.h, _fp(p)), "pcg_mlp_set_params")

    def forward(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((x.shape[0], OUTPUTS), dtype=np.float32)
        self._check(self.lib.pcg_mlp_forward(self.h, _fp(x), x.shape[0], _fp(y)), "pcg_mlp_forward")
        return y

    def forward_tc(self, x):
        """The forward pass on tcgen05 (pcg_mlp_forward_tc); returns (y, device ms)."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((x.shape[0], OUTPUTS), dtype=np.float32)
        ms = ctypes.c_float(0.0)
        self._check(self.lib.pcg_mlp_forward_tc(self.h, _fp(x), x.shape[0], _fp(y), ctypes.byref(ms)),
                    "pcg_mlp_forward_tc")
        return y, float(ms.value)

    def gradient(self, x, t):
        """Full-batch gradient and value of mean((y - t)^2)."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(PARAMS, dtype=np.float32)
        loss = ctypes.c_float()
        self._check(self.lib.pcg_mlp_gradient(self.h, _fp(x), _fp(t), x.shape[0], _fp(g), ctypes.byref(loss)),
                    "pcg_mlp_gradient")
        return g, float(loss.value)

    def set_data(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        self._check(self.lib.pcg_mlp_set_data(self.h, _fp(x), _fp(t), x.shape[0]), "pcg_mlp_set_data")

    def train(self, steps: int, batch: int = 4096, lr: float = 1e-3) -> float:
        loss = ctypes.c_float()
        self._check(self.lib.pcg_mlp_train(self.h, int(steps), int(batch), float(lr), ctypes.byref(loss)),
                    "pcg_mlp_train")
        return float(loss.value)
