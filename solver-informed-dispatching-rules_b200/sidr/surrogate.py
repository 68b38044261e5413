"""Python front end of the surrogate model (include/sidr_surrogate.h): the
tensor-core GEMM and the 40 -> 256 -> 256 -> 1 MLP trained with Adam on the
device."""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _check, load

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_u16 = C.POINTER(C.c_uint16)

INPUTS, HIDDEN = 40, 256
PARAM_NAMES = ["W1", "b1", "W2", "b2", "w3", "b3"]
PARAM_SHAPES = {"W1": (HIDDEN, 48), "b1": (HIDDEN,), "W2": (HIDDEN, HIDDEN), "b2": (HIDDEN,),
                "w3": (HIDDEN,), "b3": (1,)}


def _lib():
    L = load()
    if not getattr(L, "_surrogate_ready", False):
        L.sidr_gemm_bf16.argtypes = [_u16, _u16, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int,
                                     _fp]
        L.sidr_mlp_create.argtypes = [C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]
        L.sidr_mlp_destroy.argtypes = [C.c_void_p]
        L.sidr_mlp_param.argtypes = [C.c_void_p, C.c_int32, C.c_int32, _fp, _fp, C.POINTER(C.c_int64)]
        L.sidr_mlp_predict.argtypes = [C.c_void_p, _fp, C.c_int32, _fp]
        L.sidr_mlp_gradients.argtypes = [C.c_void_p, _fp, _fp, C.c_int32, _fp]
        L.sidr_mlp_train.argtypes = [C.c_void_p, _fp, _fp, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                     C.c_uint64, _fp]
        L._surrogate_ready = True
    return L


def to_bf16_bits(x) -> np.ndarray:
    """Round-to-nearest-even FP32 -> BF16, as 16-bit patterns."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return r.astype(np.uint16)


def from_bf16_bits(b) -> np.ndarray:
    return (np.asarray(b, dtype=np.uint32) << 16).view(np.float32)


def gemm_bf16(A_bits, B_bits, splits: int = 1, device: int = 0) -> np.ndarray:
    """C = A B^T on the tensor-core kernel; A [M x K], B [N x K] BF16 bits."""
    A = np.ascontiguousarray(A_bits, dtype=np.uint16)
    B = np.ascontiguousarray(B_bits, dtype=np.uint16)
    M, K = A.shape
    N = B.shape[0]
    out = np.zeros((M, N), np.float32)
    _check(_lib().sidr_gemm_bf16(A.ctypes.data_as(_u16), B.ctypes.data_as(_u16), M, N, K, splits,
                                 device, out.ctypes.data_as(_fp)))
    return out


class MLP:
    def __init__(self, seed: int = 0, device: int = 0):
        h = C.c_void_p()
        _check(_lib().sidr_mlp_create(device, seed, C.byref(h)))
        self.h = h.value

    def param(self, name: str):
        L = _lib()
        i = PARAM_NAMES.index(name)
        v = np.zeros(PARAM_SHAPES[name], np.float32)
        g = np.zeros(PARAM_SHAPES[name], np.float32)
        n = C.c_int64()
        _check(L.sidr_mlp_param(self.h, i, 0, v.ctypes.data_as(_fp), g.ctypes.data_as(_fp),
                                C.byref(n)))
        return v, g

    def set_param(self, name: str, values) -> None:
        v = np.ascontiguousarray(values, dtype=np.float32).reshape(PARAM_SHAPES[name])
        _check(_lib().sidr_mlp_param(self.h, PARAM_NAMES.index(name), 1, v.ctypes.data_as(_fp), None,
                                     None))

    def predict(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros(x.shape[0], np.float32)
        _check(_lib().sidr_mlp_predict(self.h, x.ctypes.data_as(_fp), x.shape[0],
                                       y.ctypes.data_as(_fp)))
        return y

    def gradients(self, x, t) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = C.c_float()
        _check(_lib().sidr_mlp_gradients(self.h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp),
                                         x.shape[0], C.byref(loss)))
        return loss.value

    def train(self, x, t, steps: int, batch: int = 1024, lr: float = 1e-3, seed: int = 0) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = C.c_float()
        _check(_lib().sidr_mlp_train(self.h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp),
                                     x.shape[0], steps, batch, lr, seed, C.byref(loss)))
        return loss.value

    def close(self):
        if getattr(self, "h", None):
            _lib().sidr_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
