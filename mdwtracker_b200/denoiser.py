"""Python binding of the learned denoiser (include/mdwt_denoiser.h).

Buffers are device pointers (ints) or CUDA torch tensors on the denoiser's device:
features [n][h][w][16] float32 (the tracker's per-pixel features, Renderer.setFeatures),
targets and outputs [n][h][w][4] float32 RGBA.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from .renderer import MdwtError, load_library


def _ptr(x) -> C.c_void_p:
    if hasattr(x, "data_ptr"):
        if not x.is_cuda or not x.is_contiguous() or str(x.dtype) != "torch.float32":
            raise ValueError("denoiser buffers are contiguous float32 CUDA tensors")
        return C.c_void_p(x.data_ptr())
    return C.c_void_p(int(x))


class Denoiser:
    def __init__(self, device: int = 0, seed: int = 0, lib: Optional[C.CDLL] = None):
        self._lib = lib if lib is not None else load_library()
        self._lib.mdwt_denoiser_num_params.restype = C.c_int64
        self._lib.mdwt_denoiser_last_error.restype = C.c_char_p
        self._d = C.c_void_p()
        st = self._lib.mdwt_denoiser_create(C.byref(self._d), C.c_int(device), C.c_uint64(seed))
        if st != 0:
            raise MdwtError(st, "denoiser_create", f"device {device}")

    @staticmethod
    def numParams(lib: Optional[C.CDLL] = None) -> int:
        lib = lib if lib is not None else load_library()
        lib.mdwt_denoiser_num_params.restype = C.c_int64
        return int(lib.mdwt_denoiser_num_params())

    def _call(self, name: str, *args):
        st = getattr(self._lib, "mdwt_denoiser_" + name)(self._d, *args)
        if st != 0:
            raise MdwtError(st, "denoiser_" + name, (self._lib.mdwt_denoiser_last_error(self._d) or b"").decode())

    def close(self):
        if self._d:
            self._lib.mdwt_denoiser_destroy(self._d)
            self._d = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def setTensorCores(self, on, overlap: bool = True) -> None:
        """tcgen05 convolutions (default: two TMEM accumulators, a tile's epilogue
        overlapping the next tile's MMAs; `overlap=False`: one accumulator with the most
        rows per tile) or the mma.sync kernels."""
        self._call("set_tensor_cores", C.c_int((1 if overlap else 2) if on else 0))

    def autotune(self, features, n: int, h: int, w: int, backward: bool = False) -> None:
        """Time the candidate tensor-core tilings of every layer for this input shape."""
        self._call("autotune", _ptr(features), C.c_int(n), C.c_int(h), C.c_int(w), C.c_int(1 if backward else 0))

    def check(self) -> None:
        """Synchronise; raises when a tensor-core kernel's bounded wait gave up (reported
        once)."""
        self._call("check")

    def testStall(self, launches: int) -> None:
        """Test hook: the next `launches` tensor-core convolutions issue no operand loads,
        so their bounded waits give up and check() raises (no GPU fault involved)."""
        self._call("test_stall", C.c_int(launches))

    def params(self) -> np.ndarray:
        out = np.empty(self.numParams(self._lib), np.float32)
        self._call("get_params", out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def setParams(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.numParams(self._lib):
            raise ValueError(f"expected {self.numParams(self._lib)} parameters, got {p.size}")
        self._call("set_params", p.ctypes.data_as(C.POINTER(C.c_float)))

    def grads(self) -> np.ndarray:
        out = np.empty(self.numParams(self._lib), np.float32)
        self._call("get_grads", out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def infer(self, features, out, n: int, h: int, w: int, stream: int = 0) -> None:
        self._call("infer", _ptr(features), _ptr(out), C.c_int(n), C.c_int(h), C.c_int(w), C.c_void_p(stream or None))

    def backward(self, features, target, n: int, h: int, w: int, stream: int = 0) -> float:
        loss = C.c_double()
        self._call("backward", _ptr(features), _ptr(target), C.c_int(n), C.c_int(h), C.c_int(w), C.byref(loss),
                   C.c_void_p(stream or None))
        return loss.value

    def _grad_buffer(self, x):
        if hasattr(x, "numel") and x.numel() != self.numParams(self._lib):
            raise ValueError(f"expected {self.numParams(self._lib)} gradient entries, got {x.numel()}")
        return _ptr(x)

    def copyGrads(self, out, stream: int = 0) -> None:
        """The gradient buffer into `out` (a float32 CUDA tensor of numParams entries, in
        params() order), asynchronously on `stream`."""
        self._call("copy_grads", self._grad_buffer(out), C.c_void_p(stream or None))

    def loadGrads(self, src, stream: int = 0) -> None:
        """Replace the gradient buffer by `src` (as copyGrads lays it out), on `stream`."""
        self._call("load_grads", self._grad_buffer(src), C.c_void_p(stream or None))

    def adamStep(self, lr: float, stream: int = 0) -> None:
        """One Adam step from the current gradient buffer (the update of trainStep)."""
        self._call("adam_step", C.c_float(lr), C.c_void_p(stream or None))

    def trainStep(self, features, target, n: int, h: int, w: int, lr: float, stream: int = 0,
                  want_loss: bool = True) -> Optional[float]:
        loss = C.c_double()
        self._call("train_step", _ptr(features), _ptr(target), C.c_int(n), C.c_int(h), C.c_int(w), C.c_float(lr),
                   C.byref(loss) if want_loss else None, C.c_void_p(stream or None))
        return loss.value if want_loss else None

    def save(self, path: str) -> None:
        np.save(path, self.params())

    def load(self, path: str) -> None:
        self.setParams(np.load(path))

