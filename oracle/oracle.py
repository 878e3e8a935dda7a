"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker for libmdwt.so.  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may import this module.

The oracle exposes the renderer entry points of include/mdwt.h with the ``orc_``
prefix, so :class:`OracleRenderer` reuses the product's Python mirror of the reference
``dtracker::Renderer`` API and a test script drives both the same way.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from mdwtracker_b200.renderer import Renderer, MdwtError

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")

_lib = None


def build_oracle(force: bool = False) -> str:
    if force or not os.path.exists(ORACLE_LIB):
        subprocess.run(["make", "-C", HERE], check=True, stdout=subprocess.DEVNULL)
    return ORACLE_LIB


def load_oracle() -> C.CDLL:
    global _lib
    if _lib is None:
        build_oracle()
        _lib = C.CDLL(ORACLE_LIB)
        _lib.orc_log.restype = C.c_float
        _lib.orc_log.argtypes = [C.c_float]
        _lib.orc_capped_samples.restype = C.c_uint64
        _lib.orc_rng_stream.argtypes = [C.c_uint32, C.c_uint32, C.c_int, C.POINTER(C.c_float)]
    return _lib


def set_threads(n: int) -> int:
    return load_oracle().orc_set_threads(C.c_int(n))


def oracle_log(x: float) -> float:
    return load_oracle().orc_log(C.c_float(x))


def rng_stream(v0: int, v1: int, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.float32)
    load_oracle().orc_rng_stream(C.c_uint32(v0), C.c_uint32(v1), C.c_int(n),
                                 out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


class OracleRenderer(Renderer):
    """The reference renderer restated on the CPU (OpenMP)."""

    _prefix = "orc_"

    def __init__(self):
        super().__init__(device=0, lib=load_oracle())

    def _create(self, device: int):
        st = self._lib.orc_create(C.byref(self._ctx))
        if st != 0:
            raise MdwtError(st, "orc_create")

    def renderRows(self, row0: int, row1: int):
        """One frame restricted to pixel rows [row0, row1) (frame ids still advance)."""
        self._call("render_rows", C.c_int(row0), C.c_int(row1))

    def renderRowStride(self, row0: int, stride: int) -> int:
        """One frame over the rows row0, row0 + stride, ... of the frame (frame ids still
        advance); returns how many rows were rendered."""
        self._call("render_row_stride", C.c_int(row0), C.c_int(stride))
        return (self.fbSize[1] - 1 - row0) // stride + 1

    _band = (0, 0)

    def setRenderRows(self, row0: int, row1: int):
        self._band = (row0, row1)

    def Render(self, stream=None):
        self.renderRows(*self._band)

    def RenderFrames(self, n: int, stream=None):
        for _ in range(n):
            self.Render()

    _expected = None

    def renderExpected(self, jitter: int = 4, stepVoxels: float = 0.5, stream=None):
        w, h = self.fbSize
        out = np.empty(w * h * 3, dtype=np.float64)
        self._call("expected_image", C.c_int(jitter), C.c_double(stepVoxels),
                   out.ctypes.data_as(C.POINTER(C.c_double)))
        self._expected = out.reshape(h, w, 3)

    def expectedImage(self, jitter: int = 4, stepVoxels: float = 0.5) -> np.ndarray:
        self.renderExpected(jitter, stepVoxels)
        return self._expected.copy()

    def accumRmse(self) -> float:
        if self._expected is None:
            raise MdwtError(6, "renderExpected first")
        d = self.accum()[..., :3].astype(np.float64) - self._expected
        return float(np.sqrt(np.mean(d * d)))

    def cappedSamples(self) -> int:
        return int(self._lib.orc_capped_samples(self._ctx))
