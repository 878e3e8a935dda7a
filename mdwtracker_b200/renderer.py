"""Python mirror of ``dtracker::Renderer`` (renderer.h:52-222) over the C ABI.

The methods keep the reference names and argument meanings (``PushMesh``, ``Init``,
``Render``, ``SetXFColormap``, ``SetXFOpacityScale``, ``SetXFRange``, ``Setdt``,
``Resetdt``, ``ResetAccumulation``, ``Resize``, ``UpdateCamera``...), so a script written
against the reference reads the same.  Two differences in error behaviour: a failing
call raises :class:`MdwtError` (the reference prints and returns, or calls ``exit``), and
member writes (``spp``, ``enableAccumulation``...) take effect at once instead of at
the next ``Update()``.

The binding is generic over a ctypes library and a symbol prefix so that the CPU
oracle, which exposes the same entry points with the ``orc_`` prefix, can be driven by
the very same test scripts; the product library is ``libmdwt.so`` with ``mdwt_``.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmdwt.so")

STATUS = {
    0: "ok", 1: "bad argument", 2: "CUDA error", 3: "I/O error", 4: "too many channels",
    5: "unsupported", 6: "wrong call order", 7: "out of memory", 8: "device wait timed out",
    9: "bad raw file name", 10: "sample step cap reached", 11: "scratch limit of a no-alloc entry point",
}
MDWT_HOST_ONLY = -1

# raw::DataFormat numbering (rawFile.h:21-35)
FORMATS = {
    np.dtype(np.int8): 1, np.dtype(np.int16): 2, np.dtype(np.int32): 3, np.dtype(np.uint8): 4,
    np.dtype(np.uint16): 5, np.dtype(np.uint32): 6, np.dtype(np.float32): 7, np.dtype(np.float64): 8,
}


class MdwtError(RuntimeError):
    def __init__(self, status: int, where: str, message: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS.get(status, status)} ({message})")


_lib_cache = {}


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load libmdwt.so.  There is no fallback: a missing library is an error."""
    if path in _lib_cache:
        return _lib_cache[path]
    if not os.path.exists(path):
        raise ImportError(f"{path} is not built; run `make -C mdwtracker_b200` or __graft_entry__.build()")
    lib = C.CDLL(path)
    _lib_cache[path] = lib
    return lib


def _f3(v) -> C.Array:
    return (C.c_float * 3)(*[float(x) for x in v])


class Renderer:
    """Headless renderer on one device (``device=MDWT_HOST_ONLY`` for a host-only context)."""

    _prefix = "mdwt_"

    def __init__(self, device: int = 0, lib: Optional[C.CDLL] = None):
        self._lib = lib if lib is not None else load_library()
        self._ctx = C.c_void_p()
        self._create(device)
        self.fbSize = (1024, 1024)
        self.mode = None

    # ---------------------------------------------------------------- plumbing
    def _fn(self, name: str):
        return getattr(self._lib, self._prefix + name)

    def _create(self, device: int):
        st = self._fn("create")(C.byref(self._ctx), C.c_int(device))
        if st != 0:
            raise MdwtError(st, "create", f"device {device}")

    def _call(self, name: str, *args):
        st = self._fn(name)(self._ctx, *args)
        if st != 0:
            err = self._fn("last_error")
            err.restype = C.c_char_p
            raise MdwtError(st, name, (err(self._ctx) or b"").decode())
        return st

    def close(self):
        if self._ctx:
            self._fn("destroy")(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---------------------------------------------------------------- data
    def PushMesh(self, data, dims: Optional[Sequence[int]] = None) -> bool:
        """PushMesh(shared_ptr<RawR>) (renderer.cpp:1031-1044).

        ``data`` is a raw-file path (parsed like raw::RawR) or a numpy array of shape
        (Z, Y, X) (x fastest, as in the raw files)."""
        if isinstance(data, (str, os.PathLike)):
            self._call("push_channel_raw", C.c_char_p(os.fsencode(data)))
            return True
        arr = np.ascontiguousarray(data)
        if arr.dtype not in FORMATS:
            raise MdwtError(5, "push_channel", f"dtype {arr.dtype}")
        if dims is None:
            if arr.ndim != 3:
                raise MdwtError(1, "push_channel", "need a (Z, Y, X) array or explicit dims")
            dims = (arr.shape[2], arr.shape[1], arr.shape[0])
        d = (C.c_int64 * 3)(*[int(x) for x in dims])
        self._call("push_channel", arr.ctypes.data_as(C.c_void_p), C.c_int(FORMATS[arr.dtype]), d)
        return True

    def reshapeBounds(self, channel: int, scale: Optional[Sequence[float]] = None):
        """raw::RawR::reshapeBounds (rawFile.cpp:217-237), viewer ``-cb``."""
        self._call("reshape_bounds", C.c_int(channel), _f3(scale) if scale is not None else None)

    @property
    def numChannels(self) -> int:
        n = C.c_int()
        self._call("num_channels", C.byref(n))
        return n.value

    def channelInfo(self, channel: int):
        dims = (C.c_int64 * 3)()
        b = (C.c_float * 8)()
        self._call("get_channel_info", C.c_int(channel), dims, b)
        return tuple(dims), np.array(b[:], dtype=np.float32)

    # ---------------------------------------------------------------- set-up
    @property
    def macrocellDims(self):
        d = (C.c_uint32 * 3)()
        self._call("get_macrocell_dims", d)
        return tuple(d)

    @macrocellDims.setter
    def macrocellDims(self, dims):
        if isinstance(dims, int):
            dims = (dims, dims, dims)
        self._call("set_macrocells", (C.c_uint32 * 3)(*[int(x) for x in dims]))

    def Init(self, mode: int = 0, autoSetCamera: bool = True):
        """Renderer::Init (renderer.cpp:324-942)."""
        self._call("init", C.c_int(mode), C.c_int(1 if autoSetCamera else 0))
        self.mode = mode

    # ---------------------------------------------------------------- TF
    def SetXFColormap(self, colormap, tfID: int = 0):
        cm = np.ascontiguousarray(np.asarray(colormap, dtype=np.float32).reshape(-1, 4))
        self._call("set_tf", C.c_int(tfID), cm.ctypes.data_as(C.POINTER(C.c_float)), C.c_int(cm.shape[0]))

    def SetXFOpacityScale(self, opacityScale: float, tfID: int = 0):
        self._call("set_opacity_scale", C.c_int(tfID), C.c_float(opacityScale))

    def SetXFRange(self, xfDomain, tfID: int = 0):
        self._call("set_tf_range", C.c_int(tfID), C.c_float(xfDomain[0]), C.c_float(xfDomain[1]))

    def RecalculateDensityRanges(self):
        self._call("recalculate_majorants")

    # ---------------------------------------------------------------- parameters
    def Setdt(self, dt: float):
        self._call("set_dt", C.c_float(dt))

    def Resetdt(self):
        self._call("reset_dt")

    @property
    def dt(self) -> float:
        v = C.c_float()
        self._call("get_dt", C.byref(v))
        return v.value

    def setCamera(self, lookFrom, lookAt, lookUp, fovy: float):
        """camera.setOrientation + UpdateCamera (viewer ``-c``)."""
        self._call("set_camera", _f3(lookFrom), _f3(lookAt), _f3(lookUp), C.c_float(fovy))

    def cameraBasis(self) -> np.ndarray:
        out = (C.c_float * 12)()
        self._call("get_camera_basis", out)
        return np.array(out[:], dtype=np.float32).reshape(4, 3)

    def Resize(self, newSize):
        self._call("resize", C.c_int(int(newSize[0])), C.c_int(int(newSize[1])))
        self.fbSize = (int(newSize[0]), int(newSize[1]))

    def setSpp(self, spp: int):
        self._call("set_spp", C.c_int(spp))

    def setAccumulation(self, enable: bool):
        self._call("set_accumulation", C.c_int(1 if enable else 0))

    def setBackground(self, rgb):
        self._call("set_background", _f3(rgb))

    def setLight(self, shadows: bool, gradient: bool, direction, intensity: float = 1.0, ambient: float = 0.1):
        self._call("set_light", C.c_int(int(shadows)), C.c_int(int(gradient)), _f3(direction),
                   C.c_float(intensity), C.c_float(ambient))

    def setMaterial(self, channel: int, diffuse=0.8, specular=0.3, shininess=8.0, gradientStep=0.01,
                    specularColor=(1.0, 1.0, 1.0)):
        self._call("set_material", C.c_int(channel), C.c_float(diffuse), C.c_float(specular),
                   C.c_float(shininess), C.c_float(gradientStep), _f3(specularColor))

    def setMirror(self, enable: bool):
        self._call("set_mirror", C.c_int(1 if enable else 0))

    def setSeedBlock(self, edge: int):
        """Seed the generator from the pixel (0) or from its position in an edge x edge
        thread block, the reference's threadIdx under such a launch (deviceCode.cu:297)."""
        self._call("set_seed_block", C.c_int(edge))

    def setArithmetic(self, fast: bool):
        """Free-flight arithmetic: exact (the default, bit-identical to the CPU oracle) or
        fast (hardware log2 flight lengths; per-pixel events match the oracle on at least
        99.9 % of pixels).  After Init the majorant table is rebuilt."""
        self._call("set_arithmetic", C.c_int(int(fast)))

    def arithmetic(self) -> int:
        """0 = exact, 1 = fast."""
        v = C.c_int()
        self._call("get_arithmetic", C.byref(v))
        return v.value

    # ---------------------------------------------------------------- frames
    def Render(self, stream: Optional[int] = None):
        """Renderer::Render (renderer.cpp:944-973); asynchronous on ``stream``."""
        self._call("render", C.c_void_p(stream) if stream else None)

    def sync(self):
        self._call("sync")

    def ResetAccumulation(self):
        self._call("reset_accumulation")

    def autotuneSchedule(self, frames: int = 2):
        """Time `frames`-frame launches for each schedule candidate and keep the fastest:
        for -m 2 the tracker (regrouped or warp-local) first, then the trips, then the
        warp-local tracker's pool and quorum.  Frame ids and counters are restored and the
        accumulation reset.  Returns (pool, trips); getTuning(4) tells the tracker."""
        best = (C.c_int * 2)()
        self._call("autotune_schedule", C.c_int(frames), best)
        return tuple(best)

    def autotuneMacrocells(self, edges=(4, 8, 16, 32), frames: int = 2) -> int:
        """Time frames for each macrocell edge length (voxels per side), keep the fastest
        grid; frame ids are restored and the accumulation reset."""
        from .batch import autotune_macrocells
        return autotune_macrocells(self, edges, frames)

    def RenderFrames(self, n: int, stream: Optional[int] = None):
        """n successive frames (as n Render calls), traced in one launch where they fit."""
        self._call("render_frames", C.c_int(n), C.c_void_p(stream) if stream else None)

    def setFrameId(self, frame_id: int):
        """The next frame renders with frame id `frame_id` (the reference's public frameID)."""
        self._call("set_frame_id", C.c_int(frame_id))

    def frameIds(self):
        out = (C.c_int * 4)()
        self._call("get_frame_ids", out)
        return tuple(out)

    def framebuffer(self) -> np.ndarray:
        w, h = self.fbSize
        out = np.empty(w * h, dtype=np.uint32)
        self._call("get_framebuffer", out.ctypes.data_as(C.POINTER(C.c_uint32)))
        return out.reshape(h, w)

    def accum(self) -> np.ndarray:
        w, h = self.fbSize
        out = np.empty(w * h * 4, dtype=np.float32)
        self._call("get_accum", out.ctypes.data_as(C.POINTER(C.c_float)))
        return out.reshape(h, w, 4)

    def counters(self) -> np.ndarray:
        out = (C.c_uint64 * 4)()
        self._call("get_counters", out)
        return np.array(out[:], dtype=np.uint64)

    def resetCounters(self):
        self._call("reset_counters")

    def enablePixelStats(self, enable: bool = True):
        self._call("enable_pixel_stats", C.c_int(1 if enable else 0))

    def pixelStats(self) -> np.ndarray:
        w, h = self.fbSize
        out = np.empty(w * h * 4, dtype=np.uint32)
        self._call("get_pixel_stats", out.ctypes.data_as(C.POINTER(C.c_uint32)))
        return out.reshape(h, w, 4)

    # ---------------------------------------------------------------- majorants
    def _num_cells(self) -> int:
        d = self.macrocellDims
        return int(d[0]) * int(d[1]) * int(d[2])

    def majorants(self) -> np.ndarray:
        n = self._num_cells() * (1 if self.mode >= 3 else self.numChannels)
        out = np.empty(n, dtype=np.float32)
        self._call("get_majorants", out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def ranges(self) -> np.ndarray:
        n = self._num_cells() * self.numChannels
        out = np.empty(2 * n, dtype=np.float32)
        self._call("get_ranges", out.ctypes.data_as(C.POINTER(C.c_float)))
        return out.reshape(n, 2)

    # ---------------------------------------------------------------- denoiser features
    def setFeatures(self, enable: bool):
        """Write the 16 denoiser input features per pixel with every frame."""
        self._call("set_features", C.c_int(1 if enable else 0))

    def features(self) -> np.ndarray:
        """(H, W, 16) float32 features of the last frame."""
        w, h = self.fbSize
        out = np.empty(w * h * 16, dtype=np.float32)
        self._call("get_features", out.ctypes.data_as(C.POINTER(C.c_float)))
        return out.reshape(h, w, 16)

    def copyFeatures(self, dst, stream: int = 0):
        """Device-to-device copy of the last frame's features into `dst` (pointer or tensor)."""
        from .denoiser import _ptr
        self._call("copy_features", _ptr(dst), C.c_void_p(stream or None))

    def deviceFeatures(self) -> int:
        p = C.c_void_p()
        self._call("get_device_features", C.byref(p))
        return p.value or 0

    def denoise(self, denoiser, out) -> None:
        """Denoise the last frame's features into `out` ([H][W][4] float32 on the device)."""
        from .denoiser import _ptr
        self._call("denoise", denoiser._d, _ptr(out))

    def imageRmse(self, img) -> float:
        """RMSE of a device RGBA image [H][W][4] against the last expected image."""
        from .denoiser import _ptr
        out = C.c_double()
        self._call("image_rmse", _ptr(img), C.byref(out))
        return out.value

    # ---------------------------------------------------------------- FP64 ground truth
    def renderExpected(self, jitter: int = 4, stepVoxels: float = 0.5, stream: Optional[int] = None):
        """Compute the FP64 expected image of the unshaded estimator (asynchronous)."""
        self._call("render_expected", C.c_int(jitter), C.c_float(stepVoxels),
                   C.c_void_p(stream) if stream else None)

    def expectedImage(self, jitter: int = 4, stepVoxels: float = 0.5) -> np.ndarray:
        """(H, W, 3) float64 expected image (row 0 = framebuffer row 0)."""
        self.renderExpected(jitter, stepVoxels)
        w, h = self.fbSize
        out = np.empty(w * h * 3, dtype=np.float64)
        self._call("get_expected", out.ctypes.data_as(C.POINTER(C.c_double)))
        return out.reshape(h, w, 3)

    def accumRmse(self) -> float:
        """RMSE of the accumulation buffer's RGB against the last expected image."""
        out = C.c_double()
        self._call("accum_rmse", C.byref(out))
        return out.value

    def setRenderRows(self, row0: int, row1: int):
        """Render only rows [row0, row1) (row1 <= row0: all rows); ids advance per frame."""
        self._call("set_render_rows", C.c_int(row0), C.c_int(row1))

    def copyFrameRows(self, row0: int, row1: int, accum_ptr: Optional[int], fb_ptr: Optional[int],
                      stream: Optional[int] = None):
        """Copy rows [row0, row1) of the accumulation / RGBA8 buffers to raw (device or
        host) pointers."""
        self._call("copy_frame_rows", C.c_int(row0), C.c_int(row1), C.c_void_p(accum_ptr), C.c_void_p(fb_ptr),
                   C.c_void_p(stream) if stream else None)

    def loadFrameRows(self, row0: int, row1: int, accum_ptr: Optional[int], fb_ptr: Optional[int],
                      stream: Optional[int] = None):
        """Write rows [row0, row1) of the accumulation / RGBA8 buffers from raw (device or
        host) pointers: the inverse of copyFrameRows."""
        self._call("load_frame_rows", C.c_int(row0), C.c_int(row1), C.c_void_p(accum_ptr), C.c_void_p(fb_ptr),
                   C.c_void_p(stream) if stream else None)

    def setTiming(self, enable: bool = True):
        self._call("set_timing", C.c_int(1 if enable else 0))

    def kernelTimes(self):
        """(trace ms, resolve ms) of the last frame (timing on, one sample batch)."""
        out = (C.c_float * 2)()
        self._call("get_kernel_times", out)
        return float(out[0]), float(out[1])

    def setTuning(self, key: int, value: int):
        """Tracker tuning knob (0 pool, 1 batch, 2 trips, 3 quorum, 4 regroup); results do
        not depend on it."""
        self._call("set_tuning", C.c_int(key), C.c_int(value))

    def getTuning(self, key: int) -> int:
        v = C.c_int()
        self._call("get_tuning", C.c_int(key), C.byref(v))
        return v.value

    def renderInfo(self):
        """(kernels launched so far, per-frame parameter bytes, last grid, last block)."""
        out = (C.c_int64 * 4)()
        self._call("get_render_info", out)
        return tuple(out)

    def deviceBuffers(self):
        a, f = C.c_void_p(), C.c_void_p()
        self._call("get_device_buffers", C.byref(a), C.byref(f))
        return a.value, f.value
