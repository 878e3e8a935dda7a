"""Python binding of batched rendering and the autotuner (include/mdwt_batch.h)."""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

from .renderer import MdwtError, load_library


class Batch:
    """Renders one frame of every added request (a set-up :class:`Renderer`) per call,
    with one persistent tracker launch per kernel variant, optionally as a CUDA graph."""

    def __init__(self, device: int = 0, lib: Optional[C.CDLL] = None):
        self._lib = lib if lib is not None else load_library()
        self._lib.mdwt_batch_last_error.restype = C.c_char_p
        self._b = C.c_void_p()
        self._reqs = []
        st = self._lib.mdwt_batch_create(C.byref(self._b), C.c_int(device))
        if st != 0:
            raise MdwtError(st, "batch_create", f"device {device}")

    def _call(self, name: str, *args):
        st = getattr(self._lib, "mdwt_batch_" + name)(self._b, *args)
        if st != 0:
            raise MdwtError(st, "batch_" + name, (self._lib.mdwt_batch_last_error(self._b) or b"").decode())

    def close(self):
        if self._b:
            self._lib.mdwt_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, renderer) -> None:
        self._call("add", renderer._ctx)
        self._reqs.append(renderer)   # keep the request alive while batched

    def clear(self) -> None:
        self._call("clear")
        self._reqs = []

    def render(self, stream: int = 0) -> None:
        self._call("render", C.c_void_p(stream or None))

    def sync(self) -> None:
        self._call("sync")

    def setSchedule(self, unit_items: int = 0, pool: int = 0, trips: int = 0) -> None:
        self._call("set_schedule", C.c_int(unit_items), C.c_int(pool), C.c_int(trips))

    def setGraph(self, enable: bool) -> None:
        self._call("set_graph", C.c_int(1 if enable else 0))

    def setFusion(self, enable: bool) -> None:
        """Regroupable requests in one shared launch (default) or one launch per variant."""
        self._call("set_fusion", C.c_int(1 if enable else 0))

    def traceLaunches(self) -> int:
        """Trace-kernel launches of the last batch frame."""
        out = (C.c_int * 2)()
        self._call("fusion_info", out)
        return int(out[0])

    def lastMs(self) -> float:
        v = C.c_float()
        self._call("last_ms", C.byref(v))
        return v.value

    def info(self) -> dict:
        out = (C.c_int64 * 8)()
        self._call("info", out)
        keys = ["launches", "groups", "requests", "graph_replays", "graph_captures", "chunk_items", "pool", "trips"]
        return dict(zip(keys, [int(x) for x in out]))

    def autotune(self, frames: int = 2):
        best = (C.c_int * 3)()
        self._call("autotune", C.c_int(frames), best)
        return tuple(best)


def autotune_macrocells(renderer, edges: Sequence[int] = (4, 8, 16, 32), frames: int = 2) -> int:
    lib = renderer._lib
    arr = (C.c_int * len(edges))(*[int(e) for e in edges])
    best = C.c_int()
    renderer._call("autotune_macrocells", arr, C.c_int(len(edges)), C.c_int(frames), C.byref(best))
    return best.value
