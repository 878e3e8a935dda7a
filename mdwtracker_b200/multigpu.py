"""Multi-GPU frames: one process per GPU renders a band of image rows, and the bands are
gathered with torch.distributed (NCCL between GPUs, gloo on CPU).

Pixels are independent in the tracker (every path-sample depends only on its pixel,
sample index and frame id, deviceCode.cu:293-298), so disjoint row bands rendered by
N contexts assemble exactly into the frame one context renders: the gather is the only
exchange.  Every rank renders every frame (the frame and accumulation ids advance on
all ranks alike) and holds the whole assembled frame after `gather_*`.
"""
from __future__ import annotations

from typing import Optional, Tuple

import numpy as np


def band(height: int, world: int, rank: int) -> Tuple[int, int]:
    """Rows [lo, hi) of rank `rank`: contiguous, sizes differ by at most one row."""
    base, rem = divmod(height, world)
    lo = rank * base + min(rank, rem)
    return lo, lo + base + (1 if rank < rem else 0)


class BandRenderer:
    """Wraps a Renderer (libmdwt) or an OracleRenderer; renders this rank's band."""

    def __init__(self, renderer, group=None):
        import torch.distributed as dist
        self.r = renderer
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.height = renderer.fbSize[1]
        self.width = renderer.fbSize[0]
        self.lo, self.hi = band(self.height, self.world, self.rank)

    def render(self, stream: Optional[int] = None):
        self.r.setRenderRows(self.lo, self.hi)
        self.r.Render(stream) if stream else self.r.Render()

    def _gather_rows(self, local, channels: int, dtype):
        import torch
        import torch.distributed as dist
        rows = max(band(self.height, self.world, k)[1] - band(self.height, self.world, k)[0] for k in range(self.world))
        pad = torch.zeros((rows, self.width, channels), dtype=dtype, device=local.device)
        pad[: self.hi - self.lo] = local
        parts = [torch.empty_like(pad) for _ in range(self.world)]
        dist.all_gather(parts, pad, group=self.group)
        out = [parts[k][: band(self.height, self.world, k)[1] - band(self.height, self.world, k)[0]]
               for k in range(self.world)]
        return torch.cat(out, dim=0)

    def gather_accum(self):
        """The whole accumulation buffer (H, W, 4) float32, on every rank."""
        import torch
        n = self.hi - self.lo
        if self._on_gpu():
            local = torch.empty((n, self.width, 4), dtype=torch.float32, device="cuda")
            self.r.copyFrameRows(self.lo, self.hi, local.data_ptr() if n else None, None)
            self.r.sync()
        else:
            local = torch.from_numpy(np.ascontiguousarray(self.r.accum()[self.lo:self.hi]))
        return self._gather_rows(local, 4, torch.float32)

    def gather_framebuffer(self):
        """The whole RGBA8 framebuffer (H, W) uint32 as int32 bits, on every rank."""
        import torch
        n = self.hi - self.lo
        if self._on_gpu():
            local = torch.empty((n, self.width, 1), dtype=torch.int32, device="cuda")
            self.r.copyFrameRows(self.lo, self.hi, None, local.data_ptr() if n else None)
            self.r.sync()
        else:
            local = torch.from_numpy(np.ascontiguousarray(self.r.framebuffer()[self.lo:self.hi]).view(np.int32))[..., None]
        return self._gather_rows(local, 1, torch.int32)[..., 0]

    def reduce_counters(self):
        """Frame counters summed over the ranks (samples, rejections, cells, paths)."""
        import torch
        import torch.distributed as dist
        c = torch.tensor(np.asarray(self.r.counters(), dtype=np.int64), device="cuda" if self._on_gpu() else "cpu")
        dist.all_reduce(c, group=self.group)
        return c.cpu().numpy()

    def _on_gpu(self) -> bool:
        import torch.distributed as dist
        return dist.get_backend(self.group) == "nccl"
