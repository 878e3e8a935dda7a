"""Multi-GPU frames and denoiser training over torch.distributed (NCCL between GPUs, gloo on
CPU).

Frames: one process per GPU renders a band of image rows, and the bands are gathered.

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


class DataParallelTrainer:
    """Data-parallel training of the learned denoiser, one process per GPU.

    Every rank runs the backward pass on its shard of each minibatch.  One all-reduce
    averages the gradient vector (470,640 floats for the committed network) over the ranks,
    and every rank applies the same Adam step, so the parameters stay identical
    everywhere.  With equal shard sizes the averaged gradient is the full minibatch's,
    because the loss is a mean over the shard.  `denoiser` is a Denoiser, or any object
    with its params / backward / copyGrads / loadGrads / adamStep calls."""

    def __init__(self, denoiser, group=None):
        import torch
        import torch.distributed as dist
        self.d = denoiser
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        p = np.asarray(denoiser.params())
        dev = "cuda" if dist.is_initialized() and dist.get_backend(group) == "nccl" else getattr(denoiser, "device", "cuda")
        self.g = torch.empty(p.size, dtype=torch.float32 if p.dtype == np.float32 else torch.float64, device=dev)

    def step(self, features, target, n: int, h: int, w: int, lr: float, stream: int = 0) -> float:
        """One training step on this rank's shard [n][h][w]; returns the loss averaged over
        the ranks."""
        import torch
        import torch.distributed as dist
        loss = self.d.backward(features, target, n, h, w, stream)
        if self.world > 1:
            self.d.copyGrads(self.g, stream)
            if self.g.is_cuda:
                torch.cuda.synchronize(self.g.device)   # the copy on `stream` before the collective
            dist.all_reduce(self.g, group=self.group)
            self.g /= self.world
            if self.g.is_cuda:
                torch.cuda.synchronize(self.g.device)   # the collective before the library reads it
            self.d.loadGrads(self.g, stream)
            t = torch.tensor([loss], dtype=torch.float64, device=self.g.device)
            dist.all_reduce(t, group=self.group)
            loss = float(t.item()) / self.world
        self.d.adamStep(lr, stream)
        return loss
