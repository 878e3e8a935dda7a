"""Multi-GPU frames and denoiser training over torch.distributed (NCCL between GPUs, gloo on
CPU).

Frames: one process per GPU renders a band of image rows, and the bands are gathered.

Pixels are independent in the tracker (every path-sample depends only on its pixel,
sample index and frame id, deviceCode.cu:293-298), so disjoint row bands rendered by
N contexts assemble exactly into the frame one context renders: the gather is the only
exchange.  Every rank renders every frame (the frame and accumulation ids advance on
all ranks alike) and holds the whole assembled frame after `gather_*`.

The cost of a row is far from uniform: rows that miss the volume cost almost nothing
and rows through its thickest part the most.  Bands therefore start equal and are then
rebalanced from measured render times (`rebalance`): each rank's time is spread evenly
over its rows, giving a per-row cost estimate that every rank holds identically, and the
frame is re-split so that each band carries an equal share of the estimated cost.
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np


def band(height: int, world: int, rank: int) -> Tuple[int, int]:
    """Rows [lo, hi) of rank `rank`: contiguous, sizes differ by at most one row."""
    base, rem = divmod(height, world)
    lo = rank * base + min(rank, rem)
    return lo, lo + base + (1 if rank < rem else 0)


def split_by_cost(cost: Sequence[float], world: int, align: int = 4) -> List[Tuple[int, int]]:
    """Contiguous row bands [lo, hi), one per rank, covering all rows, each carrying about
    1/world of the total of the per-row `cost`; inner boundaries fall on multiples of
    `align` rows (the tracker's tile height), and no band is narrower than `align` rows
    when the frame has room for that (an empty band would mean "all rows" to
    mdwt_set_render_rows).  Deterministic: equal inputs give equal bands on every rank."""
    c = np.asarray(cost, dtype=np.float64)
    h = int(c.size)
    if h < world * align:
        return [band(h, world, k) for k in range(world)]
    cum = np.concatenate([[0.0], np.cumsum(np.maximum(c, 0.0))])
    total = cum[-1]
    bounds = [0]
    for k in range(1, world):
        if total > 0.0:
            y = int(np.searchsorted(cum, total * k / world, side="left"))
        else:
            y = band(h, world, k)[0]
        y = int(round(y / align)) * align
        y = max(y, bounds[-1] + align)              # at least `align` rows for band k - 1
        y = min(y, (h - (world - k) * align) // align * align)   # and room for the bands after it
        bounds.append(y)
    bounds.append(h)
    return [(bounds[k], bounds[k + 1]) for k in range(world)]


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
        self.bands = [band(self.height, self.world, k) for k in range(self.world)]
        self.cost = np.ones(self.height, dtype=np.float64)   # per-row cost estimate (uniform at first)
        self.lo, self.hi = self.bands[self.rank]

    def render(self, stream: Optional[int] = None):
        self.r.setRenderRows(self.lo, self.hi)
        self.r.Render(stream) if stream else self.r.Render()

    def rebalance(self, seconds: float) -> List[Tuple[int, int]]:
        """Re-split the frame from this rank's last render time (every rank calls this with
        its own time): the times are all-gathered, each spread evenly over its band's rows
        into the per-row cost estimate, and the bands re-cut at equal shares of it.  The
        next `render` uses the new band.  When the bands move, each rank takes over the
        accumulation buffer of the rows it gains (the running mean continues there: the
        whole buffer is all-gathered once and each rank loads its new rows).  Returns the
        bands."""
        import torch
        import torch.distributed as dist
        dev = "cuda" if self._on_gpu() else "cpu"
        t = torch.zeros(self.world, dtype=torch.float64, device=dev)
        t[self.rank] = float(seconds)
        dist.all_reduce(t, group=self.group)
        times = t.cpu().numpy()
        for k, (lo, hi) in enumerate(self.bands):
            if hi > lo:
                self.cost[lo:hi] = times[k] / (hi - lo)
        # rows never measured keep their old estimate; no row is free
        floor = 1e-3 * float(self.cost.mean()) if self.cost.mean() > 0 else 1.0
        self.cost = np.maximum(self.cost, floor)
        bands = split_by_cost(self.cost, self.world)
        if bands != self.bands:
            whole = self.gather_accum()   # the old bands' rows, on every rank
            lo, hi = bands[self.rank]
            if hi > lo:
                rows = whole[lo:hi].contiguous()
                self.r.loadFrameRows(lo, hi, rows.data_ptr(), None)
                if self._on_gpu():
                    self.r.sync()
            self.bands = bands
        self.lo, self.hi = self.bands[self.rank]
        return list(self.bands)

    def _gather_rows(self, local, channels: int, dtype):
        import torch
        import torch.distributed as dist
        rows = max(hi - lo for lo, hi in self.bands)
        pad = torch.zeros((max(rows, 1), self.width, channels), dtype=dtype, device=local.device)
        pad[: self.hi - self.lo] = local
        parts = [torch.empty_like(pad) for _ in range(self.world)]
        dist.all_gather(parts, pad, group=self.group)
        return torch.cat([parts[k][: hi - lo] for k, (lo, hi) in enumerate(self.bands)], dim=0)

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

    def gather_framebuffer(self, stream: Optional[int] = None):
        """The whole RGBA8 framebuffer (H, W) uint32 as int32 bits, on every rank.  With
        `stream` (GPU), the band's copy is enqueued on it and the gather follows it on the
        current stream without a host synchronisation."""
        import torch
        n = self.hi - self.lo
        if self._on_gpu():
            local = torch.empty((n, self.width, 1), dtype=torch.int32, device="cuda")
            self.r.copyFrameRows(self.lo, self.hi, None, local.data_ptr() if n else None, stream)
            if stream is None:
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
