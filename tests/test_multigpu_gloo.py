"""The multi-process row split (mdwtracker_b200.multigpu) on CPU: two gloo ranks each render
a band of every frame with the oracle and gather the bands; the assembled frames must
equal a single-process render bit for bit, also when the bands are re-cut between frames
from measured render times."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from mdwtracker_b200.multigpu import band, split_by_cost


def test_band_partition():
    for H in (1, 2, 7, 1024, 1081):
        for world in (1, 2, 3, 8):
            bands = [band(H, world, r) for r in range(world)]
            assert bands[0][0] == 0 and bands[-1][1] == H
            for (a, b), (c, d) in zip(bands, bands[1:]):
                assert b == c
            sizes = [b - a for a, b in bands]
            assert max(sizes) - min(sizes) <= 1


def _free_port() -> int:
    """A TCP port on 127.0.0.1 that nothing listens on now (for the gloo rendezvous)."""
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def test_split_by_cost_balances_and_covers():
    rng = np.random.default_rng(3)
    for H in (8, 37, 1080):
        for world in (1, 2, 3, 8):
            for cost in (np.ones(H), rng.random(H) ** 4, np.r_[np.zeros(H // 2), np.ones(H - H // 2)]):
                bands = split_by_cost(cost, world)
                assert len(bands) == world and bands[0][0] == 0 and bands[-1][1] == H
                for (a, b), (c, d) in zip(bands, bands[1:]):
                    assert b == c and a <= b
                for a, b in bands:
                    assert b - a >= (4 if H >= 4 * world else 0)
                for a, b in bands[:-1]:
                    assert b % 4 == 0 or H < 4 * world
                share = [cost[a:b].sum() for a, b in bands]
                # each share is within one 4-row alignment step (either side) of the mean
                if H >= 16 * world:
                    step = 8 * float(cost.max())
                    assert max(share) <= cost.sum() / world + step + 1e-9


def test_split_follows_a_centre_heavy_cost():
    H = 1080
    y = np.arange(H)
    cost = np.exp(-((y - H / 2) / (H / 8)) ** 2) + 1e-3
    bands = split_by_cost(cost, 4)
    sizes = [b - a for a, b in bands]
    assert sizes[0] > 2 * sizes[1] and sizes[3] > 2 * sizes[2]   # wide outer bands, narrow centre bands


def _scene():
    from mdwtracker_b200 import synthetic as syn
    vols = [syn.value_noise_sparse(24, occ, 200 + i, octaves=3) for i, occ in enumerate([0.2, 0.3])]
    tfs = [syn.ramp_tf(syn.HUES[i]) for i in range(2)]
    return vols, tfs


def _setup(r, vols, tfs, res):
    for v in vols:
        r.PushMesh(v)
    r.macrocellDims = (3, 3, 3)
    r.Resize(res)
    r.Init(2)
    for i, tf in enumerate(tfs):
        r.SetXFColormap(tf, i)
        r.SetXFOpacityScale(1.0, i)
        r.SetXFRange((0.0, 1.0), i)
    r.setSpp(3)
    return r


def _worker(rank, world, port, out_dir, frames, res, rebalance=False):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle.oracle import OracleRenderer, set_threads
    from mdwtracker_b200.multigpu import BandRenderer
    set_threads(1)
    vols, tfs = _scene()
    br = BandRenderer(_setup(OracleRenderer(), vols, tfs, res))
    accs, fbs, bands = [], [], []
    import time
    for _ in range(frames):
        t0 = time.perf_counter()
        br.render()
        dt = time.perf_counter() - t0
        accs.append(br.gather_accum().numpy())
        fbs.append(br.gather_framebuffer().numpy())
        if rebalance:   # a skewed time so that the bands move
            bands.append(br.rebalance(dt * (1.0 + 3.0 * rank)))
    cnt = br.reduce_counters()
    if rank == 0:
        np.savez(os.path.join(out_dir, "dist.npz"), acc=np.stack(accs), fb=np.stack(fbs), cnt=cnt,
                 bands=np.asarray(bands, dtype=np.int64).reshape(-1, world, 2))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,rebalance", [(2, False), (2, True)])
def test_row_split_equals_single_process(oracle, world, rebalance):
    res, frames = (21, 17), 3
    port = _free_port()
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_worker, args=(world, port, d, frames, res, rebalance), nprocs=world, join=True)
        got = np.load(os.path.join(d, "dist.npz"))
    if rebalance:   # the bands moved off the equal split
        assert any(tuple(map(tuple, b)) != tuple(band(res[1], world, k) for k in range(world)) for b in got["bands"])
    vols, tfs = _scene()
    o = _setup(oracle.OracleRenderer(), vols, tfs, res)
    for f in range(frames):
        o.Render()
        np.testing.assert_array_equal(got["acc"][f].view(np.uint32), o.accum().view(np.uint32))
        np.testing.assert_array_equal(got["fb"][f].view(np.uint32), o.framebuffer())
    np.testing.assert_array_equal(got["cnt"], o.counters().astype(np.int64))


class _LinearStandIn:
    """The denoiser's training calls (params / backward / copyGrads / loadGrads / adamStep)
    on a float64 least-squares model y = X w on the host: mean squared error over the
    shard, Adam with the denoiser's constants.  It stands in for the GPU network so that
    the data-parallel step can be checked with gloo ranks on the CPU."""

    device = "cpu"

    def __init__(self, nparam, seed=3):
        rng = np.random.default_rng(seed)
        self.w = rng.standard_normal(nparam)
        self.m = np.zeros(nparam)
        self.v = np.zeros(nparam)
        self.t = 0
        self.grad = np.zeros(nparam)

    def params(self):
        return self.w.copy()

    def backward(self, X, y, n, h, w, stream=0):
        r = X @ self.w - y
        self.grad = 2.0 * (X.T @ r) / len(y)
        return float(np.mean(r * r))

    def copyGrads(self, out, stream=0):
        import torch
        out.copy_(torch.from_numpy(self.grad))

    def loadGrads(self, src, stream=0):
        self.grad = src.numpy().copy()

    def adamStep(self, lr, stream=0):
        self.t += 1
        self.m = 0.9 * self.m + 0.1 * self.grad
        self.v = 0.999 * self.v + 0.001 * self.grad * self.grad
        self.w -= lr * (self.m / (1 - 0.9 ** self.t)) / (np.sqrt(self.v / (1 - 0.999 ** self.t)) + 1e-8)


def _regression(rows=16, nparam=5):
    rng = np.random.default_rng(11)
    X = rng.standard_normal((rows, nparam))
    return X, X @ rng.standard_normal(nparam) + 0.1 * rng.standard_normal(rows)


def _dp_worker(rank, world, port, out_dir, steps):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from mdwtracker_b200.multigpu import DataParallelTrainer
    X, y = _regression()
    per = len(y) // world
    Xs, ys = X[rank * per:(rank + 1) * per], y[rank * per:(rank + 1) * per]
    model = _LinearStandIn(X.shape[1])
    tr = DataParallelTrainer(model)
    losses = [tr.step(Xs, ys, per, 1, 1, 0.05) for _ in range(steps)]
    mine = torch.from_numpy(model.params())
    every = [torch.empty_like(mine) for _ in range(world)]
    dist.all_gather(every, mine)
    if rank == 0:
        np.savez(os.path.join(out_dir, "dp.npz"), params=np.stack([e.numpy() for e in every]), losses=losses)
    dist.barrier()
    dist.destroy_process_group()


def test_data_parallel_training_equals_full_batch_training():
    """Two ranks, each training on half of every minibatch, keep identical parameters and
    follow single-process training on the whole minibatch."""
    world, steps = 2, 25
    port = _free_port()
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_dp_worker, args=(world, port, d, steps), nprocs=world, join=True)
        got = np.load(os.path.join(d, "dp.npz"))
    np.testing.assert_array_equal(got["params"][0], got["params"][1])
    from mdwtracker_b200.multigpu import DataParallelTrainer
    X, y = _regression()
    ref = _LinearStandIn(X.shape[1])
    tr = DataParallelTrainer(ref)
    assert tr.world == 1
    losses = [tr.step(X, y, len(y), 1, 1, 0.05) for _ in range(steps)]
    np.testing.assert_allclose(got["params"][0], ref.params(), rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(got["losses"], losses, rtol=1e-10)
    assert losses[-1] < 0.5 * losses[0]
