"""The multi-process row split (mdwtracker_b200.multigpu) on CPU: two gloo ranks each render
a band of every frame with the oracle and gather the bands; the assembled frames must
equal a single-process render bit for bit."""
import os
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from mdwtracker_b200.multigpu import band


def test_band_partition():
    for H in (1, 2, 7, 1024, 1081):
        for world in (1, 2, 3, 8):
            bands = [band(H, world, r) for r in range(world)]
            assert bands[0][0] == 0 and bands[-1][1] == H
            for (a, b), (c, d) in zip(bands, bands[1:]):
                assert b == c
            sizes = [b - a for a, b in bands]
            assert max(sizes) - min(sizes) <= 1


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


def _worker(rank, world, port, out_dir, frames, res):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle.oracle import OracleRenderer, set_threads
    from mdwtracker_b200.multigpu import BandRenderer
    set_threads(1)
    vols, tfs = _scene()
    br = BandRenderer(_setup(OracleRenderer(), vols, tfs, res))
    accs, fbs = [], []
    for _ in range(frames):
        br.render()
        accs.append(br.gather_accum().numpy())
        fbs.append(br.gather_framebuffer().numpy())
    cnt = br.reduce_counters()
    if rank == 0:
        np.savez(os.path.join(out_dir, "dist.npz"), acc=np.stack(accs), fb=np.stack(fbs), cnt=cnt)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_row_split_equals_single_process(oracle, world):
    res, frames = (21, 17), 3
    port = 29500 + (os.getpid() % 2000)
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_worker, args=(world, port, d, frames, res), nprocs=world, join=True)
        got = np.load(os.path.join(d, "dist.npz"))
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
    port = 31500 + (os.getpid() % 2000)
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
