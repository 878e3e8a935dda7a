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
