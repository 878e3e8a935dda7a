"""Batched rendering (include/mdwt_batch.h): many requests of different modes, voxel
formats, resolutions and spp in one persistent launch per kernel variant must give each
request exactly the frames mdwt_render gives it alone (bit for bit), with and without
the CUDA graph, before and after autotuning; macrocell regrids after init match the
oracle."""
import numpy as np
import pytest

from mdwtracker_b200 import Batch, Renderer
from mdwtracker_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def _requests():
    u8 = [syn.value_noise_sparse(40, occ, 80 + i, octaves=3) for i, occ in enumerate([0.15, 0.3, 0.25])]
    f32 = [syn.lognormal(32, 90 + i, octaves=3) for i in range(2)]
    specs = [
        dict(vols=u8[:2], mode=2, res=(64, 48), spp=3, mc=(5, 5, 5), stats=True),
        dict(vols=u8, mode=0, res=(33, 29), spp=2, mc=(4, 4, 4), stats=False),
        dict(vols=f32, mode=2, res=(80, 40), spp=4, mc=(4, 3, 5), stats=False, xf=(0.0, 0.05)),
        dict(vols=u8[1:], mode=2, res=(24, 70), spp=1, mc=(6, 6, 6), stats=False),
        dict(vols=f32[:1], mode=3, res=(40, 40), spp=5, mc=(3, 3, 3), stats=True, xf=(0.0, 0.05)),
        dict(vols=u8[:1], mode=1, res=(50, 30), spp=2, mc=(4, 4, 4), stats=False),
        dict(vols=u8, mode=5, res=(36, 44), spp=3, mc=(5, 5, 5), stats=True),
        dict(vols=f32, mode=4, res=(30, 30), spp=2, mc=(4, 4, 4), stats=False, xf=(0.0, 0.05)),
    ]
    return specs


def _setup(spec):
    r = Renderer(0)
    for v in spec["vols"]:
        r.PushMesh(v)
    r.macrocellDims = spec["mc"]
    r.Resize(spec["res"])
    r.Init(spec["mode"])
    for i in range(len(spec["vols"])):
        r.SetXFColormap(syn.ramp_tf(syn.HUES[i % len(syn.HUES)], alpha_max=0.7), i)
        r.SetXFOpacityScale(1.0, i)
        r.SetXFRange(spec.get("xf", (0.0, 1.0)), i)
    r.setSpp(spec["spp"])
    if spec["stats"]:
        r.enablePixelStats(True)
    return r


def _same(a, b, stats):
    np.testing.assert_array_equal(a.accum().view(np.uint32), b.accum().view(np.uint32))
    np.testing.assert_array_equal(a.framebuffer(), b.framebuffer())
    if stats:
        np.testing.assert_array_equal(a.pixelStats(), b.pixelStats())
    assert a.frameIds() == b.frameIds()


@pytest.mark.parametrize("graph,fusion", [(True, True), (False, True), (True, False)])
def test_batch_equals_individual_renders(graph, fusion):
    specs = _requests()
    batched = [_setup(s) for s in specs]
    alone = [_setup(s) for s in specs]
    b = Batch(0)
    b.setGraph(graph)
    b.setFusion(fusion)
    for r in batched:
        b.add(r)
    for f in range(3):
        b.render()
        for r in alone:
            r.Render()
        b.sync()
        for s, x, y in zip(specs, batched, alone):
            _same(x, y, s["stats"])
    for x, y in zip(batched, alone):
        np.testing.assert_array_equal(x.counters(), y.counters())
    info = b.info()
    assert info["groups"] >= 4 and info["requests"] == len(specs)
    # the two regroupable variants (-m 2 float32, -m 2 uint8; -m 0 runs the warp-local
    # tracker by default) share one launch
    assert b.traceLaunches() == info["groups"] - (1 if fusion else 0)
    if graph:
        assert info["graph_captures"] == 1 and info["graph_replays"] == 3


def test_batch_autotune_and_schedule_do_not_change_results():
    specs = _requests()
    batched = [_setup(s) for s in specs]
    alone = [_setup(s) for s in specs]
    b = Batch(0)
    for r in batched:
        b.add(r)
    b.render()
    for r in alone:
        r.Render()
    best = b.autotune(frames=1)
    assert best[0] % 32 == 0 and best[1] in (4, 8, 16, 32) and best[2] in (1, 2, 3, 4)
    for r in alone:
        r.ResetAccumulation()      # the tuner restores frame ids and resets accumulation
    for sched in [(64, 1, 1), (4096, 32, 4)]:
        b.setSchedule(*sched)
        b.render()
        for r in alone:
            r.Render()
        b.sync()
        for s, x, y in zip(specs, batched, alone):
            _same(x, y, s["stats"])


def test_regrid_after_init_matches_the_oracle(oracle):
    vols = [syn.value_noise_sparse(40, occ, 60 + i, octaves=3) for i, occ in enumerate([0.2, 0.3])]
    p, o = Renderer(0), oracle.OracleRenderer()
    for r in (p, o):
        for v in vols:
            r.PushMesh(v)
        r.macrocellDims = (4, 4, 4)
        r.Resize((40, 32))
        r.Init(2)
        for i in range(2):
            r.SetXFColormap(syn.ramp_tf(syn.HUES[i]), i)
            r.SetXFOpacityScale(1.0, i)
            r.SetXFRange((0.0, 1.0), i)
        r.setSpp(3)
        r.Render()
        r.macrocellDims = (7, 3, 5)    # new grid after init, transfer functions kept
    np.testing.assert_array_equal(p.macrocellDims, (7, 3, 5))
    np.testing.assert_array_equal(p.ranges(), o.ranges())
    np.testing.assert_array_equal(p.majorants(), o.majorants())
    for _ in range(2):
        p.Render()
        o.Render()
        np.testing.assert_array_equal(p.accum().view(np.uint32), o.accum().view(np.uint32))


def test_macrocell_autotuner_picks_a_candidate(oracle):
    spec = _requests()[0]
    r = _setup(spec)
    ids = r.frameIds()
    best = r.autotuneMacrocells((4, 8, 16), frames=1)
    assert best in (4, 8, 16)
    assert r.frameIds()[0] == ids[0]
    n = -(-40 // best)
    assert r.macrocellDims == (n, n, n)


def test_schedule_autotuner_keeps_results(oracle):
    spec = _requests()[2]
    r, twin = _setup(spec), _setup(spec)
    r.Render()
    twin.Render()
    pool, trips = r.autotuneSchedule(frames=1)
    assert pool in (4, 8, 16, 32) and trips in (1, 2, 3, 4, 6, 8, 12, 16)
    twin.ResetAccumulation()
    for _ in range(2):
        r.Render()
        twin.Render()
    _same(r, twin, spec["stats"])


def test_batch_rejects_duplicates_and_foreign_state():
    from mdwtracker_b200 import MdwtError
    r = _setup(_requests()[0])
    b = Batch(0)
    b.add(r)
    with pytest.raises(MdwtError):
        b.add(r)
    with pytest.raises(MdwtError):
        Batch(0).render()            # empty batch
