"""The regrouped syncDDA (-m 2) and N-DDA (-m 0) tracker (MDWT_TUNE_REGROUP = 1, the
default; trace_regroup_kernel) against the oracle and against the warp-local tracker
(MDWT_TUNE_REGROUP = 0), bit for bit.

Regrouping changes only which lane runs which path when, so the accumulation buffer,
the framebuffer, the frame ids, the whole-frame counters and, with denoiser features or
gradient shading on, the per-path hit distances must be identical.  Per-pixel statistics
are off here (with them on, frames run the warp-local tracker)."""
import numpy as np
import pytest

from mdwtracker_b200 import Renderer
from mdwtracker_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

TUNE_POOL, TUNE_BATCH, TUNE_TRIPS, TUNE_REGROUP = 0, 1, 2, 4


def setup(r, vols, tfs, mc, res, spp, xf=None, camera=None, mode=2):
    for v in vols:
        r.PushMesh(v)
    r.macrocellDims = mc
    r.Resize(res)
    r.Init(mode, camera is None)
    if camera is not None:
        r.setCamera(*camera)
    for i, tf in enumerate(tfs):
        r.SetXFColormap(tf, i)
        r.SetXFOpacityScale(1.0, i)
        r.SetXFRange((0.0, 1.0) if xf is None else xf[i], i)
    r.setSpp(spp)
    return r


def regrouped(r, trips=4, batch=0):
    r.setTuning(TUNE_REGROUP, 1)
    r.setTuning(TUNE_TRIPS, trips)
    r.setTuning(TUNE_BATCH, batch)
    return r


def assert_same(p, o, tag):
    ap, ao = p.accum(), o.accum()
    bad = np.argwhere(np.any(ap.view(np.uint32) != ao.view(np.uint32), axis=-1))
    assert not len(bad), f"{tag}: {len(bad)} pixels differ, first {bad[0]}"
    np.testing.assert_array_equal(p.framebuffer(), o.framebuffer())
    assert p.frameIds() == o.frameIds()


def ran_regrouped(p):
    return p.renderInfo()[3] == 256


def noise_u8(n, occ, seed):
    return syn.value_noise_sparse(n, occ, seed, octaves=3)


def c2_like(n=48):
    vols = [noise_u8(n, occ, 10 + i) for i, occ in enumerate([0.1, 0.2, 0.3])]
    return vols, [syn.ramp_tf(syn.HUES[i]) for i in range(3)]


@pytest.mark.parametrize("mode", [2, 0])
@pytest.mark.parametrize("trips,batch", [(4, 0), (1, 0), (8, 2), (3, 5)])
def test_matches_the_oracle_uint8(oracle, trips, batch, mode):
    vols, tfs = c2_like()
    p = regrouped(setup(Renderer(0), vols, tfs, (6, 6, 6), (64, 48), 6, mode=mode), trips, batch)
    o = setup(oracle.OracleRenderer(), vols, tfs, (6, 6, 6), (64, 48), 6, mode=mode)
    for f in range(2):
        p.Render()
        o.Render()
        assert ran_regrouped(p)
        assert_same(p, o, f"frame {f}")
    np.testing.assert_array_equal(p.counters(), o.counters())


@pytest.mark.parametrize("mode", [2, 0])
def test_matches_the_oracle_float32_and_twelve_channels(oracle, mode):
    vols = [syn.lognormal(32, 5 + i, octaves=3) for i in range(12)]
    tfs = [syn.ramp_tf(syn.HUES[i % len(syn.HUES)], alpha_max=0.6) for i in range(12)]
    xf = [(0.0, 0.05)] * 12
    p = regrouped(setup(Renderer(0), vols, tfs, (4, 5, 3), (40, 36), 3, xf=xf, mode=mode))
    o = setup(oracle.OracleRenderer(), vols, tfs, (4, 5, 3), (40, 36), 3, xf=xf, mode=mode)
    for f in range(2):
        p.Render()
        o.Render()
        assert ran_regrouped(p)
        assert_same(p, o, f"frame {f}")
    np.testing.assert_array_equal(p.counters(), o.counters())


@pytest.mark.parametrize("mode", [2, 0])
def test_matches_the_oracle_with_a_culled_rectangle_and_frames(oracle, mode):
    """A camera that sees the volume in part of the image (traced rectangle smaller than
    the frame, partial tiles) and multi-frame launches."""
    vols, tfs = c2_like(40)
    cam = ((1.9, 0.7, 2.2), (0.9, 0.55, 0.4), (0.0, 1.0, 0.0), 38.0)
    p = regrouped(setup(Renderer(0), vols, tfs, (5, 5, 5), (53, 45), 2, camera=cam, mode=mode), trips=2)
    o = setup(oracle.OracleRenderer(), vols, tfs, (5, 5, 5), (53, 45), 2, camera=cam, mode=mode)
    for n in (3, 1):
        p.RenderFrames(n)
        o.RenderFrames(n)
        assert ran_regrouped(p)
        assert_same(p, o, f"{n} frames")
    np.testing.assert_array_equal(p.counters(), o.counters())


@pytest.mark.parametrize("mode", [2, 0])
@pytest.mark.parametrize("scene", ["c2", "lognormal"])
def test_matches_the_warp_local_tracker_at_size(scene, mode):
    if scene == "c2":
        vols, tfs = c2_like(128)
        mc, xf = (8, 8, 8), None
    else:
        vols = [syn.lognormal(128, 7 + i, octaves=4) for i in range(3)]
        tfs = [syn.ramp_tf(syn.HUES[i], alpha_max=0.3, start=0.4) for i in range(3)]
        mc, xf = (16, 16, 16), [(0.0, 0.05)] * 3
    a = setup(Renderer(0), vols, tfs, mc, (384, 256), 16, xf=xf, mode=mode)
    a.setTuning(TUNE_REGROUP, 0)
    b = regrouped(setup(Renderer(0), vols, tfs, mc, (384, 256), 16, xf=xf, mode=mode))
    for f in range(2):
        a.Render()
        b.Render()
        assert ran_regrouped(b) and not ran_regrouped(a)
        assert_same(b, a, f"frame {f}")
    np.testing.assert_array_equal(a.counters(), b.counters())
    assert a.counters()[0] > 0


def test_autotuner_picks_a_tracker_and_keeps_results(oracle):
    """The schedule autotuner tries both trackers for -m 2; whichever it keeps, frames stay
    identical to the oracle's."""
    vols, tfs = c2_like()
    p = setup(Renderer(0), vols, tfs, (6, 6, 6), (64, 48), 4)
    o = setup(oracle.OracleRenderer(), vols, tfs, (6, 6, 6), (64, 48), 4)
    p.autotuneSchedule(frames=2)
    assert p.getTuning(TUNE_REGROUP) in (0, 1) and 1 <= p.getTuning(TUNE_TRIPS) <= 8
    p.Render()
    o.Render()
    assert_same(p, o, "after tuning")
    np.testing.assert_array_equal(p.counters(), o.counters())


@pytest.mark.parametrize("mode", [2, 0])
def test_features_and_gradient_shading_match_the_oracle(oracle, mode):
    """Frames that carry the denoiser's features (hit distances per path) and frames with
    gradient shading (the hit point's gradient) run the regrouped tracker too."""
    vols, tfs = c2_like()
    p = regrouped(setup(Renderer(0), vols, tfs, (6, 6, 6), (64, 48), 4, mode=mode))
    o = setup(oracle.OracleRenderer(), vols, tfs, (6, 6, 6), (64, 48), 4, mode=mode)
    for r in (p, o):
        r.setFeatures(True)
    p.Render()
    o.Render()
    assert ran_regrouped(p)
    assert_same(p, o, "features")
    np.testing.assert_array_equal(p.features().view(np.uint32), o.features().view(np.uint32))
    for r in (p, o):
        r.setFeatures(False)
        r.setLight(False, True, (0.3, -1.0, 0.2), 1.3, 0.15)
    p.Render()
    o.Render()
    assert ran_regrouped(p)
    assert_same(p, o, "gradient shading")
    np.testing.assert_array_equal(p.counters(), o.counters())
