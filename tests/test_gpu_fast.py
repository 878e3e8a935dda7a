"""The fast free-flight arithmetic (mdwt_set_arithmetic(ctx, MDWT_ARITH_FAST)) against
the exact CPU oracle, held to the per-pixel event bar: at equal spp, the per-pixel
collision events -- density samples, rejections, hits and the hit channels over the
frame's samples -- equal the oracle's on at least 99.9 % of the pixels, and the
converged image stays within noise of the exact one.

Under the fast arithmetic every free flight t - log(1 - u) / majorant * dt * w2g
(deviceCode.cu:805, 913) is the hardware log2 times dt * w2g * ln 2 / majorant, where the
exact arithmetic runs the project's software log and correctly rounded quotients.  The
lengths differ in the last bits, so a path's events change only where a flight ends that
close to a cell or volume boundary, or a density lands that close to its acceptance
threshold; after such a change the path draws a different stream, and so can its pixel's
later samples.  The per-pixel statistics come from the warp-local tracker; the regrouped
tracker must give the warp-local tracker's frames bit for bit under either arithmetic.
"""
import numpy as np
import pytest

from mdwtracker_b200 import Renderer
from mdwtracker_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

TUNE_REGROUP = 4
EVENT_BAR = 0.999


def setup(r, vols, tfs, mc, res, spp, mode):
    for v in vols:
        r.PushMesh(v)
    r.macrocellDims = mc
    r.Resize(res)
    r.Init(mode)
    for i, tf in enumerate(tfs):
        r.SetXFColormap(tf, i)
        r.SetXFOpacityScale(1.0, i)
        r.SetXFRange((0.0, 1.0), i)
    r.setSpp(spp)
    return r


def c2_like(n=64):
    vols = [syn.value_noise_sparse(n, occ, 10 + i, octaves=3) for i, occ in enumerate([0.1, 0.2, 0.3])]
    return vols, [syn.ramp_tf(syn.HUES[i]) for i in range(3)], (n // 16,) * 3


def c3_like(n=48):
    """The 1080p scene's generators at n^3: 6 log-normal fields log-scaled into the TF
    domain, opacity ramps over the upper half, 8-voxel macrocells."""
    vols = [syn.lognormal_log10(n, 40 + i, octaves=3) for i in range(6)]
    tfs = [syn.ramp_tf(syn.HUES[i % len(syn.HUES)], alpha_max=0.25, start=0.5) for i in range(6)]
    return vols, tfs, (n // 8,) * 3


def event_agreement(p, o):
    sp, so = p.pixelStats(), o.pixelStats()
    same = np.all(sp == so, axis=-1)
    return float(same.mean()), int((~same).sum())


@pytest.mark.parametrize("scene", ["c2", "c3"])
@pytest.mark.parametrize("mode", [2, 0])
def test_events_match_the_exact_oracle_on_999_permille_of_pixels(oracle, scene, mode):
    vols, tfs, mc = c2_like() if scene == "c2" else c3_like()
    res, spp = (192, 160), 16
    p = setup(Renderer(0), vols, tfs, mc, res, spp, mode)
    o = setup(oracle.OracleRenderer(), vols, tfs, mc, res, spp, mode)
    p.setArithmetic(True)
    assert p.arithmetic() == 1
    np.testing.assert_array_equal(p.majorants(), o.majorants())   # the majorant grid is unchanged
    p.enablePixelStats(True)
    o.enablePixelStats(True)
    worst = 1.0
    for f in range(2):
        p.Render()
        o.Render()
        frac, n_diff = event_agreement(p, o)
        worst = min(worst, frac)
        assert frac >= EVENT_BAR, f"frame {f}: events differ on {n_diff} of {res[0] * res[1]} pixels"
    # the whole-frame counters agree to the same order
    cp, co = p.counters().astype(np.float64), o.counters().astype(np.float64)
    assert np.all(np.abs(cp - co) <= 1e-3 * np.maximum(co, 1.0) + 2.0), (cp, co)
    # images: bit-identical on nearly every pixel, close overall
    ap, ao = p.accum(), o.accum()
    same = np.all(ap.view(np.uint32) == ao.view(np.uint32), axis=-1)
    assert same.mean() >= 0.995, same.mean()
    d = ap[..., :3].astype(np.float64) - ao[..., :3]
    assert np.sqrt(np.mean(d * d)) < 1e-2
    print(f"{scene} -m {mode}: worst frame agreement {worst:.6f}")


@pytest.mark.parametrize("mode", [2, 0])
def test_regrouped_and_warp_local_trackers_agree_under_the_fast_arithmetic(mode):
    vols, tfs, mc = c3_like(40)
    frames = []
    for regroup in (1, 0):
        r = setup(Renderer(0), vols, tfs, mc, (96, 80), 8, mode)
        r.setArithmetic(True)
        r.setTuning(TUNE_REGROUP, regroup)
        r.Render()
        r.Render()
        assert (r.renderInfo()[3] == 256) == (regroup == 1)
        frames.append((r.accum(), r.framebuffer(), r.counters()))
        r.close()
    (a1, f1, c1), (a0, f0, c0) = frames
    np.testing.assert_array_equal(a1.view(np.uint32), a0.view(np.uint32))
    np.testing.assert_array_equal(f1, f0)
    np.testing.assert_array_equal(c1, c0)


def test_back_to_exact_is_bit_identical_to_the_oracle(oracle):
    vols, tfs, mc = c2_like(48)
    p = setup(Renderer(0), vols, tfs, mc, (64, 48), 8, 2)
    o = setup(oracle.OracleRenderer(), vols, tfs, mc, (64, 48), 8, 2)
    p.setArithmetic(True)
    p.Render()
    p.setArithmetic(False)
    p.ResetAccumulation()
    o.Render()            # keep the frame ids in step
    o.ResetAccumulation()
    p.Render()
    o.Render()
    np.testing.assert_array_equal(p.accum().view(np.uint32), o.accum().view(np.uint32))
    np.testing.assert_array_equal(p.framebuffer(), o.framebuffer())


def test_converged_image_is_within_noise_of_the_exact_one():
    """64 frames of 1 spp each way against the FP64 expected image of the estimator: the
    fast image's RMSE is the exact image's within a few per cent, and the two images
    are far closer to each other than either is to the expected image."""
    vols, tfs, mc = c3_like(40)
    imgs, rmses = [], []
    for fast in (False, True):
        r = setup(Renderer(0), vols, tfs, mc, (96, 80), 1, 2)
        r.setArithmetic(fast)
        e = r.expectedImage(8, 0.5)
        for _ in range(64):
            r.Render()
        imgs.append(r.accum()[..., :3].astype(np.float64))
        rmses.append(float(np.sqrt(np.mean((imgs[-1] - e) ** 2))))
        r.close()
    exact, fast = rmses
    assert abs(fast - exact) <= 0.05 * exact, rmses
    between = float(np.sqrt(np.mean((imgs[0] - imgs[1]) ** 2)))
    assert between < 0.25 * exact, (between, rmses)
