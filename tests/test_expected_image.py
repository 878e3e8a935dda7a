"""The FP64 expected image (the ground truth of convergence measurements).

CPU: the oracle's quadrature against a closed form (constant medium: Beer-Lambert with the
shaded colour) and against its own high-spp Monte Carlo render.
GPU: libmdwt's FP64 kernel against the oracle's quadrature, and the tracker's accumulated
render converging to it.
"""
import math

import numpy as np
import pytest

from mdwtracker_b200 import synthetic as syn


def _constant_scene(r, value=0.5, alpha=0.3, res=(12, 10), bg=(0.2, 0.4, 0.6)):
    tf = np.zeros((32, 4), np.float32)
    tf[:, :3] = (0.7, 0.5, 0.1)
    tf[:, 3] = np.float32(alpha) ** (1.0 / 3.0)
    r.PushMesh(np.full((16, 16, 16), value, np.float32))
    r.macrocellDims = (4, 4, 4)
    r.Resize(res)
    r.Init(2)
    r.SetXFColormap(tf, 0)
    r.SetXFOpacityScale(1.0, 0)
    r.SetXFRange((0.0, 1.0), 0)
    r.setBackground(bg)
    return r, tf


def _noise_scene(r, res=(16, 12), mode=2, n=32):
    vols = [syn.value_noise_sparse(n, occ, 70 + i, octaves=3) for i, occ in enumerate([0.2, 0.35])]
    for v in vols:
        r.PushMesh(v)
    r.macrocellDims = (4, 4, 4)
    r.Resize(res)
    r.Init(mode)
    for i in range(2):
        r.SetXFColormap(syn.ramp_tf(syn.HUES[i], alpha_max=0.6), i)
        r.SetXFOpacityScale(1.0, i)
        r.SetXFRange((0.0, 1.0), i)
    r.setBackground((0.1, 0.1, 0.1))
    return r


def test_constant_medium_closed_form(oracle):
    """E = mean_j [(1 - exp(-alpha L_j / dt)) colour + exp(-alpha L_j / dt) bg], L_j the
    chord of jitter ray j through the unit cube (the quadrature is exact for a constant
    extinction)."""
    o, tf = _constant_scene(oracle.OracleRenderer())
    J = 4
    e = o.expectedImage(J, 0.5)
    alpha = float(np.float32(np.float32(tf[0, 3]) ** np.float32(3.0)))
    dt = float(o.dt)
    alb = np.array([0.7, 0.5, 0.1], np.float64).astype(np.float32).astype(np.float64)
    colour = 0.1 * (0.75 * alb + 0.25) + 1.0 * alb
    bg = np.array([0.2, 0.4, 0.6], np.float32).astype(np.float64)
    basis = o.cameraBasis().astype(np.float64)
    org, llc, hor, ver = basis
    W, H = o.fbSize
    for py in range(H):
        for px in range(W):
            want = np.zeros(3)
            for m in range(J):
                j = (m + 0.5) / J
                d = llc + (px + j) / W * hor + (py + j) / H * ver - org
                d /= math.sqrt(d @ d)
                with np.errstate(divide="ignore"):
                    t0, t1 = (0.0 - org) / d, (1.0 - org) / d
                ta = max(0.0, np.max(np.minimum(t0, t1)))
                tb = np.min(np.maximum(t0, t1))
                L = max(0.0, tb - ta)
                T = math.exp(-alpha / dt * L)
                want += (1.0 - T) * colour + T * bg
            np.testing.assert_allclose(e[py, px], want / J, rtol=1e-7, atol=1e-12)   # alpha^3 rounding


def test_quadrature_converges_in_step_and_jitter(oracle):
    o = _noise_scene(oracle.OracleRenderer())
    coarse = o.expectedImage(8, 0.5)
    fine = o.expectedImage(32, 0.125)
    rmse = float(np.sqrt(np.mean((coarse - fine) ** 2)))
    assert rmse < 4e-3, rmse


def test_monte_carlo_render_converges_to_the_expected_image(oracle):
    """4096 spp of the tracker (same estimator) against the FP64 expectation: the RMSE is
    the Monte Carlo noise, at most sqrt(var / spp) with per-sample colour variance below
    0.25 per channel."""
    spp = 4096
    o = _noise_scene(oracle.OracleRenderer(), res=(12, 9))
    o.setSpp(spp)
    o.Render()
    o.renderExpected(32, 0.125)
    rmse = o.accumRmse()
    bias = float(np.mean(o.accum()[..., :3] - o._expected))
    assert rmse < math.sqrt(0.25 / spp) * 1.2 + 2e-3, rmse
    assert abs(bias) < 2e-3, bias


def test_shaded_expected_image_is_refused(oracle):
    from mdwtracker_b200.renderer import MdwtError
    o, _ = _constant_scene(oracle.OracleRenderer())
    o.setLight(True, False, (0.0, -1.0, 0.0))
    with pytest.raises(MdwtError):
        o.expectedImage()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 2])
def test_gpu_expected_image_matches_the_oracle(oracle, mode):
    from mdwtracker_b200 import Renderer
    p = _noise_scene(Renderer(0), mode=mode)
    o = _noise_scene(oracle.OracleRenderer(), mode=mode)
    for J, step in [(4, 0.5), (3, 0.3)]:
        ep, eo = p.expectedImage(J, step), o.expectedImage(J, step)
        np.testing.assert_allclose(ep, eo, rtol=1e-10, atol=1e-12)


@pytest.mark.gpu
def test_gpu_float_channels_expected_image_matches_the_oracle(oracle):
    from mdwtracker_b200 import Renderer
    vols = [syn.lognormal(28, 40 + i, octaves=3) for i in range(3)]

    def setup(r):
        for v in vols:
            r.PushMesh(v)
        r.macrocellDims = (3, 4, 5)
        r.Resize((20, 14))
        r.Init(2)
        for i in range(3):
            r.SetXFColormap(syn.ramp_tf(syn.HUES[i], alpha_max=0.7), i)
            r.SetXFOpacityScale(0.8, i)
            r.SetXFRange((0.0, 0.05), i)
        return r
    p, o = setup(Renderer(0)), setup(oracle.OracleRenderer())
    np.testing.assert_allclose(p.expectedImage(4, 0.5), o.expectedImage(4, 0.5), rtol=1e-10, atol=1e-12)


@pytest.mark.gpu
def test_gpu_accumulation_converges_and_rmse_matches_host(oracle):
    from mdwtracker_b200 import Renderer
    p = _noise_scene(Renderer(0), res=(64, 48))
    p.setSpp(1)     # one sample per frame: frame f draws with seed factor f + 1, all distinct
    e = p.expectedImage(16, 0.25)
    prev = None
    for f in range(512):
        p.Render()
        if f in (7, 63, 511):
            r = p.accumRmse()
            d = p.accum()[..., :3].astype(np.float64) - e
            assert abs(r - math.sqrt(float(np.mean(d * d)))) < 1e-9
            if prev is not None:
                assert r < prev
            prev = r
    assert prev < 0.03
