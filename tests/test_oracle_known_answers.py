"""Known-answer tests that pin the CPU oracle.

The reference ships no tests or golden vectors and cannot be built here, so the oracle
is pinned against answers derived from the domain and from published algorithms:
  * the RNG's TEA hash and LCG against their published test vectors;
  * the project log against libm;
  * an empty volume renders the background exactly;
  * a constant-density slab gives the Beer-Lambert collision probability 1-exp(-alpha*L/dt)
    (Woodcock tracking is unbiased; the reference's dt scales every free-flight step,
    deviceCode.cu:800-806, so the world extinction is alpha/dt);
  * a single bright voxel gives the hand-derived macrocell ranges and majorants
    (renderer.cu:387-392, 487-519, 835-893, 159-203);
  * a transfer function with zero opacity gives zero majorants.
"""
import ctypes as C
import math

import numpy as np
import pytest


def test_tea_published_vector(oracle):
    lib = oracle.load_oracle()
    k = (C.c_uint32 * 4)(0, 0, 0, 0)
    out = (C.c_uint32 * 2)()
    lib.orc_tea(C.c_uint32(0), C.c_uint32(0), k, 32, out)
    # TEA, 32 cycles, key 0, plaintext 0 (Wheeler & Needham reference cipher)
    assert (out[0], out[1]) == (0x41EA3A0A, 0x94BAA940)


def test_lcg_numerical_recipes_sequence(oracle):
    lib = oracle.load_oracle()
    out = (C.c_uint32 * 5)()
    lib.orc_lcg_states(C.c_uint32(0), 5, out)
    # Numerical Recipes in C (2nd ed.) sec. 7.1, quick-and-dirty generator from idum = 0
    assert list(out) == [0x3C6EF35F, 0x47502932, 0xD1CCF6E9, 0xAAF95334, 0x6252E503]


def test_rng_stream_is_uniform(oracle):
    xs = np.concatenate([oracle.rng_stream(i, 7 * i + 1, 256) for i in range(64)])
    assert xs.min() >= 0.0 and xs.max() < 1.0
    hist, _ = np.histogram(xs, bins=16, range=(0, 1))
    exp = len(xs) / 16
    chi2 = float(((hist - exp) ** 2 / exp).sum())
    assert chi2 < 40.0  # 15 dof, p ~ 5e-4


def test_log_accuracy(oracle):
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.random(2000).astype(np.float32), np.float32(2.0) ** -np.arange(1, 25, dtype=np.float32),
                         np.float32(1) - np.arange(1, 200, dtype=np.float32) * np.float32(2 ** -24)])
    xs = xs[xs > 0]
    for x in xs:
        got = oracle.oracle_log(float(x))
        ref = math.log(float(x))
        assert abs(got - ref) <= 3e-7 * max(abs(ref), 1e-30) + 1e-12, (x, got, ref)
    assert oracle.oracle_log(1.0) == 0.0


def _scene(oracle, vol, tf, res=(32, 32), spp=1, mode=0, mc=(4, 4, 4), bg=(0.0, 0.0, 0.0)):
    o = oracle.OracleRenderer()
    vols = vol if isinstance(vol, list) else [vol]
    for v in vols:
        o.PushMesh(v)
    o.macrocellDims = mc
    o.Resize(res)
    o.Init(mode)
    for i in range(len(vols)):
        o.SetXFColormap(tf, i)
        o.SetXFOpacityScale(1.0, i)
        o.SetXFRange((0.0, 1.0), i)
    o.setSpp(spp)
    o.setBackground(bg)
    return o


def ramp(n=256):
    tf = np.zeros((n, 4), np.float32)
    tf[:, 0] = 1.0
    tf[:, 3] = np.linspace(0, 1, n)
    return tf


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_empty_volume_renders_background(oracle, mode):
    vol = np.zeros((16, 16, 16), np.uint8)
    bg = (0.25, 0.5, 0.75)
    o = _scene(oracle, [vol, vol], ramp(), spp=4, mode=mode, bg=bg)
    assert np.all(o.majorants() == 0.0)
    o.Render()
    acc = o.accum()
    np.testing.assert_array_equal(acc[..., :3], np.broadcast_to(np.float32(bg), acc[..., :3].shape))
    # alpha: finalColor starts at 1 and gains 1 per sample (deviceCode.cu:289, 433): (spp+1)/spp
    np.testing.assert_array_equal(acc[..., 3], np.float32(1.25))
    assert o.counters()[0] == 0


def test_zero_alpha_tf_gives_zero_majorants(oracle):
    from mdwtracker_b200.synthetic import blobs
    tf = ramp()
    tf[:, 3] = 0.0
    o = _scene(oracle, blobs(32, 6, 3), tf)
    assert np.all(o.majorants() == 0.0)


def test_single_voxel_ranges_and_majorants(oracle):
    vol = np.zeros((16, 16, 16), np.uint8)
    vol[5, 5, 5] = 255
    o = _scene(oracle, vol, ramp(), mc=(4, 4, 4))
    rng = o.ranges().reshape(4, 4, 4, 2)     # [cz, cy, cx]
    # voxels 4, 5, 6 have voxel 5 in their 3x3x3 neighbourhood; their boxes
    # [p-1, p+1]/16 project onto cells {0,1} (voxel 4) and {1} (voxels 5, 6)
    hot = np.zeros((4, 4, 4), bool)
    hot[:2, :2, :2] = True
    assert np.all(rng[..., 0] == 0.0)
    np.testing.assert_array_equal(rng[..., 1][hot], 65025.0)
    np.testing.assert_array_equal(rng[..., 1][~hot], 0.0)
    maj = o.majorants().reshape(4, 4, 4)
    np.testing.assert_array_equal(maj[hot], 1.0)       # full texel range: max alpha = 1^3
    np.testing.assert_array_equal(maj[~hot], 0.0)      # texel 0: alpha 0


def test_beer_lambert_slab(oracle):
    """Constant density alpha over the unit cube: P(hit) = 1 - exp(-alpha * L / dt)."""
    alpha = 0.004
    tf = np.zeros((256, 4), np.float32)
    tf[:, 0] = 1.0
    tf[:, 3] = np.float32(alpha) ** (1.0 / 3.0)   # cubed on upload
    vol = np.full((32, 32, 32), 128, np.uint8)
    res = (33, 33)
    o = _scene(oracle, vol, tf, res=res, spp=2048, mode=2, mc=(4, 4, 4))
    o.enablePixelStats(True)
    o.Render()
    st = o.pixelStats()
    dt = o.dt                                   # 0.5 / 32
    basis = o.cameraBasis()
    org = basis[0].astype(np.float64)
    n = 0
    for (py, px) in [(16, 16), (14, 18), (10, 12), (20, 22)]:
        # expected path length through [0,1]^3 of the (jitter-averaged) pixel ray
        hits = st[py, px, 2]
        ps = []
        for j in np.linspace(0.0, 1.0, 33)[:-1] + 1.0 / 64:
            s = (np.array([px, py]) + j) / np.array(res)
            d = basis[1] + s[0] * basis[2] + s[1] * basis[3] - org
            d /= np.linalg.norm(d)
            with np.errstate(divide="ignore"):
                t0 = (0.0 - org) / d
                t1 = (1.0 - org) / d
            tn = np.max(np.minimum(t0, t1))
            tf_ = np.min(np.maximum(t0, t1))
            L = max(0.0, tf_ - tn)
            ps.append(1.0 - math.exp(-alpha * L / dt))
        p = float(np.mean(ps))
        phat = hits / 2048.0
        sigma = math.sqrt(p * (1 - p) / 2048.0)
        assert abs(phat - p) < 4.5 * sigma, (px, py, phat, p, sigma)
        n += 1
    assert n == 4


def _shading_scene(oracle, light_dir, shadows, gradient, spp, value=0.5, alpha=1.0, dt=None, res=(9, 9)):
    """Constant float volume over [0,1]^3 seen along +z from z = -2, one flat-colour TF."""
    tf = np.zeros((64, 4), np.float32)
    tf[:, :3] = (0.6, 0.3, 0.2)
    tf[:, 3] = np.float32(alpha) ** (1.0 / 3.0)   # cubed on upload
    o = oracle.OracleRenderer()
    o.PushMesh(np.full((16, 16, 16), value, np.float32))
    o.macrocellDims = (4, 4, 4)
    o.Resize(res)
    o.Init(2, False)
    o.setCamera((0.5, 0.5, -2.0), (0.5, 0.5, 0.5), (0.0, 1.0, 0.0), 8.0)
    if dt is not None:
        o.Setdt(dt)
    o.SetXFColormap(tf, 0)
    o.SetXFOpacityScale(1.0, 0)
    o.SetXFRange((0.0, 1.0), 0)
    o.setMaterial(0, diffuse=0.5, specular=0.3, shininess=8.0, gradientStep=0.01)
    o.setLight(shadows, gradient, light_dir, 1.0, 0.1)
    o.setSpp(spp)
    o.setBackground((0.0, 0.0, 0.0))
    o.enablePixelStats(True)
    return o


def _hit_colour(diffuse_times_shadow, ambient=0.1):
    alb = np.float32([0.6, 0.3, 0.2])
    mix = alb * np.float32(0.75) + np.float32(0.25)
    return np.float32(ambient) * mix + np.float32(diffuse_times_shadow) * alb


def test_gradient_of_constant_volume_is_material_diffuse(oracle):
    """Zero opacity gradient -> diffuse = material diffuse, no specular (deviceCode.cu:372-376)."""
    spp = 16
    o = _shading_scene(oracle, (0.3, -1.0, 0.2), False, True, spp, alpha=0.5)
    o.Render()
    acc, st = o.accum(), o.pixelStats()
    hits = st[..., 2].astype(np.float64)
    assert hits.sum() > 0
    want = hits[..., None] * _hit_colour(0.5)[None, None, :] / spp
    np.testing.assert_allclose(acc[..., :3], want, rtol=2e-6, atol=1e-7)


def test_shadow_rays_into_a_dense_medium_are_always_blocked(oracle):
    """Light from behind the volume: the shadow ray crosses ~1 unit of a medium with
    extinction 64 per unit, so every hit is shadowed: colour = ambient * mix only."""
    spp = 16
    o = _shading_scene(oracle, (0.0001, 0.0001, -1.0), True, False, spp, dt=1.0 / 64)
    o.Render()
    acc, st = o.accum(), o.pixelStats()
    hits = st[..., 2].astype(np.float64)
    assert hits.sum() > 0.9 * spp * acc.shape[0] * acc.shape[1] * 0.5
    want = hits[..., None] * _hit_colour(0.0)[None, None, :] / spp
    np.testing.assert_allclose(acc[..., :3], want, rtol=2e-6, atol=1e-7)


def test_shadow_rays_back_towards_the_camera_follow_the_shared_shadow_seed(oracle):
    """Light from the camera side.  Every shadow ray of a pixel in one frame starts from the
    same generator state, seeded from the frame and pixel only (deviceCode.cu:385-386).
    In a constant medium (majorant = density, every tentative collision is real) the shadow
    ray's first free flight s = -ln(1 - u1) / sigma, u1 the generator's first draw, ends the
    walk unless it leaves the front macrocell -- which here is leaving the volume.  A hit at
    depth d (density sigma*exp(-sigma*d)) is lit iff d < s, so the lit fraction of the
    pixel's samples is 1 - exp(-sigma*s) = u1."""
    spp = 2048
    o = _shading_scene(oracle, (0.0001, 0.0001, 1.0), True, False, spp, dt=1.0 / 64, res=(5, 5))
    o.Render()
    acc, st = o.accum(), o.pixelStats()
    lit, dark = _hit_colour(0.9), _hit_colour(0.0)
    us = []
    for (py, px) in [(2, 2), (1, 2), (2, 3), (3, 1)]:
        hits = float(st[py, px, 2])
        assert hits > 0.99 * spp
        # red channel: hits * (dark + u * (lit - dark)) / spp, u = lit fraction
        u = (acc[py, px, 0] * spp / hits - dark[0]) / (lit[0] - dark[0])
        u1 = float(oracle.rng_stream(px + 1, py + 1, 1)[0])    # frame 0: seed W*H*0
        sigma = math.sqrt(max(u1 * (1 - u1), 1e-4) / hits)
        assert abs(u - u1) < 4.5 * sigma + 0.01, (px, py, u, u1)
        us.append(u1)
    assert max(us) - min(us) > 0.05    # the pixels' generators differ


def _two_channel_scene(oracle, mode, alphas, colours, spp, res=(33, 33)):
    """Two constant channels over the unit cube with constant TF opacities `alphas` (cubed
    on upload, so given as their cube roots) and flat colours."""
    o = oracle.OracleRenderer()
    for _ in alphas:
        o.PushMesh(np.full((32, 32, 32), 128, np.uint8))
    o.macrocellDims = (4, 4, 4)
    o.Resize(res)
    o.Init(mode)
    for c, (a, rgb) in enumerate(zip(alphas, colours)):
        tf = np.zeros((256, 4), np.float32)
        tf[:, :3] = rgb
        tf[:, 3] = np.float32(a) ** (1.0 / 3.0)
        o.SetXFColormap(tf, c)
        o.SetXFOpacityScale(1.0, c)
        o.SetXFRange((0.0, 1.0), c)
    o.setSpp(spp)
    o.setBackground((0.0, 0.0, 0.0))
    o.enablePixelStats(True)
    return o


def _path_length(o, px, py, res):
    """Mean length through [0,1]^3 of the pixel's rays over its diagonal jitter."""
    basis = o.cameraBasis()
    org = basis[0].astype(np.float64)
    out = []
    for j in np.linspace(0.0, 1.0, 33)[:-1] + 1.0 / 64:
        s = (np.array([px, py]) + j) / np.array(res)
        d = basis[1] + s[0] * basis[2] + s[1] * basis[3] - org
        d /= np.linalg.norm(d)
        with np.errstate(divide="ignore"):
            t0, t1 = (0.0 - org) / d, (1.0 - org) / d
        out.append(max(0.0, np.min(np.maximum(t0, t1)) - np.max(np.minimum(t0, t1))))
    return out


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 4, 5])
def test_superposed_constant_channels(oracle, mode):
    """Every tracker samples the first collision of the superposed medium: with constant
    channel densities a0, a1 the hit probability is 1 - exp(-(a0 + a1) L / dt), and a hit
    lands on channel c with probability a_c / (a0 + a1).  The blends (-m 4, -m 5) sample
    the maximum channel opacity: 1 - exp(-max(a0, a1) L / dt)."""
    alphas, colours, spp, res = (0.003, 0.006), ((1.0, 0.0, 0.0), (0.0, 1.0, 0.0)), 2048, (33, 33)
    o = _two_channel_scene(oracle, mode, alphas, colours, spp, res)
    o.Render()
    st, acc, dt = o.pixelStats(), o.accum(), o.dt
    density = max(alphas) if mode >= 4 else sum(alphas)
    # the shaded colour of a hit on each channel: a single dense channel hits on every sample
    hit_rgb = []
    for rgb in colours:
        d = _two_channel_scene(oracle, 2, (1.0,), (rgb,), 4, (3, 3))
        d.Render()
        hit_rgb.append(d.accum()[1, 1, :3].astype(np.float64))
        assert d.pixelStats()[1, 1, 2] == 4
    M = np.stack(hit_rgb, axis=1)[:2]          # [R, G] rows, channel columns
    for (py, px) in [(16, 16), (14, 18), (10, 12), (20, 22)]:
        p = float(np.mean([1.0 - math.exp(-density * L / dt) for L in _path_length(o, px, py, res)]))
        hits = int(st[py, px, 2])
        sigma = math.sqrt(p * (1 - p) / spp)
        assert abs(hits / spp - p) < 4.5 * sigma, (mode, px, py, hits / spp, p)
        if mode <= 3:   # channel shares from the colour: rgb = sum_c (hits_c / spp) * hit_rgb_c
            n0, n1 = np.linalg.solve(M, acc[py, px, :2].astype(np.float64)) * spp
            assert abs(n0 + n1 - hits) < 0.05 * hits + 1.0
            share = alphas[0] / sum(alphas)
            s_sigma = math.sqrt(share * (1 - share) / hits)
            assert abs(n0 / (n0 + n1) - share) < 4.5 * s_sigma, (mode, px, py, n0 / (n0 + n1))


def test_majorants_follow_the_tf_range_and_opacity_scale(oracle):
    """renderer.cu:159-203: a cell's value range [lo, hi] is remapped through the TF range,
    addr = r * N; the majorant is the largest TF opacity over texels floor(addr(lo)) ..
    ceil(addr(hi)) (clamped), times the opacity scale.  With a monotone ramp that is the
    texel at the ceiling.  Volume 16^3 float32: 0.33 for z < 8, 0.05 above; 4^3 cells; TF
    range (0.1, 0.7): 0.33 -> r = 0.3833, addr 98.1 -> texels 98..99; 0.05 -> r < 0 ->
    texel 0 (opacity 0)."""
    vol = np.full((16, 16, 16), 0.05, np.float32)
    vol[:8] = 0.33                                 # [z][y][x]
    tf = np.zeros((256, 4), np.float32)
    tf[:, 0] = 1.0
    tf[:, 3] = np.arange(256, dtype=np.float32) / np.float32(255)   # cubed on upload
    o = oracle.OracleRenderer()
    o.PushMesh(vol)
    o.macrocellDims = (4, 4, 4)
    o.Resize((8, 8))
    o.Init(2)
    o.SetXFColormap(tf, 0)
    o.SetXFOpacityScale(0.5, 0)
    o.SetXFRange((0.1, 0.7), 0)
    maj = o.majorants().reshape(4, 4, 4)           # [cz][cy][cx]
    top = np.float32(0.5) * np.float32(np.float32(99) / np.float32(255)) ** 3
    # cells 0..2 along z see 0.33 (cell 1 and 2 through the 27-neighbour boxes at z = 7|8)
    np.testing.assert_allclose(maj[:3], top, rtol=1e-6)
    np.testing.assert_array_equal(maj[3], 0.0)
    # doubling the opacity scale doubles the majorants
    o.SetXFOpacityScale(1.0, 0)
    np.testing.assert_allclose(o.majorants().reshape(4, 4, 4)[:3], 2 * top, rtol=1e-6)


@pytest.mark.parametrize("cam", [((0.5, 0.5, -2.0), (0.5, 0.5, 0.5), (0.0, 1.0, 0.0), 30.0),
                                 ((2.1, 1.3, 1.7), (0.4, 0.6, 0.3), (0.0, 1.0, 0.0), 45.0),
                                 ((-1.0, 2.5, 0.2), (0.5, 0.5, 0.5), (0.0, 0.0, 1.0), 60.0)])
def test_camera_is_a_pinhole(oracle, cam):
    """UpdateCamera (renderer.cpp:1058-1092) with camera.h:83-110: pixel (sx, sy) looks
    along llc + sx horiz + sy vert - from.  The image centre looks at the point of interest,
    the image plane's axes are perpendicular to the view direction and to each other, the
    vertical field of view is fovy, and the plane's extents have the ratio W / H."""
    W, H = 64, 48
    o = oracle.OracleRenderer()
    o.PushMesh(np.zeros((8, 8, 8), np.uint8))
    o.Resize((W, H))
    o.Init(2, False)
    frm, at, up, fovy = cam
    o.setCamera(frm, at, up, fovy)
    org, llc, hor, ver = (b.astype(np.float64) for b in o.cameraBasis())
    np.testing.assert_allclose(org, frm, rtol=0, atol=1e-6)
    fwd = np.asarray(at, np.float64) - org
    fwd /= np.linalg.norm(fwd)
    centre = llc + 0.5 * hor + 0.5 * ver - org
    np.testing.assert_allclose(centre / np.linalg.norm(centre), fwd, atol=1e-5)
    assert abs(np.dot(hor, fwd)) < 1e-4 * np.linalg.norm(hor)
    assert abs(np.dot(ver, fwd)) < 1e-4 * np.linalg.norm(ver)
    assert abs(np.dot(hor, ver)) < 1e-4 * np.linalg.norm(hor) * np.linalg.norm(ver)
    top, bottom = llc + 0.5 * hor + ver - org, llc + 0.5 * hor - org
    angle = math.degrees(math.acos(np.dot(top, bottom) / (np.linalg.norm(top) * np.linalg.norm(bottom))))
    assert abs(angle - fovy) < 1e-3, angle
    assert abs(np.linalg.norm(hor) / np.linalg.norm(ver) - W / H) < 1e-5
    # up stays up: the vertical axis leans towards the up vector
    assert np.dot(ver, np.asarray(up, np.float64)) > 0


def test_default_dt_follows_the_last_channel(oracle):
    """Resetdt (renderer.cpp:1444-1454): dt = max(0.5 * min over axes of span / dims, 1e-4)
    of the LAST channel pushed, not the finest one."""
    for shapes, expect in [([(64, 64, 64), (16, 16, 16)], 0.5 / 16), ([(16, 16, 16), (64, 32, 128)], 0.5 / 128)]:
        o = oracle.OracleRenderer()
        for z, y, x in shapes:
            o.PushMesh(np.zeros((z, y, x), np.uint8))
        o.Resize((8, 8))
        o.Init(2)
        assert o.dt == np.float32(expect), (shapes, o.dt)


def test_accumulation_is_the_running_mean_of_the_frames(oracle):
    """deviceCode.cu:463-471: acc = (frame + a * acc) / (a + 1) with the frame's accumulation
    id a.  Render k sees the ids the previous Render left (renderer.cpp:957-958), so renders
    0 and 1 share frame and accumulation id 0: render 1 repeats render 0's frame and starts
    the mean afresh.  After K renders the buffer is the mean of renders 1 .. K-1, each of
    which is a frame of its own (checked by rendering every frame after a reset, which
    keeps the frame ids running)."""
    from mdwtracker_b200.synthetic import blobs
    vol = blobs(24, 5, 2)
    K = 5
    acc_on = _scene(oracle, vol, ramp(), res=(20, 16), spp=2, mode=2)
    for _ in range(K):
        acc_on.Render()
    ref = _scene(oracle, vol, ramp(), res=(20, 16), spp=2, mode=2)
    single = []
    for _ in range(K):
        ref.ResetAccumulation()
        ref.Render()
        single.append(ref.accum().astype(np.float64))
    np.testing.assert_array_equal(single[0], single[1])                 # the shared first seed
    assert np.std([f[..., :3].mean() for f in single[1:]]) > 0           # later frames differ
    np.testing.assert_allclose(acc_on.accum(), np.mean(single[1:], axis=0), rtol=1e-5, atol=1e-6)


def test_denoiser_features_at_the_extremes(oracle):
    """The 16 per-pixel features (mean radiance RGB, depth, miss fraction, hit fractions of
    channels 0..7, 1/sqrt(spp), two zeros): an empty volume gives the background, depth 0,
    miss fraction 1 and no hits; a dense single-channel medium gives miss fraction 0, a hit
    fraction of 1 on channel 0 and a positive depth."""
    spp = 4
    bg = (0.25, 0.5, 0.75)
    empty = _scene(oracle, np.zeros((16, 16, 16), np.uint8), ramp(), res=(12, 10), spp=spp, mode=2, bg=bg)
    empty.setFeatures(True)
    empty.Render()
    f = empty.features()
    np.testing.assert_array_equal(f[..., :3], np.broadcast_to(np.float32(bg), f[..., :3].shape))
    np.testing.assert_array_equal(f[..., 3], 0.0)
    np.testing.assert_array_equal(f[..., 4], 1.0)
    np.testing.assert_array_equal(f[..., 5:13], 0.0)
    np.testing.assert_allclose(f[..., 13], 1.0 / math.sqrt(spp), rtol=1e-6)
    np.testing.assert_array_equal(f[..., 14:], 0.0)
    dense = _two_channel_scene(oracle, 2, (1.0,), ((1.0, 0.0, 0.0),), spp, (12, 10))
    dense.setFeatures(True)
    dense.Render()
    g = dense.features()
    centre = g[3:7, 4:8]
    np.testing.assert_array_equal(centre[..., 4], 0.0)
    np.testing.assert_array_equal(centre[..., 5], 1.0)
    np.testing.assert_array_equal(centre[..., 6:13], 0.0)
    assert np.all(centre[..., 3] > 0)
