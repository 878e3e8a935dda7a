"""GPU parity: libmdwt.so (sm_100a kernels) against the CPU oracle, bit for bit.

Every case runs the same scene script through both renderers and compares
  * the per-(cell, channel) value ranges and the majorant grid (bit-exact),
  * the accumulation buffer (float4, bit-exact) and the RGBA8 framebuffer,
  * per-pixel event statistics (density samples, rejections, hits, hit channels),
  * the whole-frame counters,
after every frame.  The bar is bit-identity; the tolerance is zero.
"""
import numpy as np
import pytest

from mdwtracker_b200 import Renderer
from mdwtracker_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


def make_pair(oracle, vols, tfs, mode, mc, res, spp, opacity=None, xf=None, camera=None, dt=None,
              reshape=None, bg=None):
    p = Renderer(0)
    o = oracle.OracleRenderer()
    for r in (p, o):
        for i, v in enumerate(vols):
            r.PushMesh(v)
            if reshape is not None:
                r.reshapeBounds(i, reshape)
        r.macrocellDims = mc
        r.Resize(res)
        r.Init(mode, camera is None)
        if camera is not None:
            r.setCamera(*camera)
        if dt is not None:
            r.Setdt(dt)
        for i, tf in enumerate(tfs):
            r.SetXFColormap(tf, i)
            r.SetXFOpacityScale(1.0 if opacity is None else opacity[i], i)
            r.SetXFRange((0.0, 1.0) if xf is None else xf[i], i)
        r.setSpp(spp)
        if bg is not None:
            r.setBackground(bg)
        r.enablePixelStats(True)
    return p, o


def assert_same_grid(p, o):
    np.testing.assert_array_equal(p.macrocellDims, o.macrocellDims)
    rp, ro = p.ranges(), o.ranges()
    np.testing.assert_array_equal(rp, ro)
    np.testing.assert_array_equal(p.majorants(), o.majorants())


def assert_same_frame(p, o, tag=""):
    ap, ao = p.accum(), o.accum()
    bad = np.argwhere(np.any(ap.view(np.uint32) != ao.view(np.uint32), axis=-1))
    if len(bad):
        sp, so = p.pixelStats(), o.pixelStats()
        y, x = bad[0]
        raise AssertionError(f"{tag}: {len(bad)} pixels differ; first ({x},{y}) gpu {ap[y, x]} {sp[y, x]} "
                             f"oracle {ao[y, x]} {so[y, x]}")
    np.testing.assert_array_equal(p.framebuffer(), o.framebuffer())
    np.testing.assert_array_equal(p.pixelStats(), o.pixelStats())
    assert p.frameIds() == o.frameIds()


def run_frames(p, o, frames, between=None):
    for f in range(frames):
        if between is not None:
            between(f, p)
            between(f, o)
        p.Render()
        o.Render()
        assert_same_frame(p, o, f"frame {f}")
    np.testing.assert_array_equal(p.counters(), o.counters())


def noise_u8(n, occ, seed):
    return syn.value_noise_sparse(n, occ, seed, octaves=3)


def test_c1_like_ndda(oracle):
    vol = syn.blobs(64, 16, 1)
    p, o = make_pair(oracle, [vol], [syn.viridis_like()], 0, (8, 8, 8), (96, 80), 1)
    assert_same_grid(p, o)
    assert np.array_equal(p.cameraBasis(), o.cameraBasis()) and p.dt == o.dt
    run_frames(p, o, 5)
    c = p.counters()
    assert c[0] > 0 and c[3] == 96 * 80 * 5


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 4, 5])
def test_c2_like_three_channels(oracle, mode):
    vols = [noise_u8(48, occ, 10 + i) for i, occ in enumerate([0.1, 0.2, 0.3])]
    tfs = [syn.ramp_tf(syn.HUES[i]) for i in range(3)]
    p, o = make_pair(oracle, vols, tfs, mode, (6, 6, 6), (64, 48), 6)
    assert_same_grid(p, o)
    run_frames(p, o, 2)


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 4, 5])
def test_float32_lognormal(oracle, mode):
    vols = [syn.lognormal(40, 5 + i, octaves=4) for i in range(2)]
    tfs = [syn.ramp_tf(syn.HUES[i], alpha_max=0.7) for i in range(2)]
    p, o = make_pair(oracle, vols, tfs, mode, (5, 5, 5), (40, 40), 4, xf=[(0.0, 0.05)] * 2)
    assert_same_grid(p, o)
    run_frames(p, o, 2)


def test_mixed_formats_and_ragged_dims(oracle):
    """uint8 + float32 + int8 channels of different shapes; macrocells that do not divide."""
    rng = np.random.default_rng(3)
    a = noise_u8(32, 0.3, 3)                                         # 32^3 uint8
    b = (syn.value_noise(24, 3, 4) * 40.0).astype(np.float32)[:, :20, :]  # dims (24, 20, 24)
    c = rng.integers(-20, 60, (17, 23, 29)).astype(np.int8)          # dims (29, 23, 17)
    tfs = [syn.ramp_tf(syn.HUES[i]) for i in range(3)]
    for mode in (0, 1, 2, 3, 4, 5):
        p, o = make_pair(oracle, [a, b, c], tfs, mode, (7, 5, 3), (45, 37), 3, opacity=[1.0, 0.6, 2.0])
        assert_same_grid(p, o)
        run_frames(p, o, 2)


def test_twelve_channels(oracle):
    vols = [noise_u8(12, 0.25, 40 + i) for i in range(12)]
    tfs = [syn.ramp_tf(syn.HUES[i]) for i in range(12)]
    for mode in (0, 1, 2, 3):
        p, o = make_pair(oracle, vols, tfs, mode, (3, 3, 3), (24, 24), 2)
        assert_same_grid(p, o)
        run_frames(p, o, 1)


def test_reshaped_bounds_and_explicit_camera(oracle):
    vol = syn.blobs(32, 10, 7)
    cam = ((70.0, 40.0, -35.0), (16.0, 16.0, 16.0), (0.0, 1.0, 0.0), 35.0)
    p, o = make_pair(oracle, [vol, vol[::-1].copy()], [syn.viridis_like(), syn.ramp_tf(syn.HUES[1])], 2, (4, 4, 4),
                     (50, 30), 3, camera=cam, reshape=None)
    run_frames(p, o, 1)
    p, o = make_pair(oracle, [vol], [syn.viridis_like()], 0, (4, 8, 4), (50, 30), 3, camera=cam, reshape=(32, 32, 32))
    assert_same_grid(p, o)
    assert p.dt == o.dt
    run_frames(p, o, 2)


def test_state_changes_between_frames(oracle):
    """Mirror, accumulation off, background, dt, TF range and opacity edits, resize."""
    vols = [noise_u8(32, 0.2, 60), noise_u8(32, 0.15, 61)]
    tfs = [syn.ramp_tf(syn.HUES[0]), syn.ramp_tf(syn.HUES[2])]
    p, o = make_pair(oracle, vols, tfs, 2, (4, 4, 4), (40, 32), 2, bg=(0.1, 0.2, 0.3))

    def between(f, r):
        if f == 1:
            r.setMirror(True)
        if f == 2:
            r.setAccumulation(False)
            r.Setdt(0.02)
        if f == 3:
            r.setAccumulation(True)
            r.SetXFRange((0.1, 0.7), 1)
            r.SetXFOpacityScale(3.0, 0)
        if f == 4:
            r.ResetAccumulation()
            r.setSpp(5)

    run_frames(p, o, 6, between)
    assert_same_grid(p, o)
    for r in (p, o):
        r.Resize((23, 41))
    run_frames(p, o, 2)


@pytest.mark.parametrize("cam", [
    ((0.5, 0.5, 0.5), (0.9, 0.2, 0.1), (0.0, 1.0, 0.0), 70.0),     # inside the volume
    ((0.5, 0.5, 3.0), (0.5, 0.5, 6.0), (0.0, 1.0, 0.0), 45.0),     # looking away
    ((0.5, 0.5, 3.0), (0.5, 0.5, 0.5), (0.0, 1.0, 0.0), 1.0),      # nearly parallel rays
    ((-2.0, 0.5, 0.5), (0.5, 0.5, 0.5), (0.0, 0.0, 1.0), 40.0),    # along +x
])
def test_camera_edge_cases(oracle, cam):
    vols = [noise_u8(24, 0.3, 70), noise_u8(24, 0.2, 71)]
    for mode in (0, 1, 2, 3):
        p, o = make_pair(oracle, vols, [syn.viridis_like()], mode, (3, 3, 3), (33, 31), 3, camera=cam)
        run_frames(p, o, 1)


@pytest.mark.parametrize("mode,batch,pool", [(2, 3, 1), (0, 5, 32), (2, 1, 8), (0, 0, 4), (1, 4, 8), (3, 2, 16)])
def test_sample_batches_and_pool_sizes(oracle, mode, batch, pool):
    """Path records resolved over several sample batches (running sums carried between
    passes) and any regeneration pool give the oracle's sequential spp loop exactly."""
    vols = [noise_u8(32, 0.25, 90), noise_u8(32, 0.2, 91)]
    tfs = [syn.ramp_tf(syn.HUES[0]), syn.ramp_tf(syn.HUES[1])]
    p, o = make_pair(oracle, vols, tfs, mode, (4, 4, 4), (40, 36), 11)
    p.setTuning(1, batch)
    p.setTuning(0, pool)
    run_frames(p, o, 2)


def test_no_tf_and_empty_volume(oracle):
    """A channel without a colour map is invisible; an all-zero volume renders the background."""
    vols = [np.zeros((16, 16, 16), np.uint8), noise_u8(16, 0.3, 80)]
    p, o = make_pair(oracle, vols, [syn.viridis_like()], 2, (4, 4, 4), (32, 32), 2, bg=(0.25, 0.5, 0.75))
    assert_same_grid(p, o)
    run_frames(p, o, 1)


def test_row_bands_assemble_the_full_frame(oracle):
    """Contexts rendering disjoint row bands (mdwt_set_render_rows) give the full frame,
    read back band by band through mdwt_copy_frame_rows (the multi-GPU row split)."""
    import torch
    vols = [noise_u8(32, 0.25, 110), noise_u8(32, 0.2, 111)]
    tfs = [syn.ramp_tf(syn.HUES[0]), syn.ramp_tf(syn.HUES[1])]
    full, o = make_pair(oracle, vols, tfs, 2, (4, 4, 4), (40, 37), 4)
    bands = [(0, 13), (13, 25), (25, 37)]
    parts = [make_pair(oracle, vols, tfs, 2, (4, 4, 4), (40, 37), 4)[0] for _ in bands]
    for f in range(2):
        full.Render()
        acc = torch.empty((37, 40, 4), dtype=torch.float32, device="cuda")
        fb = torch.empty((37, 40), dtype=torch.int32, device="cuda")
        for r, (a, b) in zip(parts, bands):
            r.setRenderRows(a, b)
            r.Render()
            r.copyFrameRows(a, b, acc[a:b].data_ptr(), fb[a:b].data_ptr())
            r.sync()
        np.testing.assert_array_equal(acc.cpu().numpy().view(np.uint32), full.accum().view(np.uint32))
        np.testing.assert_array_equal(fb.cpu().numpy().view(np.uint32), full.framebuffer())
    tot = sum(np.asarray(r.counters(), dtype=np.uint64) for r in parts)
    np.testing.assert_array_equal(tot, full.counters())


def test_cli_on_the_gpu_matches_the_oracle(tmp_path, oracle):
    """The headless front end end to end on libmdwt.so: final PNG equals the oracle's."""
    from mdwtracker_b200 import cli, imageio
    vol = noise_u8(24, 0.3, 5)
    raw = str(tmp_path / "vol_24x24x24_uint8.raw")
    vol.tofile(raw)
    tf = str(tmp_path / "a.tf")
    imageio.save_tf(tf, syn.ramp_tf(syn.HUES[0]), 1.5, (0.0, 0.9))
    args = ["-fr", raw, raw, "-t", tf, tf, "-mc", "3", "-r", "20", "16", "-m", "2", "-spp", "2", "-n", "3", "-wu", "1",
            "-mf", "1"]
    a = cli.build_parser().parse_args(args + ["-o", str(tmp_path / "gpu")])
    p = cli.setup(a, Renderer(0))
    cli.run(a, p)
    b = cli.build_parser().parse_args(args + ["-o", str(tmp_path / "cpu")])
    o = cli.setup(b, oracle.OracleRenderer())
    cli.run(b, o)
    np.testing.assert_array_equal(imageio.read_png(str(tmp_path / "gpu_AMMB_w_3_shadows_off_frames.png")),
                                  imageio.read_png(str(tmp_path / "cpu_AMMB_w_3_shadows_off_frames.png")))


def _shade(r, shadows, gradient, light, nch):
    r.setLight(shadows, gradient, light, 1.3, 0.15)
    for i in range(nch):
        r.setMaterial(i, diffuse=0.6 + 0.1 * i, specular=0.4, shininess=4.0 + 6.0 * i,
                      gradientStep=(0.01, 0.2, 0.05)[i % 3], specularColor=(1.0, 0.9 - 0.2 * i, 0.8))


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 4, 5])
@pytest.mark.parametrize("shadows,gradient", [(True, False), (False, True), (True, True)])
def test_shadows_and_gradient_shading(oracle, mode, shadows, gradient):
    """Shadow rays traced by the same tracker from the hit point towards -lightDir
    (deviceCode.cu:380-397) and Blinn-Phong shading from the opacity gradient
    (deviceCode.cu:243-281, 327-378), bit for bit."""
    vols = [noise_u8(40, occ, 30 + i) for i, occ in enumerate([0.15, 0.3])]
    tfs = [syn.ramp_tf(syn.HUES[i], alpha_max=0.9) for i in range(2)]
    p, o = make_pair(oracle, vols, tfs, mode, (5, 5, 5), (48, 40), 4)
    for r in (p, o):
        _shade(r, shadows, gradient, (0.35, -0.8, 0.25), 2)
    run_frames(p, o, 3)


@pytest.mark.parametrize("mode", [0, 2])
def test_shading_float_channels_and_batches(oracle, mode):
    """Float channels, an axis-aligned light (zero direction components), sample batches."""
    vols = [syn.lognormal(36, 21 + i, octaves=4) for i in range(3)]
    tfs = [syn.ramp_tf(syn.HUES[i], alpha_max=0.8) for i in range(3)]
    p, o = make_pair(oracle, vols, tfs, mode, (4, 6, 5), (41, 33), 5, xf=[(0.0, 0.05)] * 3)
    for r in (p, o):
        _shade(r, True, True, (0.0, 0.0, -1.0), 3)
    p.setTuning(1, 2)   # two samples per batch
    run_frames(p, o, 2)


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 4, 5])
def test_denoiser_features(oracle, mode):
    """Per-pixel denoiser features (radiance, depth, transmittance, channel hit fractions),
    bit for bit, and the accumulation unchanged by turning them on."""
    vols = [noise_u8(40, occ, 50 + i) for i, occ in enumerate([0.15, 0.25, 0.3])]
    tfs = [syn.ramp_tf(syn.HUES[i]) for i in range(3)]
    p, o = make_pair(oracle, vols, tfs, mode, (5, 5, 5), (52, 36), 6)
    for r in (p, o):
        r.setFeatures(True)
    for f in range(2):
        p.Render()
        o.Render()
        assert_same_frame(p, o, f"frame {f}")
        fp, fo = p.features(), o.features()
        np.testing.assert_array_equal(fp.view(np.uint32), fo.view(np.uint32))
    st = p.pixelStats()
    np.testing.assert_allclose(fp[..., 4] * 6 + st[..., 2], 6, atol=1e-5)


@pytest.mark.parametrize("mode,extra", [(0, "stats"), (2, "stats"), (1, ""), (3, "features"), (4, "shade"),
                                        (5, "stats"), (2, "shade")])
def test_render_frames_equals_successive_renders(oracle, mode, extra):
    """mdwt_render_frames(n): n frames traced in one launch give exactly the frames, ids,
    accumulation and counters of n Render calls -- from a fresh context (the reference's
    post-increment ids: frames 0 and 1 share seeds), after a reset, and with
    accumulation off."""
    vols = [noise_u8(40, occ, 60 + i) for i, occ in enumerate([0.2, 0.3])]
    tfs = [syn.ramp_tf(syn.HUES[i]) for i in range(2)]
    p, o = make_pair(oracle, vols, tfs, mode, (5, 5, 5), (41, 35), 2)
    for r in (p, o):
        if extra == "features":
            r.setFeatures(True)
        if extra == "shade":
            _shade(r, True, True, (0.35, -0.8, 0.25), 2)
    for n in (3, 1, 5):
        p.RenderFrames(n)
        o.RenderFrames(n)
        assert_same_frame(p, o, f"{n} frames")
        if extra == "features":
            np.testing.assert_array_equal(p.features().view(np.uint32), o.features().view(np.uint32))
    for r in (p, o):
        r.ResetAccumulation()
        r.setAccumulation(False)
    p.RenderFrames(4)
    o.RenderFrames(4)
    assert_same_frame(p, o, "no accumulation")
    np.testing.assert_array_equal(p.counters(), o.counters())


@pytest.mark.parametrize("mode", [0, 2, 3])
@pytest.mark.parametrize("shadows", [False, True])
def test_thread_block_seeding(oracle, mode, shadows):
    """Seed words from the pixel's position in a 16 x 16 thread block (mdwt_set_seed_block,
    the reference's threadIdx seeding, deviceCode.cu:296-297, 385-386), with and without
    shadow rays, on both trackers, bit for bit; pixels 16 apart share their streams."""
    vols = [noise_u8(40, occ, 60 + i) for i, occ in enumerate([0.2, 0.3])]
    tfs = [syn.ramp_tf(syn.HUES[i], alpha_max=0.9) for i in range(2)]
    p, o = make_pair(oracle, vols, tfs, mode, (5, 5, 5), (50, 38), 3)
    for r in (p, o):
        r.setSeedBlock(16)
        if shadows:
            _shade(r, True, False, (0.35, -0.8, 0.25), 2)
    run_frames(p, o, 2)
    # per-pixel seeding gives another frame
    q, _ = make_pair(oracle, vols, tfs, mode, (5, 5, 5), (50, 38), 3)
    if shadows:
        _shade(q, True, False, (0.35, -0.8, 0.25), 2)
    q.Render()
    q.Render()
    assert not np.array_equal(q.accum(), p.accum())
