"""Parity at the benchmarked sizes, on the kernels the benchmark runs.

Each case sets up the configured scene at its full size in both renderers, renders
whole frames on the GPU and a set of rows spread over the frame in the oracle, and
compares those rows bit for bit: the accumulation buffer (float4) and the RGBA8
framebuffer.  With per-pixel statistics off, syncDDA and N-DDA frames run the regrouped
tracker (trace_regroup_kernel, launched as 256-thread blocks) -- the kernel `bench.py` times; a
second frame with statistics on runs the warp-local tracker and also compares the
per-pixel event counts (density samples, rejections, hits, hit channels).  The
per-pixel loop both follow is the reference's mainRG and its closest-hit trackers
(deviceCode.cu:283-471, 747-970).

  * C1: 1 x 64^3 uint8, 8^3-voxel macrocells, N-DDA, 512^2, 16 frames of 1 spp in one
    launch (mdwt_render_frames), the whole frame;
  * C2: 3 x 256^3 uint8, 16^3-voxel macrocells, syncDDA, 1024^2, 64 spp;
  * C3: 6 x 512^3 float32, 16-voxel macrocells, 1920x1080, 256 spp, syncDDA and N-DDA;
  * C3b: 3 x 1024^3 float32 (12 GB), syncDDA, 1920x1080, 16 spp;
  * a uint8 channel of more than 2^32 voxels (64-bit voxel offsets), syncDDA.
"""
import os

import numpy as np
import pytest

from mdwtracker_b200 import Renderer
from mdwtracker_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

REGROUP_BLOCK = 256


@pytest.fixture(scope="module")
def orc(oracle):
    oracle.set_threads(len(os.sched_getaffinity(0)))
    return oracle


def same_rows(p, o, rows, tag):
    ap, ao = p.accum()[rows], o.accum()[rows]
    bad = np.argwhere(np.any(ap.view(np.uint32) != ao.view(np.uint32), axis=-1))
    assert not len(bad), f"{tag}: {len(bad)} pixels differ, first (row {rows[bad[0][0]]}, x {bad[0][1]})"
    np.testing.assert_array_equal(p.framebuffer()[rows], o.framebuffer()[rows])
    assert p.frameIds() == o.frameIds()


def spread(o, h, stride):
    """Render one oracle frame over every stride-th row from stride // 2; the row indices."""
    r0 = stride // 2
    n = o.renderRowStride(r0, stride)
    return np.arange(r0, r0 + n * stride, stride)


def regrouped_then_warp_local(p, o, spp, stride, tag, expect_regroup=True):
    """Frame 1 with statistics off (the benchmarked tracker), frame 2 with statistics on
    (the warp-local tracker), both compared on the same spread rows."""
    w, h = p.fbSize
    p.enablePixelStats(False)
    p.Render()
    assert (p.renderInfo()[3] == REGROUP_BLOCK) == expect_regroup
    rows = spread(o, h, stride)
    same_rows(p, o, rows, f"{tag} frame 1")
    p.enablePixelStats(True)
    o.enablePixelStats(True)
    p.Render()
    assert p.renderInfo()[3] != REGROUP_BLOCK
    rows = spread(o, h, stride)
    same_rows(p, o, rows, f"{tag} frame 2")
    np.testing.assert_array_equal(p.pixelStats()[rows], o.pixelStats()[rows])
    # whole-frame properties of the GPU frame
    ap = p.accum()
    assert np.all(np.isfinite(ap))
    c = p.counters()
    assert 0 < c[3] <= 2 * w * h * spp


def test_c1_exactly_as_configured(orc):
    sc = syn.scene_c1()
    p = sc.setup(Renderer(0))
    o = sc.setup(orc.OracleRenderer())
    np.testing.assert_array_equal(p.majorants(), o.majorants())
    p.RenderFrames(sc.frames)
    o.RenderFrames(sc.frames)
    np.testing.assert_array_equal(p.accum().view(np.uint32), o.accum().view(np.uint32))
    np.testing.assert_array_equal(p.framebuffer(), o.framebuffer())
    np.testing.assert_array_equal(p.counters(), o.counters())
    assert p.counters()[3] == 512 * 512 * 16
    p.close()


def test_c2_full_size_on_the_benchmarked_tracker(orc):
    sc = syn.scene_c2()
    p = sc.setup(Renderer(0))
    o = sc.setup(orc.OracleRenderer())
    np.testing.assert_array_equal(p.ranges(), o.ranges())
    np.testing.assert_array_equal(p.majorants(), o.majorants())
    regrouped_then_warp_local(p, o, sc.spp, 16, "c2")
    p.close()


@pytest.fixture(scope="module")
def c3_scenes():
    return {m: syn.scene_c3(mode=m) for m in (2, 0)}


@pytest.mark.parametrize("mode", [2, 0])
def test_c3_full_size(orc, c3_scenes, mode):
    sc = c3_scenes[mode]
    assert sc.resolution == (1920, 1080) and sc.spp == 256 and sc.macrocells == (32, 32, 32)
    p = sc.setup(Renderer(0))
    p.setTuning(4, 1)   # the regrouped tracker for N-DDA too (its default there is the warp-local one)
    o = sc.setup(orc.OracleRenderer())
    np.testing.assert_array_equal(p.ranges(), o.ranges())
    np.testing.assert_array_equal(p.majorants(), o.majorants())
    regrouped_then_warp_local(p, o, sc.spp, 72, f"c3 -m {mode}")
    p.close()


def test_c3b_twelve_gigabytes(orc):
    sc = syn.scene_c3b(mode=2)
    assert sum(v.nbytes for v in sc.volumes) == 3 * 4 * 1024 ** 3
    p = sc.setup(Renderer(0), spp=16)
    o = sc.setup(orc.OracleRenderer(), spp=16)
    np.testing.assert_array_equal(p.majorants(), o.majorants())
    regrouped_then_warp_local(p, o, 16, 90, "c3b")
    p.close()


def test_sixty_four_bit_voxel_offsets(orc):
    """One uint8 channel of 2048 x 2048 x 1040 voxels (4.36 G > 2^32): offsets past 2^32
    are reached wherever a sample lies above z = 1024 voxels, which is where the default
    camera's rays enter."""
    X, Y, Z = 2048, 2048, 1040
    x = np.arange(X, dtype=np.int32)
    y = np.arange(Y, dtype=np.int32)
    z = np.arange(Z, dtype=np.int32)
    fx = ((x * 37) % 97).astype(np.uint8)
    fy = ((y * 53) % 89).astype(np.uint8)
    fz = ((z * 29) % 71).astype(np.uint8)
    vol = np.empty((Z, Y, X), dtype=np.uint8)
    for k in range(Z):   # (fx + fy + fz) with sparse zeros, one slab at a time
        s = fx[None, :] + fy[:, None] + fz[k]
        s[s < 120] = 0
        vol[k] = s
    tf = syn.ramp_tf(syn.HUES[0], alpha_max=0.5)
    sc = syn.Scene("u8_2048x2048x1040", [vol], [tf], mode=2, macrocells=(64, 64, 32),
                   resolution=(640, 480), spp=8)
    p = sc.setup(Renderer(0))
    o = sc.setup(orc.OracleRenderer())
    np.testing.assert_array_equal(p.majorants(), o.majorants())
    regrouped_then_warp_local(p, o, sc.spp, 12, "64-bit offsets")
    # the frame has hits: the offsets past 2^32 were read
    assert p.counters()[0] > 0
    p.close()
