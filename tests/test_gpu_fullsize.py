"""Parity at the benchmark's full size (3 x 256^3 uint8, syncDDA, 16^3 macrocells,
1024x1024, 64 spp): the whole range and majorant grids bit-exact, a band of rows of
the full-resolution frame bit-exact against the oracle (the oracle renders only those
rows), and size-independent properties of the whole frame."""
import numpy as np
import pytest

from mdwtracker_b200 import Renderer
from mdwtracker_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2():
    return syn.scene_c2()


def test_c2_fullsize_rows_and_grids(oracle, c2):
    p = c2.setup(Renderer(0))
    o = c2.setup(oracle.OracleRenderer())
    p.enablePixelStats(True)
    o.enablePixelStats(True)
    np.testing.assert_array_equal(p.ranges(), o.ranges())
    np.testing.assert_array_equal(p.majorants(), o.majorants())
    rows = (508, 514)
    p.Render()
    o.renderRows(*rows)
    ap, ao = p.accum(), o.accum()
    np.testing.assert_array_equal(ap[rows[0]:rows[1]].view(np.uint32), ao[rows[0]:rows[1]].view(np.uint32))
    np.testing.assert_array_equal(p.pixelStats()[rows[0]:rows[1]], o.pixelStats()[rows[0]:rows[1]])
    # whole-frame properties
    assert np.all(np.isfinite(ap))
    np.testing.assert_array_equal(ap[..., 3], np.float32(65.0 / 64.0))
    c = p.counters()
    assert c[3] == 1024 * 1024 * 64
    st = p.pixelStats()
    assert int(st[..., 0].sum(dtype=np.uint64)) == int(c[0])
    assert int(st[..., 1].sum(dtype=np.uint64)) == int(c[1])


def test_c2_fullsize_accumulation_is_the_running_mean(c2):
    """Renderer::Render sets the ids of the NEXT frame to the pre-increment counters
    (renderer.cpp:957-958), so frames 1 and 2 use the same seeds and frame 2 overwrites
    frame 1; from then on the buffer is the running mean: after 4 frames (F1+F2+F3)/3."""
    res, spp = (256, 256), 8
    a = c2.setup(Renderer(0), resolution=res, spp=spp)
    frames = []
    for _ in range(4):
        a.ResetAccumulation()
        a.Render()
        frames.append(a.accum().copy())
    np.testing.assert_array_equal(frames[0], frames[1])
    assert not np.array_equal(frames[1], frames[2])
    b = c2.setup(Renderer(0), resolution=res, spp=spp)
    for _ in range(4):
        b.Render()
    acc = b.accum()
    expect = (frames[1].astype(np.float64) + frames[2] + frames[3]) / 3.0
    np.testing.assert_allclose(acc, expect, rtol=2e-6, atol=2e-7)
    assert b.frameIds() == (4, 4, 3, 3)
