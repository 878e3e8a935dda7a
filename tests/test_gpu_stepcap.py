"""Paths that reach the per-sample step cap (2^22 Woodcock draws, a bound the reference
does not have: its loop would spin until the flight's sum leaves the cell, which a huge
majorant prevents) end as misses on the GPU exactly as in the oracle, in both trackers.

Scene: one 16^3 float32 channel of zeros with a single voxel of 1.0, 2^3 macrocells, a
transfer function opaque only at its last texel and an opacity scale of 1e30.  The
macrocell around the voxel gets the majorant 1e30, so a free flight there is shorter than
the last bit of t: a path that enters the cell where the density maps to zero opacity
draws, samples and rejects at the same point until the cap ends it."""
import numpy as np
import pytest

from mdwtracker_b200 import MdwtError, Renderer

pytestmark = pytest.mark.gpu

TUNE_REGROUP = 4


def setup(r):
    v = np.zeros((16, 16, 16), np.float32)
    v[5, 5, 5] = 1.0
    r.PushMesh(v)
    r.macrocellDims = (2, 2, 2)
    r.Resize((12, 10))
    r.Init(2)
    tf = np.zeros((256, 4), np.float32)
    tf[:, :3] = 1.0
    tf[255, 3] = 1.0
    r.SetXFColormap(tf, 0)
    r.SetXFOpacityScale(1e30, 0)
    r.SetXFRange((0.0, 1.0), 0)
    r.setSpp(1)
    return r


def counters_status(r):
    try:
        r.counters()
        return 0
    except MdwtError as e:
        return e.status


@pytest.mark.parametrize("regroup", [1, 0])
def test_capped_paths_match_the_oracle(oracle, regroup):
    p = setup(Renderer(0))
    p.setTuning(TUNE_REGROUP, regroup)
    o = setup(oracle.OracleRenderer())
    assert p.majorants().max() == np.float32(1e30)
    p.Render()
    o.Render()
    assert (p.renderInfo()[3] == 256) == (regroup == 1)
    np.testing.assert_array_equal(p.accum().view(np.uint32), o.accum().view(np.uint32))
    np.testing.assert_array_equal(p.framebuffer(), o.framebuffer())
    # five samples reached the cap: the GPU reports it (MDWT_ERR_NUMERIC from
    # mdwt_get_counters), the oracle counts the same samples
    assert counters_status(p) == 10
    assert o.cappedSamples() == 5
