"""libmdwt's value ranges and majorants against the reference's own kernels, run on the
GPU: the range raster of buildSpatialMacrocells (sizeMCs + rasterElements, renderer.cu:
280-347, 387-403, 487-519, 835-893, 1116-1179) and the majorant pass of
RecalculateDensityRanges (_recalculateDensityRangesMM and the summed
_recalculateDensityRanges, renderer.cu:111-274), whose texel fetches and probes run on the
B200's texture unit over a transfer-function texture made as Renderer::SetXFColormap
makes it (renderer.cpp:1094-1165).

`make -C oracle ref` builds oracle/_ref/libref_gpu.so from oracle/ref_gpu_pins.cu, which
includes the reference's renderer.cu unchanged (nvcc, the reference build's default
flags).  The CPU oracle's ranges and majorants equal libmdwt's bit for bit (the other
GPU tests), so these cases pin all three to the reference.  The tests skip where the
library was not built (no reference sources)."""
import ctypes as C
import os

import numpy as np
import pytest

from mdwtracker_b200 import Renderer
from mdwtracker_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_GPU = os.path.join(ROOT, "oracle", "_ref", "libref_gpu.so")
FP = C.POINTER(C.c_float)


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF_GPU):
        pytest.skip("oracle/_ref/libref_gpu.so not built (make -C oracle ref)")
    lib = C.CDLL(REF_GPU)
    lib.refgpu_majorants.argtypes = [C.c_int, FP, C.c_int, C.c_int, FP, C.c_int, FP, FP, FP, FP]
    lib.refgpu_ranges.argtypes = [FP, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int), FP, FP, FP]
    return lib


def fp(a):
    return a.ctypes.data_as(FP)


def scene(vols, tfs, mc, mode, xf=None, os_=None, reshape=False):
    r = Renderer(0)
    for v in vols:
        r.PushMesh(v)
    if reshape:
        for i in range(len(vols)):
            r.reshapeBounds(i)
    r.macrocellDims = mc
    r.Resize((16, 16))
    r.Init(mode)
    for i, tf in enumerate(tfs):
        r.SetXFColormap(tf, i)
        r.SetXFOpacityScale(1.0 if os_ is None else os_[i], i)
        r.SetXFRange((0.0, 1.0) if xf is None else xf[i], i)
    return r


def ref_scalars(v):
    """The floats the reference's RawR makes of a volume (uint8: v * 255, rawFile.cpp:103-105)."""
    return v.astype(np.float32) * np.float32(255.0) if v.dtype == np.uint8 else v.astype(np.float32)


def ref_ranges(ref, r, vols):
    C_ = len(vols)
    mc = np.array(r.macrocellDims, dtype=np.int32)
    dims = np.array([[v.shape[2], v.shape[1], v.shape[0]] for v in vols], dtype=np.int32)
    scal = np.concatenate([ref_scalars(v).ravel() for v in vols])
    b = [r.channelInfo(i)[1] for i in range(C_)]
    lo = np.array([min(x[a] for x in b) for a in range(3)], dtype=np.float32)
    hi = np.array([max(x[4 + a] for x in b) for a in range(3)], dtype=np.float32)
    out = np.empty(int(mc.prod()) * C_ * 2, dtype=np.float32)
    assert ref.refgpu_ranges(fp(scal), dims.ctypes.data_as(C.POINTER(C.c_int)), C_,
                             mc.ctypes.data_as(C.POINTER(C.c_int)), fp(lo), fp(hi), fp(out)) == 0
    return out.reshape(-1, 2)


def ref_majorants(ref, r, tfs, xf, os_, summed):
    C_ = r.numChannels
    rg = np.ascontiguousarray(r.ranges(), dtype=np.float32)
    M = rg.shape[0] // C_
    n = tfs[0].shape[0]
    tfa = np.ascontiguousarray(np.stack([np.asarray(t, np.float32).reshape(n, 4) for t in tfs]))
    vd = np.array([[r.channelInfo(i)[1][3], r.channelInfo(i)[1][7]] for i in range(C_)], dtype=np.float32)
    xd = np.array([(0.0, 1.0) if xf is None else xf[i] for i in range(C_)], dtype=np.float32)
    osc = np.array([1.0 if os_ is None else os_[i] for i in range(C_)], dtype=np.float32)
    out = np.empty(M if summed else M * C_, dtype=np.float32)
    assert ref.refgpu_majorants(1 if summed else 0, fp(rg), M, C_, fp(tfa), n, fp(vd), fp(xd), fp(osc), fp(out)) == 0
    return out


def assert_bits(a, b, what):
    a, b = np.ascontiguousarray(a, np.float32), np.ascontiguousarray(b, np.float32)
    assert a.shape == b.shape and np.any(a != 0), what   # not vacuous
    bad = np.flatnonzero(a.view(np.uint32).ravel() != b.view(np.uint32).ravel())
    assert not len(bad), f"{what}: {len(bad)} of {a.size} differ, first at {bad[0]}: {a.ravel()[bad[0]]} vs {b.ravel()[bad[0]]}"


def c2_like(n=48):
    vols = [syn.value_noise_sparse(n, occ, 10 + i, octaves=3) for i, occ in enumerate([0.1, 0.2, 0.3])]
    return vols, [syn.ramp_tf(syn.HUES[i]) for i in range(3)]


def c3_like(n=40, k=4):
    vols = [syn.lognormal_log10(n, 60 + i, octaves=3) for i in range(k)]
    return vols, [syn.ramp_tf(syn.HUES[i % len(syn.HUES)], alpha_max=0.25, start=0.5) for i in range(k)]


@pytest.mark.parametrize("mode", [2, 0, 3])
def test_uint8_scene(ref, mode):
    vols, tfs = c2_like()
    r = scene(vols, tfs, (6, 6, 6), mode)
    assert_bits(r.ranges(), ref_ranges(ref, r, vols), "ranges")
    assert_bits(r.majorants(), ref_majorants(ref, r, tfs, None, None, mode >= 3), "majorants")


@pytest.mark.parametrize("mode", [2, 3])
def test_float32_scene_with_tf_ranges_and_opacity_scales(ref, mode):
    vols, tfs = c3_like()
    xf = [(0.0, 0.05), (0.2, 0.7), (-0.3, 1.4), (0.45, 0.55)]
    osc = [0.5, 2.0, 1.0, 37.0]
    r = scene(vols, tfs, (5, 8, 4), mode, xf=xf, os_=osc)
    assert_bits(r.ranges(), ref_ranges(ref, r, vols), "ranges")
    assert_bits(r.majorants(), ref_majorants(ref, r, tfs, xf, osc, mode >= 3), "majorants")


def test_odd_texel_count_and_reshaped_bounds(ref):
    """100-texel transfer functions (texel centres that are not dyadic in normalized
    coordinates) and -cb bounds (the world box scaled to the voxel grid), a non-cubic volume."""
    rng = np.random.default_rng(5)
    vols = [syn.lognormal_log10(32, 70 + i, octaves=3)[:, :24, :] .copy() for i in range(2)]
    tfs = []
    for i in range(2):
        t = np.zeros((100, 4), np.float32)
        t[:, :3] = syn.HUES[i]
        t[:, 3] = rng.random(100).astype(np.float32)
        tfs.append(t)
    r = scene(vols, tfs, (4, 3, 5), 2, reshape=True)
    assert_bits(r.ranges(), ref_ranges(ref, r, vols), "ranges")
    assert_bits(r.majorants(), ref_majorants(ref, r, tfs, None, None, False), "majorants")


def test_c2_full_size(ref):
    """The benchmarked uint8 scene: 3 x 256^3, 16-voxel macrocells."""
    sc = syn.scene_c2()
    r = sc.setup(Renderer(0))
    assert_bits(r.ranges(), ref_ranges(ref, r, sc.volumes), "ranges")
    assert_bits(r.majorants(), ref_majorants(ref, r, sc.tfs, None, None, False), "majorants")


def texture_probe_coords(rng, n, shape):
    """Random normalized coordinates, plus texel centres, texel edges, the clamp region
    outside [0, 1] and coordinates one ulp beside texel centres (n of each)."""
    u = rng.random((n, len(shape)), dtype=np.float32)
    cen = np.stack([(rng.integers(0, s, n) + 0.5) / s for s in shape], axis=1).astype(np.float32)
    edge = np.stack([rng.integers(0, s + 1, n) / s for s in shape], axis=1).astype(np.float32)
    out = (rng.random((n, len(shape)), dtype=np.float32) * 1.4 - 0.2).astype(np.float32)
    near = np.nextafter(cen, np.where(rng.random(cen.shape) < 0.5, np.float32(2), np.float32(-1))).astype(np.float32)
    return np.ascontiguousarray(np.concatenate([u, cen, edge, out, near]).astype(np.float32))


def test_texture_unit_against_the_filter_statement(oracle, ref):
    """The B200's texture unit, with the reference's descriptors, against the oracle's
    statement of linear filtering (8 fractional weight bits, clamp, fmaf lerp, x then y
    then z), which the kernels and the host pins use: tex3D<float> on a float volume and
    tex2D<float4> on a transfer-function array.

    Measured: at texel centres, at texel edges (weight 1/2) and one ulp beside centres
    the two agree to the last bits of the blend; at random coordinates the hardware's
    weights differ from round(frac * 256) / 256 by up to about 1.5 steps of 1/256, so a
    filtered value differs by at most 2/256 of the spread of the texels it blends.  The
    reference's own run on the GPU therefore draws a statistically equal, not an
    identical, random walk; the project keeps the documented rule, which the CPU can
    restate."""
    lib = oracle.load_oracle()
    lib.orc_sample_tex3d.argtypes = [FP, C.POINTER(C.c_int), FP, C.c_int, FP]
    lib.orc_sample_tex2d.argtypes = [FP, C.c_int, FP, C.c_int, FP]
    ref.refgpu_tex3d.argtypes = [FP, C.c_int, C.c_int, C.c_int, FP, C.c_int, FP]
    ref.refgpu_tex2d.argtypes = [FP, C.c_int, FP, C.c_int, FP]
    rng = np.random.default_rng(11)
    X, Y, Z = 37, 29, 23
    vol = np.ascontiguousarray(rng.standard_normal((Z, Y, X)).astype(np.float32) * 100)
    groups = 5   # random, centres, edges, outside [0, 1], one ulp beside centres
    xyz = texture_probe_coords(rng, 40000, (X, Y, Z))
    n = xyz.shape[0]
    hw, sw = np.empty(n, np.float32), np.empty(n, np.float32)
    dims = np.array([X, Y, Z], np.int32)
    assert ref.refgpu_tex3d(fp(vol), X, Y, Z, fp(xyz), n, fp(hw)) == 0
    lib.orc_sample_tex3d(fp(vol), dims.ctypes.data_as(C.POINTER(C.c_int)), fp(xyz), n, fp(sw))
    # the spread of the eight texels each sample blends
    ix = [np.clip(np.floor(xyz[:, a].astype(np.float64) * d - 0.5).astype(np.int64) + o, 0, d - 1)
          for a, d in enumerate((X, Y, Z)) for o in (0, 1)]
    corners = np.stack([vol[ix[4 + k], ix[2 + j], ix[i]] for i in (0, 1) for j in (0, 1) for k in (0, 1)], 1)
    spread = corners.max(1).astype(np.float64) - corners.min(1)
    err = np.abs(hw.astype(np.float64) - sw)
    rel = err / np.maximum(spread, 1e-30)
    per = err.reshape(groups, -1)
    print("tex3D: share within float rounding (random, centres, edges, outside, near):",
          np.round(np.mean(per <= 1e-3, axis=1), 4), "largest error / texel spread:", float(rel.max()))
    assert per[1].max() <= 1e-3 and per[2].max() <= 1e-3 and per[4].max() <= 1e-3   # centres, edges, near
    assert rel.max() <= 2.0 / 256
    assert np.all((hw >= corners.min(1) - 1e-3) & (hw <= corners.max(1) + 1e-3))
    N = 100
    tf = np.ascontiguousarray(rng.random((N, 4), dtype=np.float32))
    uv = texture_probe_coords(rng, 40000, (N, 1))
    m = uv.shape[0]
    hw2, sw2 = np.empty((m, 4), np.float32), np.empty((m, 4), np.float32)
    assert ref.refgpu_tex2d(fp(tf), N, fp(uv), m, fp(hw2)) == 0
    lib.orc_sample_tex2d(fp(tf), N, fp(uv), m, fp(sw2))
    x = np.floor(uv[:, 0].astype(np.float64) * N - 0.5).astype(np.int64)
    i0, i1 = np.clip(x, 0, N - 1), np.clip(x + 1, 0, N - 1)
    spread2 = np.abs(tf[i1] - tf[i0]).astype(np.float64)
    err2 = np.abs(hw2.astype(np.float64) - sw2)
    rel2 = err2 / np.maximum(spread2, 1e-30)
    print("tex2D: share identical", float(np.mean(err2 == 0)), "largest error / texel spread:",
          float(rel2[spread2 > 0].max()))
    assert rel2[spread2 > 0].max() <= 2.0 / 256
    assert np.all(err2[spread2 == 0] <= 1e-6)
