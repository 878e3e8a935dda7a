"""The oracle against the reference's own tracking program: mainRG and the closest-hit
trackers of deviceCode.cu, compiled where they lie and run on the host.

`make -C oracle ref` builds oracle/_ref/libref_track.so from oracle/ref_track_pins.cpp,
which includes the reference's deviceCode.cu unchanged and supplies the OptiX SDK, OWL
and CUDA names it uses with the stand-ins of oracle/ref_shim (a host-side pipeline for
traceRay, the CUDA texture unit's linear filter, this project's generator stream, log and
RGBA8 packing).  Each case sets a scene up in the oracle, hands the oracle's launch state
(majorants, camera basis, dt, bounds, transfer functions, voxels, frame and accumulation
ids) to the reference's mainRG for every frame, and compares the accumulation buffer
(float4) and the RGBA8 framebuffer bit for bit.  The tests skip where the reference
sources are absent."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from mdwtracker_b200 import synthetic as syn

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
REF_LIB = os.path.join(ORACLE_DIR, "_ref", "libref_track.so")


class RefScene(C.Structure):
    _fields_ = [("W", C.c_int), ("H", C.c_int), ("C", C.c_int),
                ("mode", C.c_int), ("spp", C.c_int), ("accumulate", C.c_int), ("shadows", C.c_int),
                ("gradient", C.c_int),
                ("vol", C.c_void_p * 12), ("dims", (C.c_int * 3) * 12), ("tf", C.c_void_p * 12),
                ("tfN", C.c_int * 12), ("vd", (C.c_float * 2) * 12), ("xd", (C.c_float * 2) * 12),
                ("os", C.c_float * 12), ("material", (C.c_float * 7) * 12),
                ("majorants", C.c_void_p), ("mc", C.c_uint * 3),
                ("lastLo", C.c_float * 4), ("lastHi", C.c_float * 4),
                ("rootLo", C.c_float * 4), ("rootHi", C.c_float * 4),
                ("dt", C.c_float), ("cam", C.c_float * 12),
                ("lightDir", C.c_float * 3), ("lightIntensity", C.c_float), ("ambient", C.c_float),
                ("bg", C.c_float * 3)]


@pytest.fixture(scope="module")
def ref():
    r = subprocess.run(["make", "-C", ORACLE_DIR, "ref"], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    if r.returncode != 0 and not os.path.exists(REF_LIB):
        pytest.skip("the reference sources are not available to build oracle/_ref")
    lib = C.CDLL(REF_LIB)
    lib.ref_set_seed_block.argtypes = [C.c_int]
    lib.ref_mainrg_frame.restype = C.c_int
    lib.ref_mainrg_frame.argtypes = [C.POINTER(RefScene), C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                     C.c_int, C.c_int]
    return lib


class RefLaunch:
    """The reference's mainRG driven with the launch state of an oracle renderer."""

    def __init__(self, lib, o):
        self.lib, self.o = lib, o
        L = o._lib
        f = (C.c_float * 23)()
        i = (C.c_int * 8)()
        assert L.orc_get_launch_state(o._ctx, f, i) == 0
        f, i = list(f), list(i)
        self.W, self.H, nc = i[5], i[6], i[7]
        s = RefScene()
        s.W, s.H, s.C = self.W, self.H, nc
        s.mode, s.spp, s.accumulate, s.shadows, s.gradient = i[0], i[1], i[2], i[3], i[4]
        s.dt = f[0]
        s.rootLo[:] = f[1:4] + [0.0]
        s.rootHi[:] = f[4:7] + [0.0]
        s.lastLo[:] = f[7:11]
        s.lastHi[:] = f[11:15]
        s.bg[:] = f[15:18]
        s.lightDir[:] = f[18:21]
        s.lightIntensity, s.ambient = f[21], f[22]
        self.keep = []
        for c in range(nc):
            dims, _ = o.channelInfo(c)
            n = int(dims[0] * dims[1] * dims[2])
            vol = np.empty(n, dtype=np.float32)
            assert L.orc_get_channel_data(o._ctx, c, vol.ctypes.data_as(C.POINTER(C.c_float))) == 0
            self.keep.append(vol)
            s.vol[c] = vol.ctypes.data
            s.dims[c][:] = [int(d) for d in dims]
            n_t = C.c_int()
            vd, xd, osc = (C.c_float * 2)(), (C.c_float * 2)(), C.c_float()
            assert L.orc_get_tf(o._ctx, c, None, 0, C.byref(n_t), vd, xd, C.byref(osc)) == 0
            tf = np.empty(4 * n_t.value, dtype=np.float32)
            assert L.orc_get_tf(o._ctx, c, tf.ctypes.data_as(C.POINTER(C.c_float)), n_t.value, C.byref(n_t), vd, xd,
                                C.byref(osc)) == 0
            self.keep.append(tf)
            s.tf[c] = tf.ctypes.data
            s.tfN[c] = n_t.value
            s.vd[c][:] = list(vd)
            s.xd[c][:] = list(xd)
            s.os[c] = osc.value
            m = (C.c_float * 7)()
            assert L.orc_get_material(o._ctx, c, m) == 0
            s.material[c][:] = list(m)
        maj = o.majorants().astype(np.float32).ravel()
        self.keep.append(maj)
        s.majorants = maj.ctypes.data
        s.mc[:] = [int(x) for x in o.macrocellDims]
        s.cam[:] = [float(x) for x in o.cameraBasis().ravel()]
        self.s = s
        self.accum = np.zeros((self.H, self.W, 4), dtype=np.float32)
        self.fb = np.zeros((self.H, self.W), dtype=np.uint32)

    def frame(self, row0=0, stride=1):
        ids = self.o.frameIds()   # (frameID, accumID, the next launch's frameID, accumID)
        rc = self.lib.ref_mainrg_frame(C.byref(self.s), ids[2], ids[3], self.accum.ctypes.data, self.fb.ctypes.data,
                                       row0, stride, len(os.sched_getaffinity(0)))
        assert rc == 0


def setup(oracle, vols, tfs, mode, mc, res, spp, opacity=None, xf=None, camera=None, light=None, mats=None,
          bg=None, dt=None):
    o = oracle.OracleRenderer()
    for v in vols:
        o.PushMesh(v)
    o.macrocellDims = mc
    o.Resize(res)
    o.Init(mode, camera is None)
    if camera is not None:
        o.setCamera(*camera)
    if dt is not None:
        o.Setdt(dt)
    for i, tf in enumerate(tfs):
        o.SetXFColormap(tf, i)
        o.SetXFOpacityScale(1.0 if opacity is None else opacity[i], i)
        o.SetXFRange((0.0, 1.0) if xf is None else xf[i], i)
    if light is not None:
        o.setLight(*light)
    if mats is not None:
        for i, m in enumerate(mats):
            o.setMaterial(i, *m)
    if bg is not None:
        o.setBackground(bg)
    o.setSpp(spp)
    return o


# The host compiler contracts a*b + c*d as fma(a, b, c*d) where the oracle (following nvcc)
# writes fma(c, d, a*b); the colour sums of the shading and a few dot products can then
# differ in the last bit.  Alpha (the hit count of every pixel) must be identical, and the
# rest within these bounds.
MIN_IDENTICAL = 0.90
MAX_ABS_DIFF = 5e-4


def assert_pinned(lib, o, frames=2, between=None):
    r = RefLaunch(lib, o)
    for f in range(frames):
        if between is not None:
            between(f, o, r)
        r.frame()
        o.Render()
        ao = o.accum()
        np.testing.assert_array_equal(ao[..., 3], r.accum[..., 3])
        same = np.all(ao.view(np.uint32) == r.accum.view(np.uint32), axis=-1)
        assert same.mean() >= MIN_IDENTICAL, f"frame {f}: only {same.mean():.4f} of the pixels are identical"
        assert float(np.abs(ao - r.accum).max()) <= MAX_ABS_DIFF
    return r


def noise_u8(n, occ, seed):
    return syn.value_noise_sparse(n, occ, seed, octaves=3)


@pytest.mark.parametrize("mode", [0, 1, 2, 3, 4, 5])
def test_methods_uint8(oracle, ref, mode):
    vols = [noise_u8(32, occ, 40 + i) for i, occ in enumerate([0.15, 0.25, 0.3])]
    tfs = [syn.ramp_tf(syn.HUES[i]) for i in range(3)]
    o = setup(oracle, vols, tfs, mode, (4, 4, 4), (48, 40), 3)
    assert_pinned(ref, o)


@pytest.mark.parametrize("mode", [0, 2])
def test_float32_tf_ranges_and_opacity(oracle, ref, mode):
    vols = [syn.lognormal(28, 60 + i, octaves=3) for i in range(4)]
    tfs = [syn.ramp_tf(syn.HUES[i], alpha_max=0.7, start=0.2) for i in range(4)]
    o = setup(oracle, vols, tfs, mode, (5, 3, 4), (40, 30), 4, opacity=[1.0, 0.5, 2.0, 1.5],
              xf=[(0.0, 0.05), (0.01, 0.2), (0.0, 1.0), (0.02, 0.08)])
    assert_pinned(ref, o)


def test_off_axis_camera_and_background(oracle, ref):
    vols = [noise_u8(36, 0.3, 70), noise_u8(36, 0.2, 71)]
    tfs = [syn.ramp_tf(syn.HUES[i]) for i in range(2)]
    cam = ((1.9, 0.7, 2.2), (0.45, 0.55, 0.4), (0.0, 1.0, 0.0), 38.0)
    o = setup(oracle, vols, tfs, 2, (6, 6, 6), (45, 37), 2, camera=cam, bg=(0.2, 0.3, 0.4))
    assert_pinned(ref, o, frames=3)


@pytest.mark.parametrize("mode", [0, 2])
def test_shadows_and_gradient_shading(oracle, ref, mode):
    vols = [noise_u8(32, 0.3, 80), noise_u8(32, 0.25, 81)]
    tfs = [syn.ramp_tf(syn.HUES[i]) for i in range(2)]
    o = setup(oracle, vols, tfs, mode, (4, 4, 4), (40, 32), 2, light=(True, True, (0.3, -1.0, 0.2), 1.2, 0.15),
              mats=[(0.8, 0.4, 16.0, 0.01, (1.0, 0.9, 0.8)), (0.6, 0.2, 4.0, 0.02, (0.7, 0.8, 1.0))])
    assert_pinned(ref, o)


@pytest.mark.parametrize("mode", [0, 2])
def test_thread_block_seeding(oracle, ref, mode):
    """With 16 x 16 thread-block seeding (mdwt_set_seed_block), the reference's own
    LCG<4>(threadIdx.x + seed, threadIdx.y + seed) and shadow-ray seeding (deviceCode.cu:
    296-297, 385-386) run with threadIdx = the pixel's position in its block."""
    vols = [noise_u8(32, 0.3, 85), noise_u8(32, 0.25, 86)]
    tfs = [syn.ramp_tf(syn.HUES[i]) for i in range(2)]
    o = setup(oracle, vols, tfs, mode, (4, 4, 4), (40, 34), 2, light=(True, False, (0.3, -1.0, 0.2), 1.2, 0.15))
    o.setSeedBlock(16)
    ref.ref_set_seed_block(16)
    try:
        assert_pinned(ref, o)
    finally:
        ref.ref_set_seed_block(0)


def test_accumulation_off_and_frame_ids(oracle, ref):
    """Frames with accumulation off, then on after a reset: the ids each launch sees are
    the pre-increment counters (renderer.cpp:957-958)."""
    vols = [noise_u8(24, 0.3, 90)]
    tfs = [syn.viridis_like()]
    o = setup(oracle, vols, tfs, 0, (3, 3, 3), (32, 24), 2)

    def between(f, o, r):
        o.setAccumulation(f >= 2)
        r.s.accumulate = int(f >= 2)
        if f == 2:
            o.ResetAccumulation()

    assert_pinned(ref, o, frames=4, between=between)
