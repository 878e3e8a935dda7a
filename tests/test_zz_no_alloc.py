"""mdwt_build_ranges_noalloc: the value-range build for callers that may not allocate
device memory (code inside an application's own memory pool or under an allocator
that forbids cudaMalloc, plug-ins handed buffers and a stream but no allocation
rights).  It must give the same ranges as the normal path (mdwt_init), bit for bit,
on consecutive calls that share its fixed scratch, and refuse sizes beyond that
scratch.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from mdwtracker_b200 import Renderer, load_library
from mdwtracker_b200 import synthetic as syn

pytestmark = pytest.mark.gpu

FMT_UINT8, FMT_FLOAT32 = 4, 7
SCRATCH_LIMIT = 11


def _fn():
    lib = load_library()
    f = lib.mdwt_build_ranges_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int64), C.POINTER(C.c_uint32), C.POINTER(C.c_float),
                  C.POINTER(C.c_float), C.c_void_p, C.c_void_p]
    return f


def _call(f, dvol, fmt, dims, mc, out, stream, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    return f(C.c_void_p(dvol.data_ptr()), fmt, (C.c_int64 * 3)(*dims), (C.c_uint32 * 3)(*mc),
             (C.c_float * 3)(*lo), (C.c_float * 3)(*hi), C.c_void_p(out.data_ptr()),
             C.c_void_p(stream))


def _existing_ranges(vols, mc, reshape=None, box=False):
    """The ranges mdwt_init builds; `reshape` gives each channel's -cb scaling (None:
    unit bounds, "dims": by its dims, or three factors).  With box=True also the grid's
    box, the union of the channel bounds (renderer.cpp:698-716)."""
    r = Renderer(0)
    for v in vols:
        r.PushMesh(v)
    for i, sc in enumerate(reshape or []):
        if sc is not None:
            r.reshapeBounds(i, None if sc == "dims" else sc)
    r.macrocellDims = mc
    r.Resize((8, 8))
    r.Init(2)
    M = mc[0] * mc[1] * mc[2]
    out = r.ranges().reshape(M, len(vols), 2)
    if not box:
        return out
    b = np.array([r.channelInfo(i)[1] for i in range(len(vols))], dtype=np.float32)  # (C, 8)
    lo = tuple(float(x) for x in b[:, 0:3].min(axis=0))
    hi = tuple(float(x) for x in b[:, 4:7].max(axis=0))
    return out, lo, hi


def test_noalloc_ranges_match_the_init_path():
    import torch
    f = _fn()
    mc = (5, 7, 4)
    M = mc[0] * mc[1] * mc[2]
    a = syn.value_noise_sparse(40, 0.3, 11, octaves=3)                       # dims (40, 40, 40)
    b = syn.value_noise_sparse(44, 0.2, 12, octaves=3)[:36, :28, :].copy()   # dims (44, 28, 36)
    ref_u8 = _existing_ranges([a, b], mc)
    c = syn.lognormal(32, 13, octaves=3)
    ref_f32 = _existing_ranges([c], mc)
    stream = torch.cuda.current_stream().cuda_stream
    out = torch.full((2 * M,), float("nan"), dtype=torch.float32, device="cuda")
    calls = [(a, FMT_UINT8, ref_u8[:, 0]), (b, FMT_UINT8, ref_u8[:, 1]), (c, FMT_FLOAT32, ref_f32[:, 0])]
    for vol, fmt, ref in calls:          # consecutive calls share the scratch
        dvol = torch.from_numpy(np.ascontiguousarray(vol)).cuda()
        dims = (vol.shape[2], vol.shape[1], vol.shape[0])
        assert _call(f, dvol, fmt, dims, mc, out, stream) == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(M, 2)
        np.testing.assert_array_equal(got, ref)


def test_noalloc_ranges_match_the_init_path_with_reshaped_bounds():
    """-cb bounds (raw::RawR::reshapeBounds, rawFile.cpp:217-237): by the dims, by uneven
    factors, and two channels whose union box is larger than either channel's own box;
    plus an axis of 2^20 voxels, whose voxel size is below 1e-6 of the box."""
    import torch
    f = _fn()
    stream = torch.cuda.current_stream().cuda_stream
    a = syn.value_noise_sparse(40, 0.3, 21, octaves=3)
    b = syn.value_noise_sparse(44, 0.2, 22, octaves=3)[:36, :28, :].copy()
    c = syn.lognormal(32, 23, octaves=3)
    long_axis = (np.arange(1 << 21, dtype=np.uint32) * 2654435761 >> 24).astype(np.uint8).reshape(2, 1, 1 << 20)
    cases = [([a], (5, 7, 4), ["dims"], FMT_UINT8),
             ([c], (3, 8, 6), [(1000.5, 0.003, 7.25)], FMT_FLOAT32),
             ([a, b], (6, 5, 7), [(3.0, 1.5, 0.75), "dims"], FMT_UINT8),
             ([long_axis], (1024, 1, 2), None, FMT_UINT8)]
    for vols, mc, reshape, fmt in cases:
        ref, lo, hi = _existing_ranges(vols, mc, reshape, box=True)
        M = mc[0] * mc[1] * mc[2]
        out = torch.full((2 * M,), float("nan"), dtype=torch.float32, device="cuda")
        for i, vol in enumerate(vols):
            dvol = torch.from_numpy(np.ascontiguousarray(vol)).cuda()
            dims = (vol.shape[2], vol.shape[1], vol.shape[0])
            for _ in range(2):   # two calls in a row on the shared scratch
                out.fill_(float("nan"))
                assert _call(f, dvol, fmt, dims, mc, out, stream, lo, hi) == 0
                torch.cuda.synchronize()
                np.testing.assert_array_equal(out.cpu().numpy().reshape(M, 2), ref[:, i])


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    f = _fn()
    vol = torch.zeros(4 * 8 * 8, dtype=torch.uint8, device="cuda")
    out = torch.empty(2 * 2048 * 2, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert _call(f, vol, FMT_UINT8, (8, 8, 4), (2048, 1, 1), out, stream) == SCRATCH_LIMIT
    big = torch.zeros(2, dtype=torch.uint8, device="cuda")
    assert _call(f, big, FMT_UINT8, (1024, 1024, 2), (1024, 1024, 1), out, stream) == SCRATCH_LIMIT
