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


def _call(f, dvol, fmt, dims, mc, out, stream):
    return f(C.c_void_p(dvol.data_ptr()), fmt, (C.c_int64 * 3)(*dims), (C.c_uint32 * 3)(*mc),
             (C.c_float * 3)(0.0, 0.0, 0.0), (C.c_float * 3)(1.0, 1.0, 1.0), C.c_void_p(out.data_ptr()),
             C.c_void_p(stream))


def _existing_ranges(vols, mc):
    r = Renderer(0)
    for v in vols:
        r.PushMesh(v)
    r.macrocellDims = mc
    r.Resize((8, 8))
    r.Init(2)
    M = mc[0] * mc[1] * mc[2]
    return r.ranges().reshape(M, len(vols), 2)


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


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    f = _fn()
    vol = torch.zeros(4 * 8 * 8, dtype=torch.uint8, device="cuda")
    out = torch.empty(2 * 2048 * 2, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert _call(f, vol, FMT_UINT8, (8, 8, 4), (2048, 1, 1), out, stream) == SCRATCH_LIMIT
    big = torch.zeros(2, dtype=torch.uint8, device="cuda")
    assert _call(f, big, FMT_UINT8, (1024, 1024, 2), (1024, 1024, 1), out, stream) == SCRATCH_LIMIT
