"""The oracle's statement of the texture unit's linear filter (orc_sample_tex3d /
orc_sample_tex2d, the arithmetic every tracker parity test rests on) against an
independent numpy restatement of the same rule: x = fma(u, N, -0.5), i = floor(x),
weight = rint((x - i) * 256) / 256, texel indices clamped to [0, N - 1],
lerp(a, p, q) = fma(a, q, RN((1 - a) p)), along x, then y, then z.  float32 fma is
formed exactly in float64 (the products of two floats fit its 53 bits) and rounded once.
The GPU test file test_gpu_ref_majorants.py holds the same rule against the B200's
texture unit."""
import ctypes as C

import numpy as np

FP = C.POINTER(C.c_float)


def f32(x):
    return np.asarray(x, dtype=np.float64).astype(np.float32)


def fma32(a, b, c):
    """RN32(a * b + c) for float32 a, b, c (a * b exact in float64; the sum rounded once is
    RN32 of the exact value except in double-rounding corner cases, which a check of the
    float64 sum's exactness rules out below)."""
    p = a.astype(np.float64) * b.astype(np.float64)
    s = p + c.astype(np.float64)
    # the float64 sum is exact when its error term is zero; assert that for the inputs used
    err = (s - p) - c.astype(np.float64)
    assert np.all(err == 0)
    return s.astype(np.float32)


def axis(u, n):
    x = fma32(f32(u), f32(np.full_like(u, n)), f32(np.full_like(u, -0.5)))
    fl = np.floor(x)
    a = f32(np.rint(f32(x - fl).astype(np.float64) * 256.0) / 256.0)
    i = fl.astype(np.int64)
    return np.clip(i, 0, n - 1), np.clip(i, -1, n - 2) + 1, a


def lerp(a, p, q):
    return fma32(a, q, f32((f32(1.0) - a) * p))


def test_tex3d_statement(oracle):
    lib = oracle.load_oracle()
    lib.orc_sample_tex3d.argtypes = [FP, C.POINTER(C.c_int), FP, C.c_int, FP]
    rng = np.random.default_rng(2)
    X, Y, Z = 13, 7, 9
    # values on a coarse grid keep every float64 sum exact (see fma32)
    vol = np.ascontiguousarray((rng.integers(-512, 512, (Z, Y, X)) / 8.0).astype(np.float32))
    n = 20000
    xyz = np.concatenate([rng.random((n, 3), dtype=np.float32),
                          (rng.random((n, 3), dtype=np.float32) * 1.4 - 0.2).astype(np.float32),
                          np.stack([(rng.integers(0, s, n) + 0.5) / s for s in (X, Y, Z)], 1).astype(np.float32)])
    xyz = np.ascontiguousarray(xyz)
    out = np.empty(len(xyz), np.float32)
    dims = np.array([X, Y, Z], np.int32)
    lib.orc_sample_tex3d(vol.ctypes.data_as(FP), dims.ctypes.data_as(C.POINTER(C.c_int)),
                         xyz.ctypes.data_as(FP), len(xyz), out.ctypes.data_as(FP))
    ax, ay, az = axis(xyz[:, 0], X), axis(xyz[:, 1], Y), axis(xyz[:, 2], Z)
    at = lambda i, j, k: vol[k, j, i]
    c00 = lerp(ax[2], at(ax[0], ay[0], az[0]), at(ax[1], ay[0], az[0]))
    c10 = lerp(ax[2], at(ax[0], ay[1], az[0]), at(ax[1], ay[1], az[0]))
    c01 = lerp(ax[2], at(ax[0], ay[0], az[1]), at(ax[1], ay[0], az[1]))
    c11 = lerp(ax[2], at(ax[0], ay[1], az[1]), at(ax[1], ay[1], az[1]))
    ref = lerp(az[2], lerp(ay[2], c00, c10), lerp(ay[2], c01, c11))
    np.testing.assert_array_equal(out.view(np.uint32), ref.view(np.uint32))
    # texel centres return the texel itself
    cen = out[2 * n:]
    ic = [np.floor(xyz[2 * n:, a].astype(np.float64) * d).astype(np.int64) for a, d in enumerate((X, Y, Z))]
    np.testing.assert_array_equal(cen, vol[ic[2], ic[1], ic[0]])


def test_tex2d_statement_and_weight_ties(oracle):
    lib = oracle.load_oracle()
    lib.orc_sample_tex2d.argtypes = [FP, C.c_int, FP, C.c_int, FP]
    N = 64
    tf = np.zeros((N, 4), np.float32)
    tf[:, 0] = np.arange(N) * 256.0          # a ramp: the filtered value reads the weight
    tf[:, 3] = 1.0
    # coordinates whose fractional part times 256 is k + 1/2: ties round to even
    k = np.arange(0, 255)
    i = 10
    u = ((i + 0.5 + (k + 0.5) / 256.0) / N).astype(np.float32)
    uv = np.ascontiguousarray(np.stack([u, np.full_like(u, 0.5)], 1))
    out = np.empty((len(u), 4), np.float32)
    lib.orc_sample_tex2d(np.ascontiguousarray(tf).ctypes.data_as(FP), N, uv.ctypes.data_as(FP), len(u),
                         out.ctypes.data_as(FP))
    w = out[:, 0] - i * 256.0
    np.testing.assert_array_equal(w, np.rint(k + 0.5))
    assert np.all(out[:, 3] == 1.0)
