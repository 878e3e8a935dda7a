"""Host-side logic of libmdwt.so against the oracle, bit for bit, without a GPU:
raw-file parsing and conversion (rawFile.cpp:31-128), bounds reshaping
(rawFile.cpp:217-237), dt (renderer.cpp:1444-1466), default macrocell dims
(renderer.cpp:1342-1355) and the camera basis (camera.h:83-125, renderer.cpp:1058-1092).
The oracle's own camera/dt code runs only after init, so it is compared there."""
import os

import numpy as np
import pytest

from mdwtracker_b200 import MDWT_HOST_ONLY, MdwtError, Renderer


def write_raw(tmp_path, name, arr):
    p = os.path.join(str(tmp_path), name)
    arr.tofile(p)
    return p


FORMATS = [("int8", np.int8), ("int16", np.int16), ("int32", np.int32), ("uint8", np.uint8),
           ("uint16", np.uint16), ("uint32", np.uint32), ("float32", np.float32), ("double64", np.float64)]


def reference_convert(arr, name):
    """rawFile.cpp:94-121 in float32 arithmetic."""
    f = np.float32
    a = arr.astype(np.float64).astype(np.float32) if name != "double64" else arr.astype(np.float32)
    if name == "int8":
        return a * f(255) - f(128)
    if name == "int16":
        return a * f(65535) - f(32768)
    if name == "int32":
        return a * f(4294967295.0) - f(2147483648.0)
    if name == "uint8":
        return a * f(255)
    if name == "uint16":
        return a * f(65535)
    if name == "uint32":
        return a * f(4294967295.0)
    return a


@pytest.mark.parametrize("tname,dt", FORMATS)
def test_raw_files_parse_and_convert_like_rawr(tmp_path, oracle, tname, dt):
    rng = np.random.default_rng(5)
    if np.issubdtype(dt, np.integer):
        info = np.iinfo(dt)
        arr = rng.integers(max(info.min, -100), min(info.max, 100), (5, 4, 3)).astype(dt)
    else:
        arr = (rng.standard_normal((5, 4, 3)) * 10).astype(dt)
    path = write_raw(tmp_path, f"vol_3x4x5_{tname}.raw", arr)
    prod = Renderer(MDWT_HOST_ONLY)
    prod.PushMesh(path)
    orc = oracle.OracleRenderer()
    orc.PushMesh(path)
    dims_p, b_p = prod.channelInfo(0)
    dims_o, b_o = orc.channelInfo(0)
    assert dims_p == dims_o == (3, 4, 5)
    vals = reference_convert(arr, tname)
    exp_lo = min(0.0, float(vals.min()))
    exp_hi = max(1.0, float(vals.max()))
    np.testing.assert_array_equal(b_p, b_o)
    assert b_p[3] == np.float32(exp_lo) and b_p[7] == np.float32(exp_hi)
    np.testing.assert_array_equal(b_p[:3], [0, 0, 0])
    np.testing.assert_array_equal(b_p[4:7], [1, 1, 1])


def test_raw_name_rules(tmp_path):
    arr = np.arange(8, dtype=np.uint8)
    # type token before dims, path with a dot in a directory component
    d = tmp_path / "a.b"
    d.mkdir()
    p = write_raw(d, "x_uint8_2x2x2.raw", arr)
    r = Renderer(MDWT_HOST_ONLY)
    r.PushMesh(p)
    assert r.channelInfo(0)[0] == (2, 2, 2)
    # an unknown token after the type resets the format to Unspecified (rawFile.cpp:78-80)
    p2 = write_raw(tmp_path, "x_2x2x2_uint8_extra.raw", arr)
    with pytest.raises(MdwtError) as e:
        r.PushMesh(p2)
    assert e.value.status == 9
    # truncated data
    p3 = write_raw(tmp_path, "t_4x4x4_uint8.raw", arr)
    with pytest.raises(MdwtError) as e:
        r.PushMesh(p3)
    assert e.value.status == 3


def test_reshape_bounds_and_dt(oracle):
    vol = np.zeros((16, 8, 32), np.uint8)
    prod = Renderer(MDWT_HOST_ONLY)
    prod.PushMesh(vol)
    prod.reshapeBounds(0)
    _, b = prod.channelInfo(0)
    np.testing.assert_array_equal(b[:3], [0, 0, 0])
    np.testing.assert_array_equal(b[4:7], [32, 8, 16])
    prod.reshapeBounds(0, (0.5, 2.0, 1.0))
    _, b = prod.channelInfo(0)
    np.testing.assert_array_equal(b[4:7], [16, 16, 16])
    prod.Resetdt()
    # min voxel side 16/32 = 0.5 -> dt 0.25
    assert prod.dt == np.float32(0.25)
    prod.Setdt(1e-7)
    assert prod.dt == np.float32(1e-4)


def test_default_macrocell_dims_match_oracle(oracle):
    vols = [np.zeros((20, 13, 9), np.uint8), np.zeros((7, 30, 18), np.uint8)]
    prod = Renderer(MDWT_HOST_ONLY)
    orc = oracle.OracleRenderer()
    for v in vols:
        prod.PushMesh(v)
        orc.PushMesh(v)
    prod.macrocellDims = (0, 5, 0)
    orc.macrocellDims = (0, 5, 0)
    orc.Init(0)
    assert prod.macrocellDims == orc.macrocellDims


CAMERAS = [
    ((0.5, 0.5, 3.0), (0.5, 0.5, 0.5), (0, 1, 0), 45.0),
    ((2.0, 1.3, -1.7), (0.4, 0.55, 0.5), (0.1, 1, 0.2), 30.0),
    ((0.5, 3.0, 0.5), (0.5, 0.5, 0.5), (0, 1, 0), 60.0),      # looking along the up vector
    ((1.0, 1.0, 1.0), (1.0, 1.0, 1.0), (0, 0, 1), 90.0),      # interest == origin
]


@pytest.mark.parametrize("res", [(64, 64), (1920, 1080), (37, 101)])
def test_camera_basis_matches_oracle(oracle, res):
    vol = np.zeros((8, 8, 8), np.uint8)
    orc = oracle.OracleRenderer()
    orc.PushMesh(vol)
    orc.Resize(res)
    orc.Init(0)
    prod = Renderer(MDWT_HOST_ONLY)
    prod.PushMesh(vol)
    prod.Resize(res)
    for cam in CAMERAS:
        orc.setCamera(*cam)
        prod.setCamera(*cam)
        np.testing.assert_array_equal(prod.cameraBasis(), orc.cameraBasis())
