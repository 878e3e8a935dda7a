"""The oracle against golden outputs of the reference's own code (tests/golden, made by
tests/golden/make_golden.py from the reference's dda.h and rawFile.cpp compiled where they
lie).  Unlike tests/test_ref_pins.py these run without the reference sources."""
import ctypes as C
import os

import numpy as np
import pytest

from mdwtracker_b200 import MDWT_HOST_ONLY, Renderer

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
F3 = C.c_float * 3
U3 = C.c_uint32 * 3
TYPES = ["int8", "int16", "int32", "uint8", "uint16", "uint32", "float32", "double64"]


def test_dda_matches_the_reference_traces(oracle):
    g = np.load(os.path.join(GOLDEN, "dda_traces.npz"))
    lib = oracle.load_oracle()
    lib.orc_dda_trace.restype = C.c_int
    off = 0
    for i in range(len(g["count"])):
        gs = g["grid"][i]
        cap = int(gs.sum()) + 8
        cells = (C.c_int32 * (3 * cap))()
        t0 = (C.c_float * cap)()
        t1 = (C.c_float * cap)()
        n = lib.orc_dda_trace(F3(*g["org"][i]), F3(*g["dir"][i]), C.c_float(g["tmax"][i]), U3(*gs), C.c_int(cap),
                              cells, t0, t1)
        k = int(g["count"][i])
        assert n == k, (i, n, k)
        np.testing.assert_array_equal(np.frombuffer(cells, np.int32, 3 * n).reshape(-1, 3), g["cells"][off:off + k])
        np.testing.assert_array_equal(np.frombuffer(t0, np.uint32, n), g["t0_bits"][off:off + k])
        np.testing.assert_array_equal(np.frombuffer(t1, np.uint32, n), g["t1_bits"][off:off + k])
        off += k
    assert off == len(g["t0_bits"]) and off > 1000


@pytest.mark.parametrize("name", TYPES)
def test_loader_matches_the_reference_outputs(tmp_path, oracle, name):
    g = np.load(os.path.join(GOLDEN, "raw_loader.npz"))
    dims = tuple(int(x) for x in g[f"{name}_dims"])
    path = str(tmp_path / f"vol_{dims[0]}x{dims[1]}x{dims[2]}_{name}.raw")
    g[f"{name}_bytes"].tofile(path)
    lib = oracle.load_oracle()
    o = C.c_void_p()
    assert lib.orc_create(C.byref(o)) == 0
    try:
        assert lib.orc_push_channel_raw(o, path.encode()) == 0
        d = (C.c_int64 * 3)()
        b = (C.c_float * 8)()
        assert lib.orc_get_channel_info(o, 0, d, b) == 0
        n = int(np.prod(dims))
        vals = np.empty(n, np.float32)
        assert lib.orc_get_channel_data(o, 0, vals.ctypes.data_as(C.c_void_p)) == 0
    finally:
        lib.orc_destroy(o)
    assert tuple(d) == dims
    np.testing.assert_array_equal(np.frombuffer(b, np.uint32, 8), g[f"{name}_bounds_bits"])
    np.testing.assert_array_equal(vals.view(np.uint32), g[f"{name}_values_bits"])
    prod = Renderer(MDWT_HOST_ONLY)
    prod.PushMesh(path)
    pd, pb = prod.channelInfo(0)
    assert pd == dims
    np.testing.assert_array_equal(pb.view(np.uint32), g[f"{name}_bounds_bits"])


@pytest.mark.parametrize("by", ["dims", "scale"])
def test_reshaped_bounds_match_the_reference_outputs(tmp_path, oracle, by):
    g = np.load(os.path.join(GOLDEN, "raw_loader.npz"))
    dims = tuple(int(x) for x in g["float32_dims"])
    path = str(tmp_path / f"vol_{dims[0]}x{dims[1]}x{dims[2]}_float32.raw")
    g["float32_bytes"].tofile(path)
    scale = tuple(float(x) for x in g["reshape_scale"]) if by == "scale" else None
    for r in (Renderer(MDWT_HOST_ONLY), oracle.OracleRenderer()):
        r.PushMesh(path)
        r.reshapeBounds(0, scale)
        _, got = r.channelInfo(0)
        np.testing.assert_array_equal(got.view(np.uint32), g[f"reshape_{by}_bits"])
