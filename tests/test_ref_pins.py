"""The oracle against the reference's own code, for the parts of the path that compile
without OptiX: the 3-D DDA (dda.h:81-202) and the raw-file loader (rawFile.cpp:31-128).

`make -C oracle ref` compiles the reference's dda.h and rawFile.cpp where they lie, with a
stand-in for OWL's vector types (oracle/ref_shim), into oracle/_ref/libref_pins.so.  The
tests skip where the reference sources are absent.  Everything is compared bit for bit:
the cells a ray visits and each cell's (t0, t1), and the loader's dims, format, box4f
bounds and converted values.  The product's host-side loader (a host-only context) is
checked against the same reference results."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from mdwtracker_b200 import MDWT_HOST_ONLY, MdwtError, Renderer

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
REF_LIB = os.path.join(ORACLE_DIR, "_ref", "libref_pins.so")

F3 = C.c_float * 3
U3 = C.c_uint32 * 3


@pytest.fixture(scope="module")
def ref():
    r = subprocess.run(["make", "-C", ORACLE_DIR, "ref"], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
    if r.returncode != 0 and not os.path.exists(REF_LIB):
        pytest.skip("the reference sources are not available to build oracle/_ref")
    lib = C.CDLL(REF_LIB)
    lib.ref_dda_trace.restype = C.c_int
    lib.ref_raw_load.restype = C.c_int64
    return lib


@pytest.fixture(scope="module")
def orc(oracle):
    lib = oracle.load_oracle()
    lib.orc_dda_trace.restype = C.c_int
    return lib


def trace(fn, org, d, tmax, gs, cap):
    cells = (C.c_int32 * (3 * cap))()
    t0 = (C.c_float * cap)()
    t1 = (C.c_float * cap)()
    n = fn(F3(*org), F3(*d), C.c_float(tmax), U3(*gs), C.c_int(cap), cells, t0, t1)
    return (np.frombuffer(cells, np.int32, 3 * n).copy(), np.frombuffer(t0, np.uint32, n).copy(),
            np.frombuffer(t1, np.uint32, n).copy())


def ray_set(seed=11):
    """(org, dir, tMax, grid) cases: random rays around and inside random grids,
    rays from cell corners along diagonals (ties between axes), axis-parallel rays (the
    reference visits nothing: dda.h:100-113 assigns t_nr = -inf then +inf), components at
    generateRay's 1e-5 clamp, finite tMax inside the grid, and grid faces."""
    rng = np.random.default_rng(seed)
    f32 = np.float32
    out = []
    unit = lambda v: (np.asarray(v, np.float64) / np.linalg.norm(v)).astype(f32)
    for i in range(6000):
        gs = tuple(int(x) for x in rng.integers(1, 49, 3))
        g = np.array(gs, np.float64)
        kind = i % 6
        if kind == 0:    # anywhere around the grid
            org = (rng.uniform(-0.5, 1.5, 3) * g).astype(f32)
            d = unit(rng.standard_normal(3))
        elif kind == 1:  # inside, pointing anywhere
            org = (rng.uniform(0.0, 1.0, 3) * g).astype(f32)
            d = unit(rng.standard_normal(3))
        elif kind == 2:  # from a cell corner along a (partial) diagonal: exact ties
            org = rng.integers(-2, np.array(gs) + 3).astype(f32)
            d = unit(rng.choice([-1.0, 0.5, 1.0, 2.0], 3) * rng.choice([-1.0, 1.0], 3))
        elif kind == 3:  # axis-parallel or nearly so
            d = rng.standard_normal(3)
            d[rng.integers(0, 3)] = rng.choice([0.0, -0.0, 1e-5, -1e-5, 1e-7])
            d = unit(d)
            org = (rng.uniform(-0.2, 1.2, 3) * g).astype(f32)
        elif kind == 4:  # a camera outside looking at the grid, like the tracker's rays
            org = (g * 0.5 + unit(rng.standard_normal(3)).astype(np.float64) * g.max() * rng.uniform(1.0, 3.0)).astype(f32)
            d = unit(g * rng.uniform(0.2, 0.8, 3) - org)
        else:            # on a face, pointing in or out
            org = (rng.uniform(0.0, 1.0, 3) * g).astype(f32)
            a = rng.integers(0, 3)
            org[a] = f32(0.0 if rng.random() < 0.5 else g[a])
            d = unit(rng.standard_normal(3))
        tmax = 1e20 if rng.random() < 0.8 else float(rng.uniform(0.0, 2.0 * g.max()))
        out.append((tuple(float(x) for x in org), tuple(float(x) for x in d), tmax, gs))
    return out


def test_dda_matches_the_reference_dda3(ref, orc):
    visited = 0
    for org, d, tmax, gs in ray_set():
        cap = sum(gs) + 8
        cr, t0r, t1r = trace(ref.ref_dda_trace, org, d, tmax, gs, cap)
        co, t0o, t1o = trace(orc.orc_dda_trace, org, d, tmax, gs, cap)
        ok = np.array_equal(cr, co) and np.array_equal(t0r, t0o) and np.array_equal(t1r, t1o)
        assert ok, f"dda differs for org={org} dir={d} tMax={tmax} grid={gs}: {len(t0r)} vs {len(t0o)} cells"
        visited += len(t0r) > 0
    assert visited > 3000   # most rays cross their grid


def test_dda_axis_parallel_rays_visit_nothing(ref, orc):
    for d in [(1.0, 0.0, 0.0), (0.0, -1.0, 0.0), (0.0, 0.6, 0.8)]:
        for fn in (ref.ref_dda_trace, orc.orc_dda_trace):
            c, _, _ = trace(fn, (2.5, 2.5, 2.5), d, 1e20, (8, 8, 8), 64)
            assert c.size == 0


def ref_load(ref, path, n_max):
    dims = (C.c_int64 * 3)()
    fmt = C.c_int()
    b = (C.c_float * 8)()
    out = (C.c_float * max(n_max, 1))()
    n = ref.ref_raw_load(os.fsencode(path), dims, C.byref(fmt), b, out, C.c_int64(n_max))
    return tuple(dims), fmt.value, np.array(b[:], np.float32), np.frombuffer(out, np.float32, n).copy()


def orc_load(orc, path, n):
    o = C.c_void_p()
    assert orc.orc_create(C.byref(o)) == 0
    try:
        st = orc.orc_push_channel_raw(o, os.fsencode(path))
        if st != 0:
            return st, None, None, None
        dims = (C.c_int64 * 3)()
        b = (C.c_float * 8)()
        assert orc.orc_get_channel_info(o, 0, dims, b) == 0
        data = np.empty(n, np.float32)
        assert orc.orc_get_channel_data(o, 0, data.ctypes.data_as(C.c_void_p)) == 0
        return 0, tuple(dims), np.array(b[:], np.float32), data
    finally:
        orc.orc_destroy(o)


TYPES = [("int8", np.int8, 1), ("int16", np.int16, 2), ("int32", np.int32, 3), ("uint8", np.uint8, 4),
         ("uint16", np.uint16, 5), ("uint32", np.uint32, 6), ("float32", np.float32, 7), ("double64", np.float64, 8)]


def full_range(rng, dt, n):
    if np.issubdtype(dt, np.integer):
        info = np.iinfo(dt)
        a = rng.integers(info.min, info.max, n, endpoint=True, dtype=np.int64 if info.min < 0 else np.uint64)
        a = a.astype(dt)
        a[:2] = [info.min, info.max]
        return a
    a = (rng.standard_normal(n) * 1e3).astype(dt)
    a[:5] = [np.nan, np.inf, -np.inf, np.finfo(dt).max, -0.0]
    if dt == np.float64:
        a[5:7] = [1e300, -1e-300]   # out of float range: inf and -0 after the conversion
    return a


@pytest.mark.parametrize("tname,dt,code", TYPES)
def test_loader_matches_the_reference_rawr(tmp_path, ref, orc, tname, dt, code):
    rng = np.random.default_rng(code)
    dims = (7, 5, 3)
    n = int(np.prod(dims))
    arr = full_range(rng, dt, n)
    path = str(tmp_path / f"vol_{dims[0]}x{dims[1]}x{dims[2]}_{tname}.raw")
    arr.tofile(path)
    rd, rf, rb, rv = ref_load(ref, path, n)
    assert rd == dims and rf == code and rv.size == n
    st, od, ob, ov = orc_load(orc, path, n)
    assert st == 0 and od == rd
    np.testing.assert_array_equal(ob.view(np.uint32), rb.view(np.uint32))
    np.testing.assert_array_equal(ov.view(np.uint32), rv.view(np.uint32))
    prod = Renderer(MDWT_HOST_ONLY)
    prod.PushMesh(path)
    pd, pb = prod.channelInfo(0)
    assert pd == rd
    np.testing.assert_array_equal(pb.view(np.uint32), rb.view(np.uint32))


def test_loader_path_rules_match_the_reference(tmp_path, ref, orc):
    """Tokens are split on '_' over the whole path and cut at their first '.'
    (rawFile.cpp:36-84): directory names take part, the last dims and type tokens win."""
    d = tmp_path / "run_2x2x2_int16.d"
    d.mkdir()
    arr = np.arange(4 * 3 * 2, dtype=np.uint16) * 1000
    path = str(d / "vol_4x3x2_uint16.raw")
    arr.tofile(path)
    rd, rf, rb, rv = ref_load(ref, path, arr.size)
    assert rd == (4, 3, 2) and rf == 5
    st, od, ob, ov = orc_load(orc, path, arr.size)
    assert st == 0 and od == rd
    np.testing.assert_array_equal(ov.view(np.uint32), rv.view(np.uint32))
    np.testing.assert_array_equal(ob.view(np.uint32), rb.view(np.uint32))


def test_unknown_type_token_is_an_error_here(tmp_path, ref, orc):
    """A token after the type that names no type leaves the reference's format
    Unspecified: it reads nothing it converts and returns zeros with the default bounds.
    The oracle and the product report a format error instead of rendering an empty volume
    (the library's error convention)."""
    arr = np.arange(8, dtype=np.uint8)
    path = str(tmp_path / "vol_2x2x2_uint8_copy.raw")
    arr.tofile(path)
    rd, rf, rb, rv = ref_load(ref, path, 8)
    assert rd == (2, 2, 2) and rf == 0
    assert not rv.any()
    np.testing.assert_array_equal(rb, [0, 0, 0, 0, 1, 1, 1, 1])
    st, *_ = orc_load(orc, path, 8)
    assert st != 0
    with pytest.raises(MdwtError) as e:
        Renderer(MDWT_HOST_ONLY).PushMesh(path)
    assert e.value.status == 9


def test_golden_fixtures_are_the_reference_outputs(ref, tmp_path):
    """tests/golden holds what tests/golden/make_golden.py writes from the reference's code."""
    import sys
    gen = os.path.join(ROOT, "tests", "golden", "make_golden.py")
    import __graft_entry__   # names the reference sources that build() compiles the pins from
    r = subprocess.run([sys.executable, gen, __graft_entry__.REF_SOURCES, str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    for name in ("dda_traces.npz", "raw_loader.npz"):
        new, old = np.load(tmp_path / name), np.load(os.path.join(ROOT, "tests", "golden", name))
        assert sorted(new.files) == sorted(old.files)
        for k in new.files:
            np.testing.assert_array_equal(new[k], old[k], err_msg=f"{name}:{k}")


@pytest.mark.parametrize("scale", [None, (0.5, 2.0, 1.25), (3.0, 3.0, 3.0)])
def test_reshaped_bounds_match_the_reference(tmp_path, ref, oracle, scale):
    """raw::RawR::reshapeBounds (rawFile.cpp:217-237, the -cb flag): xyz bounds times the dims,
    or times the given factors; the value range is kept."""
    arr = (np.arange(6 * 3 * 11, dtype=np.float32) * 0.37).reshape(11, 3, 6)
    path = str(tmp_path / "vol_6x3x11_float32.raw")
    arr.tofile(path)
    b = (C.c_float * 8)()
    assert ref.ref_raw_reshape(os.fsencode(path), (C.c_float * 3)(*scale) if scale else None, b) == 0
    want = np.frombuffer(b, np.uint32, 8).copy()
    for r in (Renderer(MDWT_HOST_ONLY), oracle.OracleRenderer()):
        r.PushMesh(path)
        r.reshapeBounds(0, scale)
        _, got = r.channelInfo(0)
        np.testing.assert_array_equal(got.view(np.uint32), want)
