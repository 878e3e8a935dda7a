"""Generates the golden fixtures of tests/test_golden.py from the reference's own code.

  python tests/golden/make_golden.py [reference-source-dir [output-dir]]

Builds oracle/_ref/libref_pins.so (the reference's dda.h and rawFile.cpp compiled where they
lie, `make -C oracle ref`) and records:
  dda_traces.npz  -- dda::dda3 (dda.h:81-202) on a fixed, seeded set of rays: every visited
                     cell and its (t0, t1) as float32 bits;
  raw_loader.npz  -- raw::RawR (rawFile.cpp:31-128) on small files of all eight voxel types:
                     the file bytes, dims, format, box4f bounds and converted values; and
                     RawR::reshapeBounds (rawFile.cpp:217-237) of the float32 file, by its
                     dims and by the factors in reshape_scale.
The fixtures are reference outputs; the tests check the oracle against them where the
reference sources are not available.
"""
import ctypes as C
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
F3 = C.c_float * 3
U3 = C.c_uint32 * 3
TYPES = [("int8", np.int8), ("int16", np.int16), ("int32", np.int32), ("uint8", np.uint8),
         ("uint16", np.uint16), ("uint32", np.uint32), ("float32", np.float32), ("double64", np.float64)]


def rays(n=400, seed=23):
    """Seeded rays around and inside grids of up to 12 cells per axis, with cell-corner
    origins, diagonal directions (ties between axes), axis-parallel and near-parallel
    directions, and finite tMax."""
    rng = np.random.default_rng(seed)
    f32 = np.float32
    out = []
    for i in range(n):
        gs = rng.integers(1, 13, 3)
        g = gs.astype(np.float64)
        kind = i % 4
        if kind == 0:
            org = rng.uniform(-0.5, 1.5, 3) * g
            d = rng.standard_normal(3)
        elif kind == 1:
            org = rng.integers(-1, gs + 2).astype(np.float64)
            d = rng.choice([-1.0, 0.5, 1.0, 2.0], 3) * rng.choice([-1.0, 1.0], 3)
        elif kind == 2:
            org = rng.uniform(-0.2, 1.2, 3) * g
            d = rng.standard_normal(3)
            d[rng.integers(0, 3)] = rng.choice([0.0, 1e-5, -1e-5])
        else:
            org = g * 0.5 + rng.standard_normal(3) * g.max() * 1.5
            d = g * rng.uniform(0.2, 0.8, 3) - org
        d = d / np.linalg.norm(d)
        tmax = 1e20 if rng.random() < 0.75 else float(rng.uniform(0.0, 2.0 * g.max()))
        out.append((org.astype(f32), d.astype(f32), f32(tmax), gs.astype(np.uint32)))
    return out


def main(argv):
    ref = argv[1] if len(argv) > 1 else os.path.normpath(os.path.join(ROOT, "..", "reference"))
    out = argv[2] if len(argv) > 2 else HERE
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref", "REF=" + ref], check=True,
                   stdout=subprocess.DEVNULL)
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_pins.so"))
    lib.ref_raw_load.restype = C.c_int64
    lib.ref_raw_reshape.restype = C.c_int
    R = rays()
    orgs, dirs, tmaxs, gss, counts, cells, t0s, t1s = [], [], [], [], [], [], [], []
    for org, d, tmax, gs in R:
        cap = int(gs.sum()) + 8
        cb = (C.c_int32 * (3 * cap))()
        a = (C.c_float * cap)()
        b = (C.c_float * cap)()
        k = lib.ref_dda_trace(F3(*org), F3(*d), C.c_float(tmax), U3(*gs), C.c_int(cap), cb, a, b)
        orgs.append(org); dirs.append(d); tmaxs.append(tmax); gss.append(gs); counts.append(k)
        cells.append(np.frombuffer(cb, np.int32, 3 * k).reshape(-1, 3).copy())
        t0s.append(np.frombuffer(a, np.uint32, k).copy())
        t1s.append(np.frombuffer(b, np.uint32, k).copy())
    np.savez_compressed(os.path.join(out, "dda_traces.npz"), org=np.array(orgs), dir=np.array(dirs),
                        tmax=np.array(tmaxs), grid=np.array(gss), count=np.array(counts, np.int32),
                        cells=np.concatenate(cells), t0_bits=np.concatenate(t0s), t1_bits=np.concatenate(t1s))
    rng = np.random.default_rng(29)
    recs = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, dt in TYPES:
            dims = (5, 3, 2)
            n = int(np.prod(dims))
            if np.issubdtype(dt, np.integer):
                info = np.iinfo(dt)
                arr = rng.integers(info.min, info.max, n, endpoint=True,
                                   dtype=np.int64 if info.min < 0 else np.uint64).astype(dt)
                arr[:2] = [info.min, info.max]
            else:
                arr = (rng.standard_normal(n) * 1e3).astype(dt)
                arr[:4] = [np.nan, np.inf, -np.inf, -0.0]
            path = os.path.join(tmp, f"vol_{dims[0]}x{dims[1]}x{dims[2]}_{name}.raw")
            arr.tofile(path)
            rd = (C.c_int64 * 3)()
            fmt = C.c_int()
            bounds = (C.c_float * 8)()
            vals = (C.c_float * n)()
            got = lib.ref_raw_load(path.encode(), rd, C.byref(fmt), bounds, vals, C.c_int64(n))
            assert got == n
            recs[f"{name}_bytes"] = np.frombuffer(arr.tobytes(), np.uint8)
            recs[f"{name}_dims"] = np.array(rd[:], np.int64)
            recs[f"{name}_format"] = np.array(fmt.value, np.int32)
            recs[f"{name}_bounds_bits"] = np.frombuffer(bounds, np.uint32, 8).copy()
            recs[f"{name}_values_bits"] = np.frombuffer(vals, np.uint32, n).copy()
            if name == "float32":
                scale = np.array([0.5, 2.0, 1.25], np.float32)
                for key, sc in (("reshape_dims_bits", None), ("reshape_scale_bits", scale)):
                    rb = (C.c_float * 8)()
                    assert lib.ref_raw_reshape(path.encode(), (C.c_float * 3)(*sc) if sc is not None else None, rb) == 0
                    recs[key] = np.frombuffer(rb, np.uint32, 8).copy()
                recs["reshape_scale"] = scale
    np.savez_compressed(os.path.join(out, "raw_loader.npz"), **recs)
    print("wrote", os.path.join(out, "dda_traces.npz"), "and", os.path.join(out, "raw_loader.npz"))
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
