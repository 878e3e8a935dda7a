"""Headless counterpart of the reference's offline viewer (`mdwtOffline`, viewer.cpp built
with OFFLINE_VIEWER=true).  Same flag names and meanings (viewer.cpp:72-150):

  python -m mdwtracker_b200.cli -fr a_256x256x256_uint8.raw b_256x256x256_uint8.raw \\
      -t a.tf b.tf -mc 16 -r 1024 1024 -m 2 -spp 64 -n 10 -wu 2 -o shot

Frame loop of viewer.cpp:486-527: Init(mode, !camera-given), Setdt, UpdateCamera, the TF
of every channel, then frames while frameID < n + wu, with accumulation reset during the
warm-up frames; a PNG every -nt frames and one at the end
(`<o>_<MODE>_w_<frames>_shadows_<on|off>_frames.png`, viewer.cpp:797-827).
TF files use this project's JSON format (mdwtracker_b200.imageio.load_tf).
"""
from __future__ import annotations

import argparse
import sys
import time

import numpy as np

MODE_NAMES = {0: "BLN", 1: "MMB", 2: "AMMB", 3: "CMB", 4: "MAX", 5: "MIX", 6: "MM_RM", 7: "MAX_RM", 8: "MIX_RM",
              9: "COMP"}


def build_parser() -> argparse.ArgumentParser:
    p = argparse.ArgumentParser(prog="mdwtOffline", description="headless multi-density Woodcock tracker")
    p.add_argument("-fu", "--umesh-data", help="unstructured meshes are not supported by this renderer")
    p.add_argument("-fr", "--raw-data", nargs="*", help="path(s) to <name>_<X>x<Y>x<Z>_<type>.raw files")
    p.add_argument("-c", "--camera", nargs=10, type=float, help="pos xyz, gaze xyz, up xyz, fovy (degrees)")
    p.add_argument("-t", "--transfer-function", nargs="*", help="TF file(s), one per channel")
    p.add_argument("-mc", "--macrocells", nargs="*", type=int, help="macrocells per side (1 or 3 values)")
    p.add_argument("-bg", "--background", nargs=3, type=float)
    p.add_argument("-dt", "--delta-t", type=float)
    p.add_argument("-cb", "--correct-bounds", nargs="*", type=float, help="rescale bounds (none: to the dims)")
    p.add_argument("-r", "--resolution", nargs=2, type=int)
    p.add_argument("-l", "--light", nargs="+", type=float,
                   help="shadows(0/1) gradient(0/1) dir xyz [intensity] [ambient]")
    p.add_argument("-m", "--mode", type=int, default=0)
    p.add_argument("-spp", "--samples-per-pixel", type=int, default=1)
    p.add_argument("-acc", "--accumulation", type=int, default=1)
    p.add_argument("-mf", "--mirror-frame", type=int, default=0)
    p.add_argument("-n", "--num-frame", type=int, default=100)
    p.add_argument("-wu", "--warm-up", type=int, default=0)
    p.add_argument("-nt", "--nth-frame", type=int, default=0)
    p.add_argument("-o", "--output", default="")
    p.add_argument("-hm", "--heatmap", type=float, help="timing heat map (commented out in the reference)")
    p.add_argument("--device", type=int, default=0)
    p.add_argument("--pfm", action="store_true", help="also write the accumulation buffer as PFM")
    return p


def validate(a) -> None:
    """The reference's own argument checks (viewer.cpp:204-224, 273-283, 298-339)."""
    if a.umesh_data:
        raise SystemExit("unstructured meshes (-fu) are not supported")
    if not a.raw_data:
        raise SystemExit("No data file given")
    if a.macrocells is not None:
        if len(a.macrocells) not in (1, 3):
            raise SystemExit("-mc takes 1 or 3 values")
        if any(m < 1 for m in a.macrocells):
            raise SystemExit("Number of macrocells per side must be positive")
    if a.correct_bounds is not None and len(a.correct_bounds) not in (0, 3):
        raise SystemExit("Bounds must be given as 3 floats or not at all")
    if a.light is not None and not 5 <= len(a.light) <= 7:
        raise SystemExit("-l takes 5 to 7 values")
    if a.mode not in MODE_NAMES:
        raise SystemExit(f"unknown mode {a.mode}")


def setup(a, renderer):
    """Renderer set-up of Viewer::Viewer + Viewer::Run (viewer.cpp:152-509)."""
    from . import imageio
    from .synthetic import viridis_like
    for i, path in enumerate(a.raw_data):
        renderer.PushMesh(path)
        if a.correct_bounds is not None:
            renderer.reshapeBounds(i, a.correct_bounds if len(a.correct_bounds) == 3 else None)
    if a.macrocells:
        mc = a.macrocells * 3 if len(a.macrocells) == 1 else a.macrocells
        renderer.macrocellDims = tuple(mc)
    if a.resolution:
        renderer.Resize(tuple(a.resolution))
    if a.light is not None:
        lt = a.light
        renderer.setLight(bool(lt[0]), bool(lt[1]), lt[2:5], lt[5] if len(lt) > 5 else 1.0,
                          lt[6] if len(lt) > 6 else 0.1)
    renderer.Init(a.mode, a.camera is None)
    if a.delta_t is not None and a.delta_t > 0.0:
        renderer.Setdt(a.delta_t)
    if a.camera is not None:
        c = a.camera
        renderer.setCamera(c[0:3], c[3:6], c[6:9], c[9])
    tfs = a.transfer_function or []
    for i in range(len(a.raw_data)):
        if i < len(tfs):
            cm, os_, rng = imageio.load_tf(tfs[i])
        else:
            cm, os_, rng = viridis_like(), 1.0, (0.0, 1.0)
        renderer.SetXFColormap(cm, i)
        renderer.SetXFOpacityScale(os_, i)
        renderer.SetXFRange(rng, i)
    if a.background:
        renderer.setBackground(a.background)
    renderer.setSpp(a.samples_per_pixel)
    renderer.setAccumulation(bool(a.accumulation))
    renderer.setMirror(bool(a.mirror_frame))
    return renderer


def snapshot_name(a, frames_done: int) -> str:
    shadows = "on" if (a.light is not None and a.light[0]) else "off"
    return f"{a.output}_{MODE_NAMES[a.mode]}_w_{frames_done}_shadows_{shadows}_frames.png"


def run(a, renderer, out=None) -> dict:
    """The offline frame loop (viewer.cpp:510-527, 797-827)."""
    from . import imageio
    out = out or sys.stdout
    times = []
    frame = 0
    while frame < a.num_frame + a.warm_up:
        if frame <= a.warm_up:
            renderer.ResetAccumulation()
        t0 = time.perf_counter()
        renderer.Render()
        renderer.sync()
        times.append(time.perf_counter() - t0)
        frame += 1
        if frame >= a.warm_up and a.nth_frame and (frame - a.warm_up) % a.nth_frame == 0 and a.output:
            imageio.write_png(snapshot_name(a, frame - a.warm_up), renderer.framebuffer())
    measured = times[a.warm_up:] or times
    avg, best = float(np.mean(measured)), float(np.min(measured))
    print("============ Scene Info ============", file=out)
    print(f"Number of frames: {frame - a.warm_up}", file=out)
    print(f"Macrocell dimensions: {', '.join(str(x) for x in renderer.macrocellDims)}", file=out)
    print(f"Mode: {MODE_NAMES[a.mode]}", file=out)
    for i in range(renderer.numChannels):
        dims, _ = renderer.channelInfo(i)
        print(f"Volume #{i} size: {dims[0]}x{dims[1]}x{dims[2]}", file=out)
    print(f"avg. fps: {1.0 / avg:.3f} ({avg:.4f} sec)", file=out)
    print(f"best. fps: {1.0 / best:.3f} ({best:.4f} sec)", file=out)
    if a.output:
        imageio.write_png(snapshot_name(a, frame - a.warm_up), renderer.framebuffer())
        if a.pfm:
            imageio.write_pfm(snapshot_name(a, frame - a.warm_up)[:-4] + ".pfm", renderer.accum())
    return {"frames": frame - a.warm_up, "avg_s": avg, "best_s": best}


def main(argv=None) -> int:
    a = build_parser().parse_args(argv)
    validate(a)
    from .renderer import Renderer
    r = setup(a, Renderer(a.device))
    run(a, r)
    r.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
