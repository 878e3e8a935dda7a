#!/usr/bin/env python
"""Benchmark of the multi-density Woodcock tracker on B200.

One step = one frame of the configured scene: every pixel x spp primary path through
the tracker (Renderer::Render, renderer.cpp:944-973).  Metric: Gpath-samples/s
(pixels x spp per second), whole job.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--config c2|c1|c3] [--impl mdwt|reference]

Default workload (c3): syncDDA (-m 2), 6 channels of 512^3 float32 log-normal fields,
16-voxel macrocells, 1920x1080, 256 spp -- the configuration the headline metric is
quoted on.  Inputs (volumes, majorants) are resident in HBM before timing; L2 is flushed
by a 512 MiB write between timed steps, outside the timed events (the 3.2 GB volume is
larger than L2 in any case).  `value` is device time (CUDA events on the render stream);
`e2e` goes through the C ABI with host buffers: camera update (host to device), frame,
framebuffer copy to pinned host memory.  Under torchrun (--split rows, the default) the
ranks render ONE frame together: each renders a band of rows (mdwtracker_b200.multigpu.
BandRenderer; the bands are re-cut from measured render times during the warm-up so that
each carries an equal share of the work) and the RGBA8 bands are all-gathered over NCCL
inside the timed region -- total work is fixed, `scaling` is strong, time is the max over
ranks.  --split replicas: every rank renders its own whole frames (different frame
seeds) with no collective (`scaling` weak).  Before timing, the tracker schedule is tuned for the
workload (mdwt_autotune_schedule on launches of the step's shape; --no-autotune keeps
the defaults) and reported in config.schedule.

Extra keys on the same line (rank 0, one GPU): `c2` -- the 3 x 256^3 uint8 syncDDA
scene at 1024^2 and 64 spp, timed the same way; `edge_sweep` -- the 1080p scene's
macrocell sweep over edges 4/8/16/32 voxels for syncDDA and N-DDA (--no-sweep skips
it); `--edge` sets the headline scene's edge; `fast_arith` -- the headline scene and C2
with the fast free-flight arithmetic (mdwt_set_arithmetic: hardware-log2 flight lengths,
per-pixel events equal to the oracle's on >= 99.9 % of pixels; --no-fast skips it).  The
headline line itself runs the exact arithmetic (bit-identical to the oracle) unless
--arith fast.

time_to_rmse (rank 0, one GPU; --no-ttr skips it): the first part of the headline metric
-- how long plain accumulation takes at 1920x1080 (the 6 x 512^3 float32 log-normal scene,
syncDDA) until the accumulation buffer is within RMSE 0.01 of the FP64 expected image of
the estimator (libmdwt's mdwt_render_expected) -- and how long one low-spp frame plus the
learned denoiser (weights in mdwtracker_b200/weights, trained by
mdwtracker_b200/train_denoiser.py) takes to get there; `held_out` repeats it on volumes
generated from a seed the denoiser's training never used.

batch (--no-batch skips it): 64 render requests of mixed resolution, channel count,
voxel format, method, camera and spp rendered per frame through the batch API (one
persistent launch per kernel variant, CUDA-graph replay, autotuned schedule) against the
same requests rendered one after the other.

--impl reference times the reference's path restated on the CPU (the OpenMP oracle,
the reference itself cannot be built: no OptiX/OWL) on the same scene, on all host
cores, each step a set of image rows spread evenly over the frame; rank 0 only.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="c3", choices=["c1", "c2", "c3", "c3ndda", "c3b", "c3bndda"])
    ap.add_argument("--edge", type=int, default=16, choices=[4, 8, 16, 32],
                    help="macrocell edge in voxels of the c3/c3b scenes")
    ap.add_argument("--no-sweep", action="store_true", help="skip the c3 macrocell-edge sweep")
    ap.add_argument("--no-c2", action="store_true", help="skip the extra c2 line")
    ap.add_argument("--impl", default="mdwt", choices=["mdwt", "reference"])
    ap.add_argument("--split", default="rows", choices=["rows", "replicas"],
                    help="N > 1: one frame in row bands over the ranks (gathered), or whole frames per rank")
    ap.add_argument("--flush-mib", type=int, default=512)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU-baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--res", type=int, nargs=2, default=None, help="override the resolution (smaller profiling cases)")
    ap.add_argument("--spp", type=int, default=None, help="override samples per pixel")
    ap.add_argument("--no-ttr", action="store_true", help="skip the time-to-RMSE measurement")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched multi-request measurement")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default tracker schedule (regrouped tracker, trips 4) instead of tuning it")
    ap.add_argument("--regroup", type=int, choices=[0, 1], default=None,
                    help="force the tracker after tuning: 1 regrouped, 0 warp-local")
    ap.add_argument("--rg-blocks", type=int, choices=[0, 1, 2, 3, 4], default=None,
                    help="force the regrouped tracker's blocks per SM after tuning (0: as many as fit)")
    ap.add_argument("--arith", default="exact", choices=["exact", "fast"],
                    help="free-flight arithmetic of the headline line (exact: bit-identical to the oracle)")
    ap.add_argument("--no-fast", action="store_true", help="skip the extra fast-arithmetic lines")
    ap.add_argument("--batch-requests", type=int, default=64)
    ap.add_argument("--ttr-config", default="c3", choices=["c1", "c2", "c3", "c3ndda"])
    ap.add_argument("--ttr-target", type=float, default=0.01)
    return ap.parse_args()


def make_scene(name, res=None, spp=None, edge=16, seed=None):
    """The named scene; `seed` (c2, c3) regenerates its volumes from another seed."""
    from mdwtracker_b200 import synthetic as syn
    kw = {} if seed is None else {"seed": seed}
    if name == "c1":
        sc = syn.scene_c1()
    elif name == "c2":
        sc = syn.scene_c2(**kw)
    elif name == "c3":
        sc = syn.scene_c3(mode=2, edge=edge, **kw)
    elif name == "c3ndda":
        sc = syn.scene_c3(mode=0, edge=edge, **kw)
    elif name == "c3b":
        sc = syn.scene_c3b(mode=2, edge=edge)
    elif name == "c3bndda":
        sc = syn.scene_c3b(mode=0, edge=edge)
    else:
        raise ValueError(name)
    if seed is not None:
        sc.name += f"_seed{seed}"
    if res is not None:
        sc.resolution = (int(res[0]), int(res[1]))
    if spp is not None:
        sc.spp = int(spp)
    return sc


def workload_name(sc):
    w, h = sc.resolution
    frames = f"x{sc.frames}frames" if sc.frames > 1 else ""
    return f"{sc.name}_mc{sc.macrocells[0]}_{w}x{h}_{sc.spp}spp{frames}"


def scene_config(sc, l2note, parallelism):
    v = sc.volumes[0]
    return {
        "workload": workload_name(sc),
        "mode": sc.mode,
        "channels": len(sc.volumes),
        "volume": f"{v.shape[2]}x{v.shape[1]}x{v.shape[0]} {v.dtype}",
        "macrocells": list(sc.macrocells),
        "resolution": list(sc.resolution),
        "spp": sc.spp,
        "camera": "default (eye (0.5,0.5,3.0) -> centre, fovy 45)",
        "l2": l2note,
        "parallelism": parallelism,
    }


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(kernel, workload):
    """DRAM bytes per tracker launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("dram_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = os.path.join("/tmp", f"mdwt_clocks_{os.getpid()}.csv")

    def _lines(self):
        try:
            with open(self.path) as f:
                return f.read().splitlines()
        except OSError:
            return []

    def start(self):
        """Start sampling every 20 ms and return once the first sample is written; samples
        before mark() are not counted."""
        self.mark_at = 0
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu_id), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.perf_counter()
        while not self._lines() and time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
            time.sleep(0.01)
        self.mark()

    def mark(self):
        """The timed region starts: later samples are the ones counted."""
        self.mark_at = len(self._lines())

    def stop(self):
        if self.proc is None:
            return None
        # the sample that covers the end of the timed region (at most one interval later)
        t0 = time.perf_counter()
        while len(self._lines()) <= self.mark_at and time.perf_counter() - t0 < 0.5 and self.proc.poll() is None:
            time.sleep(0.005)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self._lines()[self.mark_at:]:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def spread_rows(o, h, budget_s):
    """Rows spread evenly over the frame for a CPU sample of about `budget_s` seconds:
    calibrated on one row at the middle of the frame (among the heaviest), then every
    stride-th row from stride // 2.  Returns (row0, stride)."""
    t0 = time.perf_counter()
    o.renderRowStride(h // 2, h)
    dt1 = max(time.perf_counter() - t0, 1e-4)
    rows = int(max(1, min(h, budget_s / dt1)))
    stride = max(1, h // rows)
    return stride // 2, stride


def cpu_baseline(sc, budget_s):
    """Oracle on the host cores over rows spread evenly over the same frame."""
    from oracle import oracle as orc
    threads = orc.set_threads(len(os.sched_getaffinity(0)))
    o = sc.setup(orc.OracleRenderer())
    w, h = sc.resolution
    r0, stride = spread_rows(o, h, budget_s)
    t0 = time.perf_counter()
    rows = o.renderRowStride(r0, stride)
    el = time.perf_counter() - t0
    ps = rows * w * sc.spp
    return {"value": ps / el / 1e9, "unit": "Gpath-samples/s", "cores": threads, "kind": "port",
            "sample": f"{rows} rows spread over the {w}x{h} frame (every {stride}th from row {r0}) at "
                      f"{sc.spp} spp ({ps} path-samples, {el:.1f} s)"}, o


# volume seed of the held-out time-to-RMSE scene: the denoiser's training frames came from
# the default c3 (seed 3) and c2 (seed 2) volumes only
HELD_OUT_SEED = 11


def time_to_rmse(name, target, device_index, max_frames=20000, seed=None):
    """Plain accumulation until the accumulation buffer's RGB is within `target` RMSE of
    the FP64 expected image: one sample per frame (frame f draws with seed factor f+1, so
    no two samples of the run share a seed); the first 16 frames one by one, then blocks
    of 8 frames per launch (mdwt_render_frames), the RMSE checked on the device after
    each.  Time = device time of the frames (CUDA events on the render stream) up to the
    first check that meets the target."""
    import torch
    from mdwtracker_b200 import Renderer
    sc = make_scene(name, seed=seed)
    r = sc.setup(Renderer(device_index))
    w, h = sc.resolution
    r.setSpp(1)
    # the tracker schedule for this scene, tuned on the 8-frame launches that make up the
    # plain accumulation (the denoised path's single frame is insensitive to it)
    r.autotuneSchedule(frames=8)
    plain_schedule = schedule_of(r, "mdwt_autotune_schedule")
    t0 = time.perf_counter()
    coarse = r.expectedImage(4, 0.5)
    ref = r.expectedImage(8, 0.25)          # stays on the device for accumRmse
    t_ref = time.perf_counter() - t0
    quad = float(np.sqrt(np.mean((coarse - ref) ** 2)))
    r.setSpp(1)
    r.ResetAccumulation()
    stream = torch.cuda.Stream(torch.device("cuda", device_index))
    evs, trace = [], []
    frames, rmse = 0, None
    torch.cuda.synchronize()
    tw = time.perf_counter()
    while frames < max_frames:
        # the first 16 frames one by one, then blocks of 8 frames in one launch
        # (mdwt_render_frames: the same frames as 8 Render calls), checked after each
        n = 1 if frames < 16 else 8
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r.RenderFrames(n, stream.cuda_stream)
        b.record(stream)
        evs.append((a, b))
        frames += n
        torch.cuda.synchronize()
        rmse = r.accumRmse()
        if frames in (1, 4, 16, 64) or frames % 256 == 0:
            trace.append([frames, rmse])
        if rmse <= target:
            break
    torch.cuda.synchronize()
    wall = time.perf_counter() - tw
    dev_ms = sum(a.elapsed_time(b) for a, b in evs)
    denoised = None
    try:
        denoised = denoised_time_to_rmse(r, target, stream)
    except Exception as ex:  # reported, never required
        denoised = {"error": str(ex)}
    r.close()
    if denoised and denoised.get("device_ms"):
        denoised["speedup_vs_plain"] = dev_ms / denoised["device_ms"]
    return {
        "target": target, "metric": "RMSE of linear RGB (accumulation buffer) vs the FP64 expected image",
        "volume_seed": seed if seed is not None else "default (the denoiser's training volumes)",
        "workload": workload_name(sc).replace(f"_{sc.spp}spp", ""), "resolution": [w, h], "mode": sc.mode,
        "schedule": plain_schedule,
        "reference": {"kind": "FP64 expected image of the estimator (mdwt_render_expected)",
                      "jitter_points": 8, "step_voxels": 0.25, "seconds": t_ref,
                      "rmse_vs_4_jitter_0.5_voxel": quad},
        "plain": {"reached": rmse is not None and rmse <= target, "frames": frames, "spp_total": frames,
                  "rmse": rmse, "device_ms": dev_ms, "wall_ms": 1e3 * wall,
                  "path_samples": frames * w * h, "trace": trace},
        "denoised": denoised,
    }


def batch_throughput(device_index, n_requests, frames=3, small=False):
    """The batched workload (64 requests of mixed resolution, channel count, format,
    method, camera and spp): one batch frame = one frame of every request through
    libmdwt's batch API (one persistent launch per kernel variant, CUDA-graph replay,
    autotuned schedule), against the same requests rendered one after the other with
    mdwt_render.  Device time from CUDA events."""
    import torch
    from mdwtracker_b200 import Batch, Renderer
    from mdwtracker_b200 import synthetic as syn
    t0 = time.perf_counter()
    scenes = (syn.scenes_c4(n=n_requests, resolutions=((256, 256),), max_spp=4) if small
              else syn.scenes_c4(n=n_requests))
    reqs = [sc.setup(Renderer(device_index)) for sc in scenes]
    setup_s = time.perf_counter() - t0
    paths = sum(sc.resolution[0] * sc.resolution[1] * sc.spp for sc in scenes)
    st = torch.cuda.Stream(torch.device("cuda", device_index))
    # one after the other
    for r in reqs:
        r.Render(st.cuda_stream)
    torch.cuda.synchronize()
    a, b2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    seq = []
    for _ in range(frames):
        a.record(st)
        for r in reqs:
            r.Render(st.cuda_stream)
        b2.record(st)
        torch.cuda.synchronize()
        seq.append(a.elapsed_time(b2))
    # batched, autotuned
    b = Batch(device_index)
    for r in reqs:
        b.add(r)
    t0 = time.perf_counter()
    best = b.autotune(frames=1)
    tune_s = time.perf_counter() - t0
    b.render(st.cuda_stream)
    torch.cuda.synchronize()
    bat = []
    for _ in range(frames):
        b.render(st.cuda_stream)
        bat.append(b.lastMs())
    info = b.info()
    launches = b.traceLaunches()
    # the same schedule with the regroupable requests in one fused launch
    b.setFusion(True)
    b.render(st.cuda_stream)
    torch.cuda.synchronize()
    fus = []
    for _ in range(frames):
        b.render(st.cuda_stream)
        fus.append(b.lastMs())
    launches_fus = b.traceLaunches()
    b.close()
    for r in reqs:
        r.close()
    ms_seq, ms_bat = min(seq), min(bat)
    return {"workload": f"c4_{n_requests}req_{'256x256_1-4spp' if small else 'mixed'}", "requests": n_requests,
            "path_samples_per_frame": paths,
            "batched": {"ms_per_frame": ms_bat, "Gpath_samples_per_s": paths / ms_bat / 1e6,
                        "kernel_variant_groups": info["groups"], "trace_launches": launches,
                        "graph_replays": info["graph_replays"], "autotuned": {"chunk_items": best[0] or "per request", "pool": best[1],
                                                                              "trips": best[2], "seconds": tune_s}},
            "batched_fused": {"ms_per_frame": min(fus), "trace_launches": launches_fus},
            "one_by_one": {"ms_per_frame": ms_seq, "Gpath_samples_per_s": paths / ms_seq / 1e6},
            "speedup": ms_seq / ms_bat, "setup_s": setup_s}


DENOISER_WEIGHTS = os.path.join(ROOT, "mdwtracker_b200", "weights", "denoiser_c3_syncdda.npy")


def denoised_time_to_rmse(r, target, stream, spps=(1, 2, 4, 8, 16, 32, 64), reps=3):
    """One k-spp frame with the denoiser features, then the learned denoiser; the smallest
    k whose denoised image is within `target` RMSE of the FP64 expected image.  Time =
    device time of the frame + the denoiser (CUDA events on the render stream, best of
    `reps` runs after a warm-up of the same k, fresh sample seeds per run)."""
    import torch
    from mdwtracker_b200 import Denoiser
    if not os.path.exists(DENOISER_WEIGHTS):
        return {"error": f"no trained weights at {os.path.relpath(DENOISER_WEIGHTS, ROOT)}"}
    den = Denoiser(torch.cuda.current_device())
    den.load(DENOISER_WEIGHTS)
    w, h = r.fbSize
    out = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
    r.setFeatures(True)
    r.setSpp(1)
    # this path renders one frame per measurement: the tracker schedule is tuned on single
    # frames (the plain path's is tuned on its 8-frame launches)
    single = r.autotuneSchedule(frames=1)
    r.Render(stream.cuda_stream)
    torch.cuda.synchronize()
    den.autotune(r.deviceFeatures(), 1, h, w)   # tensor-core tilings for this frame size
    tried = []
    found = None
    frame = 5_000_000
    for k in spps:
        r.setSpp(k)
        best = None
        for rep in range(reps + 1):
            frame += 1
            r.setFrameId(frame)
            r.ResetAccumulation()
            torch.cuda.synchronize()
            a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            a.record(stream)
            r.Render(stream.cuda_stream)
            b.record(stream)
            den.infer(r.deviceFeatures(), out, 1, h, w, stream.cuda_stream)
            c.record(stream)
            torch.cuda.synchronize()
            if rep == 0:
                continue   # warm-up: buffer growth for this k
            rec = {"render_ms": a.elapsed_time(b), "denoise_ms": b.elapsed_time(c), "rmse": r.imageRmse(out),
                   "plain_rmse_same_frame": r.accumRmse()}
            if best is None or rec["render_ms"] + rec["denoise_ms"] < best["render_ms"] + best["denoise_ms"]:
                best = rec
        best["spp"] = k
        tried.append(best)
        if best["rmse"] <= target:
            found = best
            break
    r.setFeatures(False)
    den.close()
    res = {"weights": os.path.relpath(DENOISER_WEIGHTS, ROOT), "tried": tried,
           "reached": found is not None,
           "schedule": schedule_of(r, "mdwt_autotune_schedule, single frames")}
    if found:
        res.update({"spp": found["spp"], "rmse": found["rmse"], "device_ms": found["render_ms"] + found["denoise_ms"],
                    "render_ms": found["render_ms"], "denoise_ms": found["denoise_ms"]})
    return res


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sc = make_scene(args.config, args.res, args.spp, args.edge)
    from oracle import oracle as orc
    threads = orc.set_threads(len(os.sched_getaffinity(0)))
    o = sc.setup(orc.OracleRenderer())
    w, h = sc.resolution
    # each step: rows spread evenly over the frame, about 6 s of host work
    r0, stride = spread_rows(o, h, 6.0)
    for _ in range(args.warmup):
        o.renderRowStride(r0, max(stride, h // 2))
    times = []
    rows = 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        rows = o.renderRowStride(r0, stride)
        times.append(time.perf_counter() - t0)
    ps = rows * w * sc.spp
    value = ps / statistics.mean(times) / 1e9
    line = {
        "impl": "reference",
        "metric": "Gpath-samples/s", "value": value, "unit": "Gpath-samples/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(times),
        "higher_is_better": True, "scaling": "strong" if args.split == "rows" else "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded)",
        "config": scene_config(sc, "host caches", "host threads"),
        "cpu_baseline": {"value": value, "unit": "Gpath-samples/s", "cores": threads, "kind": "port",
                         "sample": f"each step: {rows} rows spread over the {w}x{h} frame (every {stride}th "
                                   f"from row {r0}) at {sc.spp} spp ({ps} path-samples)"},
        "e2e": {"value": value, "unit": "Gpath-samples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference (OptiX 7 + OWL, GL viewer) cannot be built here; its tracking path "
                "is restated in C++/OpenMP (oracle/mdwt_oracle.cpp) and timed on the host cores",
    }
    print(json.dumps(line))
    return 0


def schedule_of(r, by):
    """The context's tracker schedule (MDWT_TUNE_*): which tracker, its trips, and the
    warp-local tracker's pool and quorum."""
    names = {4: "regroup", 5: "rg_blocks", 2: "trips", 0: "pool", 3: "quorum"}
    out = {v: r.getTuning(k) for k, v in names.items()}
    out["by"] = by
    return out


def algorithmic_bytes(sc, cnt):
    """Algorithmic bytes of the tracker over the counted work: 8*bpv per density sample
    (trilinear footprint), 4*C_read per macrocell visit (majorants; C for syncDDA, 1
    otherwise).  The resolve pass (36 B per pixel) is timed apart."""
    bpv = 1 if all(v.dtype == np.uint8 for v in sc.volumes) else 4
    creads = len(sc.volumes) if sc.mode == 2 else 1
    return 8.0 * bpv * float(cnt[0]) + 4.0 * creads * float(cnt[2])


def timed_frames(r, sc, steps, warmup, flush, stream, barrier=lambda: None, clocks=None):
    """`warmup` untimed steps, then `steps` timed ones (one step = the workload's frames),
    each bracketed by CUDA events on the render stream, with an L2 flush before each step
    outside the events.  Returns the step times, the tracker kernel's times, the counters
    of the timed steps and the number of library launches inside them."""
    import torch
    sptr = stream.cuda_stream

    def step():
        if sc.frames > 1:
            r.RenderFrames(sc.frames, sptr)
        else:
            r.Render(sptr)

    with torch.cuda.stream(stream):
        for _ in range(warmup):
            flush.fill_(1)
            step()
    torch.cuda.synchronize()
    r.resetCounters()
    timed = True
    try:
        r.setTiming(True)
    except Exception:
        timed = False
    launches0 = r.renderInfo()[0]
    # the tracker kernel the frames run: the regrouped one launches 256-thread blocks
    tracker = "trace_regroup_kernel" if r.renderInfo()[3] == 256 else "trace_kernel"
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    barrier()
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.mark()
    trace_ms = []
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.fill_(k & 0xff)
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
            if timed and sc.frames == 1:
                trace_ms.append(r.kernelTimes()[0])  # trace kernel, CUDA events on the render stream
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop() if clocks is not None else None
    step_ms = [a.elapsed_time(b) for a, b in ev]
    return {"step_ms": step_ms, "trace_ms": trace_ms, "counters": r.counters(),
            "launches": r.renderInfo()[0] - launches0, "tracker": tracker, "clocks": clk, "step": step}


def timed_split_frames(br, sc, steps, warmup, flush, stream, barrier, clocks=None):
    """One frame across the ranks: each renders its row band, then the RGBA8 bands are
    all-gathered (NCCL) -- both inside the CUDA events of a step.  The warm-up frames
    re-cut the bands from each rank's measured band time (BandRenderer.rebalance)."""
    import torch
    sptr = stream.cuda_stream
    r = br.r
    bands_seen = []
    for _ in range(warmup):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            br.render(sptr)
            e1.record(stream)
            br.gather_framebuffer(sptr)
        torch.cuda.synchronize()
        bands_seen.append(br.rebalance(e0.elapsed_time(e1) / 1e3))
    torch.cuda.synchronize()
    r.resetCounters()
    timed = True
    try:
        r.setTiming(True)
    except Exception:
        timed = False
    launches0 = r.renderInfo()[0]
    tracker = "trace_regroup_kernel" if r.renderInfo()[3] == 256 else "trace_kernel"
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    barrier()
    torch.cuda.synchronize()
    if clocks is not None:
        clocks.mark()
    trace_ms = []
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.fill_(k & 0xff)
            ev[k][0].record(stream)
            br.render(sptr)
            br.gather_framebuffer(sptr)
            ev[k][1].record(stream)
            if timed:
                trace_ms.append(r.kernelTimes()[0])
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop() if clocks is not None else None
    step_ms = [a.elapsed_time(b) for a, b in ev]
    return {"step_ms": step_ms, "trace_ms": trace_ms, "counters": r.counters(),
            "launches": r.renderInfo()[0] - launches0, "tracker": tracker, "clocks": clk,
            "bands": br.bands, "bands_warmup": bands_seen}


def throughput_summary(sc, t, peak):
    """Gpath-samples/s, the tracker's algorithmic GB/s and its roofline fraction."""
    w, h = sc.resolution
    steps = len(t["step_ms"])
    ms = statistics.mean(t["step_ms"])
    kernel_ms = statistics.mean(t["trace_ms"]) if t["trace_ms"] else ms
    alg = algorithmic_bytes(sc, t["counters"]) / steps
    cnt = t["counters"]
    return {"workload": workload_name(sc), "Gpath_samples_per_s": w * h * sc.spp * sc.frames / (ms / 1e3) / 1e9,
            "ms_per_step": ms, "kernel": t["tracker"], "kernel_ms": kernel_ms,
            "algorithmic_GB_per_s": alg / (kernel_ms / 1e3) / 1e9, "frac_of_measured_hbm": alg / (kernel_ms / 1e3) / 1e9 / peak,
            "density_samples_per_path": float(cnt[0]) / max(1, int(cnt[3])),
            "cells_per_path": float(cnt[2]) / max(1, int(cnt[3]))}


def extra_c2(args, local, flush, stream, peak):
    """The 3 x 256^3 uint8 syncDDA scene at 1024^2 and 64 spp (L2-resident volume),
    tuned and timed like the headline line."""
    from mdwtracker_b200 import Renderer
    sc = make_scene("c2")
    r = sc.setup(Renderer(local))
    if not args.no_autotune:
        r.autotuneSchedule(frames=sc.frames)
    t = timed_frames(r, sc, args.steps, args.warmup, flush, stream)
    out = throughput_summary(sc, t, peak)
    out["schedule"] = schedule_of(r, "default" if args.no_autotune else "mdwt_autotune_schedule")
    r.close()
    return out


def extra_fast(args, local, flush, stream, peak):
    """The headline scene and the C2 scene with the fast free-flight arithmetic
    (mdwt_set_arithmetic: hardware-log2 flight lengths; per-pixel events match the oracle
    on >= 99.9 % of pixels, tested), tuned and timed like the headline line."""
    from mdwtracker_b200 import Renderer
    out = {}
    for name in dict.fromkeys((args.config, "c2")):
        sc = make_scene(name, args.res if name == args.config else None, args.spp if name == args.config else None,
                        args.edge if name == args.config else 16)
        r = sc.setup(Renderer(local))
        r.setArithmetic(True)
        if not args.no_autotune:
            r.autotuneSchedule(frames=sc.frames)
        t = timed_frames(r, sc, args.steps, args.warmup, flush, stream)
        row = throughput_summary(sc, t, peak)
        row["schedule"] = schedule_of(r, "default" if args.no_autotune else "mdwt_autotune_schedule")
        out[name] = row
        r.close()
    return out


def edge_sweep(args, local, flush, stream, peak, edges=(4, 8, 16, 32), steps=3):
    """The 1080p scene (6 x 512^3 float32, 256 spp) over macrocell edges of 4/8/16/32
    voxels, syncDDA and N-DDA: the grid is rebuilt on the same context (mdwt_set_macrocells
    keeps the TFs) and the schedule tuned for each edge; `steps` timed frames each."""
    from mdwtracker_b200 import Renderer
    out = {}
    for name in ("c3", "c3ndda"):
        sc = make_scene(name, args.res, args.spp, 16)
        r = sc.setup(Renderer(local))
        rows = []
        n = sc.volumes[0].shape[0]
        for e in edges:
            mc = max(1, n // e)
            r.macrocellDims = (mc, mc, mc)
            sc.macrocells = (mc, mc, mc)
            sc.name = sc.name.rsplit("_e", 1)[0] + f"_e{e}"
            if not args.no_autotune:
                r.autotuneSchedule(frames=1)
            t = timed_frames(r, sc, steps, 1, flush, stream)
            row = throughput_summary(sc, t, peak)
            row["edge"] = e
            row["schedule"] = schedule_of(r, "default" if args.no_autotune else "mdwt_autotune_schedule")
            rows.append(row)
        out["syncdda" if sc.mode == 2 else "ndda"] = rows
        r.close()
    return out


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import ctypes as C
    import torch
    import torch.distributed as dist
    from mdwtracker_b200 import Renderer

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    sc = make_scene(args.config, args.res, args.spp, args.edge)
    r = sc.setup(Renderer(local))
    if args.arith == "fast":
        r.setArithmetic(True)
    w, h = sc.resolution
    # the tracker schedule is tuned for the workload first (outside the timed region), on
    # launches of the step's shape
    if not args.no_autotune:
        r.autotuneSchedule(frames=sc.frames)
    if args.regroup is not None:
        r.setTuning(4, args.regroup)
    if args.rg_blocks is not None:
        r.setTuning(5, args.rg_blocks)
    schedule = schedule_of(r, ("default" if args.no_autotune else "mdwt_autotune_schedule") +
                           ("" if args.regroup is None else f", regroup forced to {args.regroup}") +
                           ("" if args.rg_blocks is None else f", blocks per SM forced to {args.rg_blocks}"))
    stream = torch.cuda.Stream(dev)
    sptr = stream.cuda_stream
    flush = torch.empty(args.flush_mib << 20, dtype=torch.uint8, device=dev)

    def step():
        if sc.frames > 1:
            r.RenderFrames(sc.frames, sptr)
        else:
            r.Render(sptr)

    split = world > 1 and args.split == "rows" and sc.frames == 1
    br = None
    if split:
        from mdwtracker_b200.multigpu import BandRenderer
        br = BandRenderer(r)
    else:
        # distinct frame seeds per rank: rank r starts r*(warmup+steps) frames later
        for _ in range(rank * (args.warmup + args.steps)):
            step()
    torch.cuda.synchronize(dev)

    def barrier():
        if world > 1:
            dist.barrier()

    # clock sampler: started before the warm-up (its start-up then lies outside the timed
    # region); only the samples written after mark() are counted
    clocks = ClockSampler(torch.cuda.get_device_properties(dev).uuid and f"GPU-{torch.cuda.get_device_properties(dev).uuid}")
    clocks.start()
    if split:
        t = timed_split_frames(br, sc, args.steps, args.warmup, flush, stream, barrier, clocks)
    else:
        t = timed_frames(r, sc, args.steps, args.warmup, flush, stream, barrier, clocks)
    clk = t["clocks"]
    step_ms = t["step_ms"]
    cnt = t["counters"]
    ms = statistics.mean(step_ms)
    if world > 1:
        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    paths = w * h * sc.spp * sc.frames
    value = (1 if split else world) * paths / (ms / 1e3) / 1e9

    steps = args.steps
    alg_bytes = algorithmic_bytes(sc, cnt) / steps
    kernel_ms = statistics.mean(t["trace_ms"]) if t["trace_ms"] else statistics.mean(step_ms)
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    if world > 1:   # the mean over the ranks of each one's achieved GB/s
        tt = torch.tensor([achieved], device=dev, dtype=torch.float64)
        dist.all_reduce(tt)
        achieved = float(tt.item()) / world
    peak, peak_kind = measured_peak_hbm()
    tracker = t["tracker"]

    # ---- end to end through the C ABI with host buffers
    pinned = torch.empty(w * h, dtype=torch.int32, pin_memory=True)
    cam = ((0.5, 0.5, 3.0), (0.5, 0.5, 0.5), (0.0, 1.0, 0.0), 45.0)
    e2e_ms = []
    barrier()
    for k in range(steps):
        flush.fill_(k & 0xff)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        r.setCamera(*cam)
        if split:   # this rank's band, the gathered frame, to pinned host memory
            br.render(sptr)
            with torch.cuda.stream(stream):
                fb = br.gather_framebuffer(sptr)
                pinned.copy_(fb.reshape(-1), non_blocking=True)
            stream.synchronize()
        else:
            step()
            r._call("get_framebuffer", C.cast(C.c_void_p(pinned.data_ptr()), C.POINTER(C.c_uint32)))
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    barrier()
    e2e = statistics.mean(e2e_ms)
    if world > 1:
        tt = torch.tensor([e2e], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e = float(tt.item())
    h2d = r.renderInfo()[1] + 48  # kernel parameter block + camera vectors
    r.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu, _ = cpu_baseline(sc, args.cpu_seconds)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "error": str(ex)}

    extras = {}
    if rank == 0 and world == 1:
        if not args.no_c2 and args.config != "c2":
            try:
                extras["c2"] = extra_c2(args, local, flush, stream, peak)
            except Exception as ex:  # reported beside the throughput line, never required
                extras["c2"] = {"error": str(ex)}
        if not args.no_fast and args.arith == "exact":
            try:
                extras["fast_arith"] = extra_fast(args, local, flush, stream, peak)
            except Exception as ex:
                extras["fast_arith"] = {"error": str(ex)}
        if not args.no_sweep and args.config in ("c3", "c3ndda"):
            try:
                extras["edge_sweep"] = edge_sweep(args, local, flush, stream, peak)
            except Exception as ex:
                extras["edge_sweep"] = {"error": str(ex)}

    ttr = None
    if rank == 0 and world == 1 and not args.no_ttr:
        try:
            ttr = time_to_rmse(args.ttr_config, args.ttr_target, local)
        except Exception as ex:  # reported beside the throughput line, never required
            ttr = {"error": str(ex)}
        # the same measurement on volumes the denoiser never saw in training: the 1080p
        # scene's generator and the uint8 C2 scene's, from another seed
        try:
            ttr["held_out"] = time_to_rmse(args.ttr_config, args.ttr_target, local, seed=HELD_OUT_SEED)
        except Exception as ex:
            ttr["held_out"] = {"error": str(ex)}
        try:
            ttr["held_out_c2"] = time_to_rmse("c2", args.ttr_target, local, seed=HELD_OUT_SEED)
        except Exception as ex:
            ttr["held_out_c2"] = {"error": str(ex)}

    batch = None
    if rank == 0 and world == 1 and not args.no_batch:
        try:
            batch = {"mixed": batch_throughput(local, args.batch_requests),
                     "small": batch_throughput(local, args.batch_requests, small=True)}
        except Exception as ex:  # reported beside the throughput line, never required
            batch = {"error": str(ex)}

    l2note = f"flushed between timed steps ({args.flush_mib} MiB write, outside the timed events)"
    line = {
        "metric": "Gpath-samples/s",
        "value": value,
        "unit": "Gpath-samples/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "strong" if (split or (world == 1 and args.split == "rows")) else "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded generators in mdwtracker_b200/synthetic.py)",
        "config": dict(scene_config(sc, l2note, (f"row bands x{world}, NCCL all_gather of the RGBA8 frame" if split
                                                 else f"replicas x{world}") if world > 1 else "single GPU"),
                       schedule=schedule, arithmetic=args.arith),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": profiled_traffic(tracker, workload_name(sc)),
                     "peak_source": peak_kind, "kernel": tracker,
                     "kernel_ms": kernel_ms, "algorithmic_bytes_per_launch": alg_bytes},
        "cpu_baseline": cpu,
        "e2e": {"value": (1 if split else world) * paths / (e2e / 1e3) / 1e9, "unit": "Gpath-samples/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": w * h * 4, "ms_per_step": e2e},
        "time_to_rmse": ttr,
        "batch": batch,
        "gpu_launches": int(t["launches"]),
        "clocks": clk,
        "counters": {"density_samples": int(cnt[0]), "rejections": int(cnt[1]), "cells": int(cnt[2]),
                     "path_samples": int(cnt[3]), "samples_per_path": float(cnt[0]) / max(1, int(cnt[3]))},
        "step_ms": step_ms,
    }
    if split:
        line["config"]["bands"] = [list(b) for b in t["bands"]]
    line.update(extras)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
