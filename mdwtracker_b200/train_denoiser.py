"""Train the learned denoiser on frame pairs the tracker renders itself.

  python -m mdwtracker_b200.train_denoiser [--pairs 2000] [--steps 3000] [--out weights.npy]
  torchrun --nproc-per-node N -m mdwtracker_b200.train_denoiser ...   (data-parallel, one GPU per rank)

Data: the 6 x 512^3 float32 log-normal scene and the 3 x 256^3 uint8 sparse-noise scene
(syncDDA; half the pairs each by default), random cameras around the volume
looking at random points inside it with the pixel footprint of the 1920x1080 view (so the
crops have the noise and detail scale of the full frame), random per-channel transfer
functions (hue, opacity maximum, ramp start).  Per pair: a low-spp frame with the
denoiser features (spp drawn from --spp) and a --target-spp accumulation as the target,
rendered at frame ids whose sample seeds do not overlap (every pair uses the same two
frame ids; the pairs differ in camera and transfer functions).  Training: mean squared error
on the RGB, Adam, cosine learning-rate decay, minibatches of crops; forward and backward
run in libmdwt's own kernels (include/mdwt_denoiser.h).

Evaluation (--eval): on the default 1920x1080 view, the RMSE against the FP64 expected
image of the plain k-spp frame and of its denoised version.

Under torchrun (WORLD_SIZE > 1) every rank renders its share of the pairs (its own cameras
and transfer functions), all ranks start from the same weights, and each minibatch of
--batch crops is split over the ranks: multigpu.DataParallelTrainer averages the
gradients with one all-reduce per step (NCCL).  Rank 0 saves and evaluates.
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time

import numpy as np

FOOTPRINT = 2.0 * 2.5 * math.tan(math.radians(22.5)) / 1080.0   # world units per pixel, default view


def seeds(W, H, frame, spp):
    """The tracker's per-sample seed words W*H*(frame+1)*(s+1) mod 2^32."""
    return {(W * H * (frame + 1) * (s + 1)) & 0xFFFFFFFF for s in range(spp)}


def pick_input_frame(res, max_in, target_spp, start=104729):
    """A frame id for the low-spp inputs whose sample seeds miss those of frame 0 (the
    targets' frame) at this resolution."""
    tgt = seeds(res, res, 0, target_spp)
    for f in range(start, start + 100000, 2):
        if not (seeds(res, res, f, max_in) & tgt):
            return f
    raise RuntimeError("no seed-disjoint input frame found")


def random_view(rng, res):
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    dist = rng.uniform(1.8, 3.2)
    centre = np.array([0.5, 0.5, 0.5])
    at = centre + rng.uniform(-0.3, 0.3, 3)
    eye = centre + dist * d
    up = np.array([0.0, 1.0, 0.0]) if abs(d[1]) < 0.95 else np.array([1.0, 0.0, 0.0])
    look = float(np.linalg.norm(eye - at))
    scale = rng.uniform(0.7, 1.4)
    fovy = 2.0 * math.degrees(math.atan(res * FOOTPRINT * scale * (look / 2.5) / (2.0 * look)))
    return tuple(eye), tuple(at), tuple(up), fovy


def random_tfs(rng, n):
    from .synthetic import ramp_tf
    out = []
    for _ in range(n):
        hue = rng.uniform(0.1, 1.0, 3)
        hue /= hue.max()
        out.append(ramp_tf(tuple(hue), alpha_max=rng.uniform(0.12, 0.4), start=rng.uniform(0.3, 0.65)))
    return out


def render_pairs(r, n_pairs, res, spp_choices, target_spp, rng, log=None):
    """(features [n][res][res][16], targets [n][res][res][4]) as CUDA tensors."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    F = torch.empty((n_pairs, res, res, 16), dtype=torch.float32, device=dev)
    T = torch.empty((n_pairs, res, res, 4), dtype=torch.float32, device=dev)
    r.Resize((res, res))
    f_in = pick_input_frame(res, max(spp_choices), target_spp)
    nch = r.numChannels
    for i in range(n_pairs):
        eye, at, up, fovy = random_view(rng, res)
        r.setCamera(eye, at, up, fovy)
        for c, tf in enumerate(random_tfs(rng, nch)):
            r.SetXFColormap(tf, c)
        k = int(rng.choice(spp_choices))
        r.setFeatures(True)
        r.setSpp(k)
        r.setFrameId(f_in)
        r.ResetAccumulation()
        r.Render()
        r.copyFeatures(F[i])
        r.setFeatures(False)
        r.setSpp(target_spp)
        r.setFrameId(0)
        r.ResetAccumulation()
        r.Render()
        r.copyFrameRows(0, res, T[i].data_ptr(), None)
        if log and (i + 1) % 500 == 0:
            torch.cuda.synchronize()
            log(f"  {i + 1}/{n_pairs} pairs")
    torch.cuda.synchronize()
    return F, T


def train(den, F, T, steps, batch, lr0, rng, log=None, trainer=None):
    """Adam with cosine decay on minibatches of `batch` crops; with a data-parallel
    `trainer`, `batch` is this rank's share of the minibatch."""
    import torch
    n, h, w = F.shape[0], F.shape[1], F.shape[2]
    losses = []
    for s in range(steps):
        lr = 1e-5 + 0.5 * (lr0 - 1e-5) * (1.0 + math.cos(math.pi * s / steps))
        idx = torch.from_numpy(rng.integers(0, n, batch)).to(F.device)
        fb = F.index_select(0, idx).contiguous()
        tb = T.index_select(0, idx).contiguous()
        want = (s % 100 == 0) or s == steps - 1
        if trainer is not None:
            loss = trainer.step(fb, tb, batch, h, w, lr, torch.cuda.current_stream().cuda_stream)
        else:
            loss = den.trainStep(fb, tb, batch, h, w, lr, want_loss=want)
        if want:
            losses.append((s, loss))
            if log and s % 500 == 0:
                log(f"  step {s}: loss {loss:.3e} lr {lr:.2e}")
    return losses


def evaluate(r, den, spps, frame_base=3_000_000):
    """RMSE vs the FP64 expected image of k-spp frames, plain and denoised, with the device
    time of the frame and of the denoiser."""
    import torch
    w, h = r.fbSize
    out = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
    st = torch.cuda.Stream()
    res = []
    for k in spps:
        r.setFeatures(True)
        r.setSpp(k)
        r.setFrameId(frame_base + 1000 * k)
        r.ResetAccumulation()
        torch.cuda.synchronize()
        a, b, c = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a.record(st)
        r.Render(st.cuda_stream)
        b.record(st)
        den.infer(r.deviceFeatures(), out, 1, h, w, st.cuda_stream)
        c.record(st)
        torch.cuda.synchronize()
        plain = r.accumRmse()
        dn = r.imageRmse(out)
        res.append({"spp": k, "plain_rmse": plain, "denoised_rmse": dn, "render_ms": a.elapsed_time(b),
                    "denoise_ms": b.elapsed_time(c)})
    r.setFeatures(False)
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=4000)
    ap.add_argument("--res", type=int, default=128)
    ap.add_argument("--spp", type=int, nargs="+", default=[1, 2, 4, 8, 16, 32])
    ap.add_argument("--target-spp", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=16000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--out", default="")
    ap.add_argument("--init", default="", help="start from these weights (.npy)")
    ap.add_argument("--eval", action="store_true")
    ap.add_argument("--eval-spp", type=int, nargs="+", default=[1, 2, 4, 8, 16])
    ap.add_argument("--scenes", nargs="+", default=["c3", "c2"], choices=["c2", "c3"],
                    help="volumes of the training pairs (half the pairs each)")
    a = ap.parse_args(argv)
    import os
    import torch
    from . import Denoiser, Renderer
    from . import synthetic as syn

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    trainer = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        if a.batch % world:
            raise SystemExit(f"--batch {a.batch} must be a multiple of the {world} ranks")
        torch.cuda.set_device(dev)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", dev))

    def log(m):
        if rank == 0:
            print(m, file=sys.stderr, flush=True)

    # each rank renders and samples its own data; the weights start identical on all ranks
    rng = np.random.default_rng(a.seed + 7919 * rank)
    t0 = time.perf_counter()
    sc = syn.scene_c3(mode=2)
    scenes = [sc]
    if "c2" in a.scenes:
        scenes.append(syn.scene_c2())
    if "c3" not in a.scenes:
        scenes = scenes[1:]
    renderers = [s.setup(Renderer(dev)) for s in scenes]
    log(f"scenes ready in {time.perf_counter() - t0:.1f} s")
    den = Denoiser(dev, seed=a.seed)
    if a.init:
        den.load(a.init)
    if world > 1:
        from .multigpu import DataParallelTrainer
        trainer = DataParallelTrainer(den)
    report = {"pairs": a.pairs, "res": a.res, "spp": a.spp, "target_spp": a.target_spp, "steps": a.steps,
              "batch": a.batch, "lr": a.lr, "ranks": world}
    if a.steps > 0:
        t0 = time.perf_counter()
        share = a.pairs // world   # this rank's pairs
        parts = [render_pairs(rr, share // len(renderers), a.res, a.spp, a.target_spp, rng, log) for rr in renderers]
        F = torch.cat([p[0] for p in parts]) if len(parts) > 1 else parts[0][0]
        T = torch.cat([p[1] for p in parts]) if len(parts) > 1 else parts[0][1]
        del parts
        report["data_s"] = time.perf_counter() - t0
        report["scenes"] = [s.name for s in scenes]
        t0 = time.perf_counter()
        losses = train(den, F, T, a.steps, a.batch // world, a.lr, rng, log, trainer)
        torch.cuda.synchronize()
        report["train_s"] = time.perf_counter() - t0
        report["loss_first_last"] = [losses[0][1], losses[-1][1]]
        del F, T
        if a.out and rank == 0:
            den.save(a.out)
    if a.eval and rank == 0:
        r2 = sc.setup(Renderer(dev))
        r2.renderExpected(8, 0.25)
        report["eval"] = evaluate(r2, den, a.eval_spp)
        r2.close()
    if rank == 0:
        print(json.dumps(report))
    for rr in renderers:
        rr.close()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
