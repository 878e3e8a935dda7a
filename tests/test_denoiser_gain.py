"""What the learned denoiser gains over plain accumulation, measured against the FP64
expected image of the estimator (the same RMSE measure as for plain accumulation).

* the committed network (mdwtracker_b200/weights, trained by train_denoiser.py on the
  6 x 512^3 log-normal scene with random views and transfer functions) on the scene's
  default 1920x1080 view and transfer functions, 4 spp;
* training from scratch on the GPU by the library's kernels, on a small scene, improves
  the RMSE of held-out frames over the plain frames.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WEIGHTS = os.path.join(ROOT, "mdwtracker_b200", "weights", "denoiser_c3_syncdda.npy")


def test_committed_network_beats_plain_accumulation_at_1080p():
    import torch
    from mdwtracker_b200 import Denoiser, Renderer
    from mdwtracker_b200 import synthetic as syn
    sc = syn.scene_c3(mode=2)
    r = sc.setup(Renderer(0))
    r.renderExpected(8, 0.25)
    den = Denoiser(0)
    den.load(WEIGHTS)
    r.setFeatures(True)
    r.setSpp(4)
    r.setFrameId(123457)
    r.Render()
    w, h = r.fbSize
    out = torch.empty((h, w, 4), dtype=torch.float32, device="cuda")
    r.denoise(den, out)
    r.sync()
    plain, denoised = r.accumRmse(), r.imageRmse(out)
    assert denoised < 0.01, (plain, denoised)
    assert denoised < 0.25 * plain, (plain, denoised)


def test_training_from_scratch_improves_held_out_frames():
    import torch
    from mdwtracker_b200 import Denoiser, Renderer
    from mdwtracker_b200 import synthetic as syn
    from mdwtracker_b200.train_denoiser import render_pairs, train
    rng = np.random.default_rng(0)
    vols = [syn.value_noise_sparse(64, occ, 300 + i, octaves=3) for i, occ in enumerate([0.3, 0.4])]
    r = Renderer(0)
    for v in vols:
        r.PushMesh(v)
    r.macrocellDims = (8, 8, 8)
    r.Resize((64, 64))
    r.Init(2)
    for i in range(2):
        r.SetXFColormap(syn.ramp_tf(syn.HUES[i], alpha_max=0.5), i)
        r.SetXFOpacityScale(1.0, i)
        r.SetXFRange((0.0, 1.0), i)
    F, T = render_pairs(r, 192, 64, [4], 256, rng)
    den = Denoiser(0, seed=5)
    train(den, F[:160], T[:160], 400, 16, 1e-3, rng)
    # held-out pairs: mean squared error of the plain 4-spp radiance and of the denoised one
    # against the 256-spp targets
    Fh, Th = F[160:].contiguous(), T[160:].contiguous()
    out = torch.empty_like(Th)
    den.infer(Fh, out, Fh.shape[0], 64, 64)
    torch.cuda.synchronize()
    plain = float(((Fh[..., :3] - Th[..., :3]) ** 2).mean())
    denoised = float(((out[..., :3] - Th[..., :3]) ** 2).mean())
    assert denoised < 0.5 * plain, (plain, denoised)
