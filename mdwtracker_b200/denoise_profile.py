"""Profiling target of the learned denoiser (see _main)."""
def _main(argv=None) -> int:
    """python -m mdwtracker_b200.denoise_profile H W [runs] [tune]: inference on random features
    (a profiling target), optionally after autotuning the tilings; prints the device time
    per run."""
    import sys
    import torch
    a = list(argv if argv is not None else sys.argv[1:])
    h, w = int(a[0]), int(a[1])
    runs = int(a[2]) if len(a) > 2 else 2
    from .denoiser import Denoiser
    d = Denoiser(0, seed=1)
    F = torch.rand((1, h, w, 16), device="cuda")
    O = torch.empty((1, h, w, 4), device="cuda")
    if len(a) > 3 and a[3] == "tune":
        d.autotune(F, 1, h, w)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    d.infer(F, O, 1, h, w)
    e0.record()
    for _ in range(runs):
        d.infer(F, O, 1, h, w)
    e1.record()
    d.check()
    torch.cuda.synchronize()
    print(f"{h}x{w}: {e0.elapsed_time(e1) / runs:.3f} ms per inference")
    return 0


if __name__ == "__main__":
    raise SystemExit(_main())
