"""Seeded synthetic scenes with the shapes of the benchmark configurations.

The reference's experiment scripts render external datasets (nyx, zebrafish,
hurricane, miranda; ``mcSizeExps/*.sh``, ``numChanExps/*.sh``) that are not available
here.  These generators produce volumes with the configured shapes, dtypes and value
distributions instead:

* ``blobs``  -- 64^3 uint8: 16 isotropic Gaussians (sigma 4-12 voxels, amplitude
  0-255) plus uniform noise of +-8, clamped to [0, 255].
* ``value_noise_sparse`` -- N^3 uint8: 4-octave value noise thresholded so that a
  given fraction (10-30 %) of the voxels is non-zero.
* ``lognormal`` -- N^3 float32: 5-octave noise, exp-mapped into [1e-3, 1e3].

Transfer functions are 256-entry RGBA tables with linear opacity ramps 0 -> 1 (the
renderer cubes alpha, renderer.cpp:1100).
"""
from __future__ import annotations

from dataclasses import dataclass, field
import os
import tempfile
from typing import List, Optional, Sequence, Tuple

import numpy as np


def _upsample(lattice: np.ndarray, n: int):
    """Trilinear upsampling of a cubic lattice to n^3 (torch on the CPU: deterministic,
    independent of the thread count)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(lattice, dtype=np.float32))[None, None]
    return torch.nn.functional.interpolate(t, size=(n, n, n), mode="trilinear", align_corners=False)[0, 0]


_CACHE_DIR = os.environ.get("MDWT_SYNTH_CACHE", os.path.join(tempfile.gettempdir(), "mdwt_synth_cache"))


def _cached(key: str, make):
    """Large generated volumes are kept in a temp-dir cache (keyed by generator and
    parameters) so that runs on one machine share identical inputs."""
    path = os.path.join(_CACHE_DIR, key + ".npy")
    if os.path.exists(path):
        try:
            return np.load(path)
        except Exception:
            pass
    v = make()
    if v.nbytes >= (64 << 20):
        try:
            os.makedirs(_CACHE_DIR, exist_ok=True)
            tmp = path + f".{os.getpid()}.tmp"
            np.save(tmp, v)
            os.replace(tmp + ".npy" if not tmp.endswith(".npy") else tmp, path)
        except Exception:
            pass
    return v


def blobs(n: int = 64, nblobs: int = 16, seed: int = 1) -> np.ndarray:
    rng = np.random.default_rng(seed)
    sig = rng.uniform(4.0, 12.0, nblobs)
    amp = rng.uniform(0.0, 255.0, nblobs)
    ctr = rng.uniform(0.0, n, (nblobs, 3))
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    vol = np.zeros((n, n, n), dtype=np.float64)
    for k in range(nblobs):
        d2 = (x - ctr[k, 0]) ** 2 + (y - ctr[k, 1]) ** 2 + (z - ctr[k, 2]) ** 2
        vol += amp[k] * np.exp(-d2 / (2.0 * sig[k] ** 2))
    vol += rng.uniform(-8.0, 8.0, vol.shape)
    return np.clip(np.rint(vol), 0, 255).astype(np.uint8)


def value_noise(n: int, octaves: int, seed: int, base: int = 4) -> np.ndarray:
    """Sum of `octaves` trilinearly upsampled random lattices (4, 8, 16, ... per side),
    amplitude halving per octave."""
    import torch
    rng = np.random.default_rng(seed)
    out = torch.zeros((n, n, n), dtype=torch.float32)
    amp = 1.0
    for o in range(octaves):
        res = min(base * (2 ** o), n)
        lattice = rng.random((res, res, res), dtype=np.float32)
        out += amp * _upsample(lattice, n)
        amp *= 0.5
    return out.numpy()


def value_noise_sparse(n: int = 256, occupancy: float = 0.2, seed: int = 2, octaves: int = 4) -> np.ndarray:
    def make():
        f = value_noise(n, octaves, seed)
        t = np.quantile(f, 1.0 - occupancy)
        hi = float(f.max())
        v = np.where(f > t, 1.0 + 254.0 * (f - t) / max(hi - t, 1e-6), 0.0)
        return np.clip(np.rint(v), 0, 255).astype(np.uint8)
    return _cached(f"vns_{n}_{occupancy}_{seed}_{octaves}", make)


def lognormal(n: int = 512, seed: int = 3, octaves: int = 5) -> np.ndarray:
    """Log-normal field in [1e-3, 1e3]: normalised noise, exp-mapped."""
    def make():
        f = value_noise(n, octaves, seed)
        f = (f - f.mean()) / max(float(f.std()), 1e-6)
        return np.exp(np.clip(f / 3.0, -1.0, 1.0) * np.log(1e3)).astype(np.float32)
    return _cached(f"lgn_{n}_{seed}_{octaves}", make)


def lognormal_log10(n: int = 512, seed: int = 3, octaves: int = 5) -> np.ndarray:
    """The log-normal field log-scaled into the TF domain: log10 of `lognormal`, [-3, 3]."""
    return _cached(f"lgl_{n}_{seed}_{octaves}", lambda: np.log10(lognormal(n, seed, octaves)).astype(np.float32))


def ramp_tf(rgb: Sequence[float], n: int = 256, alpha_max: float = 1.0, start: float = 0.0) -> np.ndarray:
    """n RGBA texels: colour fades in with the ramp, opacity rises linearly from 0 at
    `start` to alpha_max at the top of the range."""
    x = np.linspace(0.0, 1.0, n, dtype=np.float32)
    tf = np.empty((n, 4), dtype=np.float32)
    for k in range(3):
        tf[:, k] = rgb[k] * (0.35 + 0.65 * x)
    tf[:, 3] = alpha_max * np.clip((x - start) / max(1.0 - start, 1e-6), 0.0, 1.0)
    return tf


def viridis_like(n: int = 256) -> np.ndarray:
    x = np.linspace(0.0, 1.0, n, dtype=np.float32)
    tf = np.empty((n, 4), dtype=np.float32)
    tf[:, 0] = np.clip(1.6 * x - 0.4, 0, 1)
    tf[:, 1] = np.clip(0.1 + 0.85 * x, 0, 1)
    tf[:, 2] = np.clip(0.55 + 0.3 * np.sin(3.0 * x), 0, 1)
    tf[:, 3] = x
    return tf


HUES = [(1.0, 0.2, 0.15), (0.2, 1.0, 0.25), (0.2, 0.35, 1.0), (1.0, 0.85, 0.2), (0.9, 0.3, 1.0), (0.2, 0.95, 0.95),
        (1.0, 0.55, 0.1), (0.6, 0.6, 0.6), (0.5, 1.0, 0.5), (1.0, 0.5, 0.7), (0.4, 0.4, 1.0), (0.8, 0.8, 0.3)]


@dataclass
class Scene:
    """One render configuration: channels, TFs, grid, method and frame settings."""
    name: str
    volumes: List[np.ndarray]
    tfs: List[np.ndarray]
    mode: int
    macrocells: Tuple[int, int, int]
    resolution: Tuple[int, int]
    spp: int
    frames: int = 1
    opacity: List[float] = field(default_factory=list)
    xf_range: List[Tuple[float, float]] = field(default_factory=list)
    camera: Optional[Tuple] = None   # (from, at, up, fovy) or None for the default camera
    dt: Optional[float] = None

    def setup(self, r, resolution: Optional[Tuple[int, int]] = None, spp: Optional[int] = None):
        """Configure a Renderer (product or oracle) like viewer.cpp:486-509 does."""
        for v in self.volumes:
            r.PushMesh(v)
        r.macrocellDims = self.macrocells
        res = resolution or self.resolution
        r.Resize(res)
        r.Init(self.mode, self.camera is None)
        if self.dt is not None:
            r.Setdt(self.dt)
        if self.camera is not None:
            r.setCamera(*self.camera)
        for i, tf in enumerate(self.tfs):
            r.SetXFColormap(tf, i)
            r.SetXFOpacityScale(self.opacity[i] if self.opacity else 1.0, i)
            r.SetXFRange(self.xf_range[i] if self.xf_range else (0.0, 1.0), i)
        r.setSpp(spp or self.spp)
        return r

    @property
    def nbytes(self) -> int:
        return int(sum(v.nbytes for v in self.volumes))


def scene_c1(seed: int = 1) -> Scene:
    """N-DDA, 1 channel 64^3 uint8 blobs, macrocell 8^3, 512x512, 1 spp x 16 frames."""
    return Scene("c1_ndda_64u8", [blobs(64, 16, seed)], [viridis_like()], mode=0, macrocells=(8, 8, 8),
                 resolution=(512, 512), spp=1, frames=16)


def scene_c2(seed: int = 2, n: int = 256) -> Scene:
    """syncDDA, 3 channels n^3 uint8 sparse value noise (10/20/30 %), macrocell 16^3 voxels,
    1024x1024, 64 spp."""
    occ = [0.10, 0.20, 0.30]
    vols = [value_noise_sparse(n, occ[i], seed * 17 + i) for i in range(3)]
    tfs = [ramp_tf(HUES[i]) for i in range(3)]
    mc = max(1, n // 16)
    return Scene(f"c2_syncdda_3x{n}u8", vols, tfs, mode=2, macrocells=(mc, mc, mc), resolution=(1024, 1024), spp=64)


def scene_c3(seed: int = 3, n: int = 512, channels: int = 6, edge: int = 16, mode: int = 2) -> Scene:
    """N-DDA / syncDDA, `channels` x n^3 float32 log-normal fields log-scaled into the
    TF domain (log10, [-3, 3]), macrocell edge `edge` voxels, 1920x1080, 256 spp.  The
    opacity ramps start at the middle of the range (the upper half of each field is
    visible), alpha_max 0.25 before cubing: a semi-transparent turbulent medium."""
    vols = [lognormal_log10(n, seed * 31 + i) for i in range(channels)]
    tfs = [ramp_tf(HUES[i % len(HUES)], alpha_max=0.25, start=0.5) for i in range(channels)]
    mc = max(1, n // edge)
    return Scene(f"c3_{'syncdda' if mode == 2 else 'ndda'}_{channels}x{n}f32_e{edge}", vols, tfs, mode=mode,
                 macrocells=(mc, mc, mc), resolution=(1920, 1080), spp=256)


def scene_c3b(seed: int = 5, n: int = 1024, channels: int = 3, edge: int = 16, mode: int = 2) -> Scene:
    """The HBM-bound variant of the 1080p scene: `channels` x n^3 float32 log-normal fields
    (3 x 1024^3 = 12 GB), otherwise as scene_c3."""
    vols = [lognormal_log10(n, seed * 31 + i) for i in range(channels)]
    tfs = [ramp_tf(HUES[i % len(HUES)], alpha_max=0.25, start=0.5) for i in range(channels)]
    mc = max(1, n // edge)
    return Scene(f"c3b_{'syncdda' if mode == 2 else 'ndda'}_{channels}x{n}f32_e{edge}", vols, tfs, mode=mode,
                 macrocells=(mc, mc, mc), resolution=(1920, 1080), spp=256)


def scenes_c4(seed: int = 4, n: int = 64, resolutions=((256, 256), (512, 512), (1024, 1024), (1920, 1080)),
              max_spp: int = 64) -> List[Scene]:
    """Batched workload: `n` render requests with resolutions drawn from {256^2, 512^2,
    1024^2, 1920x1080}, 1-8 channels drawn from the 64^3 blob and 256^3 sparse-noise
    generators (all uint8 or all float32 per request), -m 0 or -m 2, macrocells of 8 / 16
    voxels, 1-64 spp, a random camera on the bounding sphere (distance 2.5, fovy 45) and
    random transfer functions.  Volumes come from a small seeded pool shared by the
    requests."""
    rng = np.random.default_rng(seed)
    pool_u8 = [blobs(64, 16, 100 + i) for i in range(3)] + [value_noise_sparse(256, occ, 200 + i)
                                                          for i, occ in enumerate([0.1, 0.2, 0.3])]
    pool_f32 = [(v.astype(np.float32) / 255.0) for v in pool_u8]
    out = []
    for i in range(n):
        use_f32 = bool(rng.integers(0, 2))
        pool = pool_f32 if use_f32 else pool_u8
        nch = int(rng.integers(1, 9))
        idx = rng.integers(0, len(pool), nch)
        vols = [pool[j] for j in idx]
        big = any(v.shape[0] == 256 for v in vols)
        mc = 16 if big else 8
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        eye = tuple(float(x) for x in (0.5 + 2.5 * d))
        up = (0.0, 1.0, 0.0) if abs(d[1]) < 0.95 else (1.0, 0.0, 0.0)
        tfs = [ramp_tf(tuple(float(x) for x in rng.uniform(0.2, 1.0, 3)), alpha_max=float(rng.uniform(0.5, 1.0)))
               for _ in range(nch)]
        out.append(Scene(f"c4_req{i}", vols, tfs, mode=int(rng.choice([0, 2])), macrocells=(mc, mc, mc),
                         resolution=tuple(resolutions[int(rng.integers(0, len(resolutions)))]),
                         spp=int(rng.integers(1, max_spp + 1)),
                         camera=(eye, (0.5, 0.5, 0.5), up, 45.0)))
    return out
