"""NumPy restatement of the learned denoiser (forward, loss, backward) for the checks.

TEST INFRASTRUCTURE ONLY: the checker of libmdwt's denoiser kernels
(mdwtracker_b200/csrc/mdwt_nn.cu, mdwt_denoiser.cpp); only tests/ may import it.

The network and parameter layout are those of include/mdwt_denoiser.h: 10 layers of 3x3
convolutions, per layer W[tap][co][ci] (tap = 3 * (dy + 1) + (dx + 1)) then bias[co].
Arithmetic is float64; with ``bf16=True`` every tensor the GPU stores in BF16 (features,
weights, activations, activation gradients) is rounded to BF16 (round to nearest even)
at the same points, so that the GPU result differs only by FP32 accumulation order.
"""
from __future__ import annotations

import numpy as np

SPEC = [(16, 32, 1), (32, 32, 1), (32, 64, 1), (64, 64, 1), (64, 128, 1), (128, 128, 1),
        (192, 64, 1), (64, 64, 1), (96, 32, 1), (32, 16, 0)]


def num_params() -> int:
    return sum(9 * ci * co + co for ci, co, _ in SPEC)


def bf16_round(x):
    a = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((a + 0x7FFF + ((a >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(params):
    out, k = [], 0
    for ci, co, _ in SPEC:
        w = np.asarray(params[k:k + 9 * ci * co], np.float64).reshape(9, co, ci)
        k += 9 * ci * co
        b = np.asarray(params[k:k + co], np.float64)
        k += co
        out.append((w, b))
    return out


def pack(grads):
    return np.concatenate([np.concatenate([g.reshape(-1), gb]) for g, gb in grads])


def _cols(x):
    """im2col: (N, H, W, C) -> (N*H*W, 9*C), zero padding, tap-major."""
    N, H, W, C = x.shape
    xp = np.zeros((N, H + 2, W + 2, C))
    xp[:, 1:-1, 1:-1] = x
    taps = [xp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W] for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
    return np.stack(taps, axis=3).reshape(N * H * W, 9 * C)


def _col2im(dcols, shape):
    N, H, W, C = shape
    d = dcols.reshape(N, H, W, 9, C)
    xp = np.zeros((N, H + 2, W + 2, C))
    t = 0
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            xp[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W] += d[:, :, :, t]
            t += 1
    return xp[:, 1:-1, 1:-1]


def _wmat(w):
    # (9, co, ci) -> (9*ci, co) matching _cols' (tap, ci) order
    return w.transpose(0, 2, 1).reshape(-1, w.shape[1])


def conv(x, w, b, relu):
    N, H, W, _ = x.shape
    y = _cols(x) @ _wmat(w)
    if b is not None:
        y = y + b
    if relu:
        y = np.maximum(y, 0.0)
    return y.reshape(N, H, W, -1)


def pool(x):
    N, H, W, C = x.shape
    return x.reshape(N, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4))


def up2(x):
    return x.repeat(2, axis=1).repeat(2, axis=2)


def forward(params, feats, bf16=True):
    """feats (N, H, W, 16) float32 with H, W multiples of 4 -> (out rgb, cache)."""
    r = bf16_round if bf16 else (lambda v: np.asarray(v, np.float64))
    P = [(r(w), b) for w, b in unpack(params)]
    x0 = r(feats)
    c = {"x0": x0}
    c["a1"] = r(conv(x0, *P[0], 1))
    c["s0"] = r(conv(c["a1"], *P[1], 1))
    c["p0"] = r(pool(c["s0"]))
    c["a2"] = r(conv(c["p0"], *P[2], 1))
    c["s1"] = r(conv(c["a2"], *P[3], 1))
    c["p1"] = r(pool(c["s1"]))
    c["a3"] = r(conv(c["p1"], *P[4], 1))
    c["b2"] = r(conv(c["a3"], *P[5], 1))
    c["u1"] = np.concatenate([up2(c["b2"]), c["s1"]], axis=3)
    c["a4"] = r(conv(c["u1"], *P[6], 1))
    c["b1"] = r(conv(c["a4"], *P[7], 1))
    c["u0"] = np.concatenate([up2(c["b1"]), c["s0"]], axis=3)
    c["a5"] = r(conv(c["u0"], *P[8], 1))
    o = conv(c["a5"], *P[9], 0)
    if bf16:
        o = o.astype(np.float32).astype(np.float64)
    c["o"] = o
    out = np.asarray(feats, np.float64)[..., :3] + o[..., :3]
    return out, (c, P)


def backward(params, feats, target, bf16=True):
    """Loss = mean((out - target.rgb)^2) and the parameter gradients (packed)."""
    r = bf16_round if bf16 else (lambda v: np.asarray(v, np.float64))
    out, (c, P) = forward(params, feats, bf16)
    N, H, W, _ = feats.shape
    count = N * H * W * 3
    d_o = np.zeros((N, H, W, 16))
    if bf16:   # the GPU forms out, the difference and 2 * d * (1 / count) in FP32
        out32 = np.asarray(feats, np.float32)[..., :3] + c["o"][..., :3].astype(np.float32)
        d32 = out32 - np.asarray(target, np.float32)[..., :3]
        diff = d32.astype(np.float64)
        d_o[..., :3] = bf16_round(np.float32(2.0) * d32 * np.float32(1.0 / count))
    else:
        diff = out - np.asarray(target, np.float64)[..., :3]
        d_o[..., :3] = 2.0 * diff / count
    loss = float(np.mean(diff * diff))
    grads = [None] * 10

    def lb(i, x, dy, want_dx=True):
        w, b = P[i]
        cols = _cols(x)
        dyf = dy.reshape(-1, dy.shape[-1])
        gw = (cols.T @ dyf).reshape(9, x.shape[-1], -1).transpose(0, 2, 1)
        grads[i] = (gw, dyf.sum(axis=0))
        if not want_dx:
            return None
        dcols = dyf @ _wmat(w).T
        return r(_col2im(dcols, x.shape))

    def relu_mask(d, y):
        return np.where(y > 0, d, 0.0)

    d_a5 = relu_mask(lb(9, c["a5"], d_o), c["a5"])
    d_u0 = lb(8, c["u0"], d_a5)
    Cu = 64
    d_b1 = r(d_u0[..., :Cu].reshape(N, H // 2, 2, W // 2, 2, Cu).sum(axis=(2, 4)))
    d_s0 = d_u0[..., Cu:]
    d_b1 = relu_mask(d_b1, c["b1"])
    d_a4 = relu_mask(lb(7, c["a4"], d_b1), c["a4"])
    d_u1 = lb(6, c["u1"], d_a4)
    Cu = 128
    d_b2 = r(d_u1[..., :Cu].reshape(N, H // 4, 2, W // 4, 2, Cu).sum(axis=(2, 4)))
    d_s1 = d_u1[..., Cu:]
    d_b2 = relu_mask(d_b2, c["b2"])
    d_a3 = relu_mask(lb(5, c["a3"], d_b2), c["a3"])
    d_p1 = lb(4, c["p1"], d_a3)
    d_s1 = relu_mask(r(d_s1 + 0.25 * up2(d_p1)), c["s1"])
    d_a2 = relu_mask(lb(3, c["a2"], d_s1), c["a2"])
    d_p0 = lb(2, c["p0"], d_a2)
    d_s0 = relu_mask(r(d_s0 + 0.25 * up2(d_p0)), c["s0"])
    d_a1 = relu_mask(lb(1, c["a1"], d_s0), c["a1"])
    lb(0, c["x0"], d_a1, want_dx=False)
    return loss, pack(grads)


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for i, (ci, co, _) in enumerate(SPEC):
        sd = np.sqrt(2.0 / (9 * ci)) * (0.1 if i == len(SPEC) - 1 else 1.0)
        out.append(rng.normal(0, sd, 9 * co * ci))
        out.append(rng.normal(0, 0.05, co))
    return np.concatenate(out).astype(np.float32)
