// mdwt_nn.cu -- kernels of the learned denoiser (a 3-level convolutional U-Net on BF16
// NHWC activations, FP32 accumulation and FP32 master weights).
//
//   conv3x3_fwd   implicit-GEMM 3x3 convolution, zero padding: M = pixels of one image
//                 row segment, N = output channels, K = 9 taps x input channels; bias,
//                 ReLU and BF16 or FP32 output fused in the epilogue.  Also the data
//                 gradient (a forward convolution with the taps flipped and the weight
//                 matrix transposed).
//   conv3x3_wgrad weight gradient dW[tap][co][ci] = sum_p dY[p][co] X[p + tap][ci], per
//                 tap a GEMM over pixels, split over pixel chunks, FP32 atomics.
//   the rest      ReLU backward, 2x2 average pool and its backward, nearest 2x upsample
//                 + channel concat and its backward, bias gradient, feature packing,
//                 the residual output + MSE loss and its gradient, Adam with the BF16
//                 weight copies for both convolution directions.
// Tensor-core instructions: mma.sync m16n8k16 BF16 -> FP32 with ldmatrix fragment loads
// and cp.async double-buffered shared-memory staging.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "mdwt_nn.h"

namespace mdwt {
namespace nn {
namespace {

typedef __nv_bfloat16 bf16;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool valid) {
  const uint32_t n = valid ? 16u : 0u;   // 0 source bytes: the 16 destination bytes are zero-filled
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(smem)), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }

__device__ __forceinline__ void ldsm_x4(uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3, const void *p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t &r0, uint32_t &r1, uint32_t &r2, uint32_t &r3, const void *p) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(smem_u32(p)));
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// ------------------------------------------------------------------ conv3x3 forward
// CTA: 64 pixels of one image row x 64 output channels, 4 warps of 16 pixels each.
// K steps of 16 input channels of one tap; two shared-memory stages.
constexpr int kFM = 64, kFN = 64, kFK = 16, kFS = 24;   // tile M, N, K; smem row stride (bf16)

__global__ void __launch_bounds__(128) conv3x3_fwd_kernel(const bf16 *__restrict__ X, const bf16 *__restrict__ Wt,
                                                          const float *__restrict__ bias, void *Y, int N, int H,
                                                          int W, int Cin, int Cout, int relu, int outF32) {
  __shared__ __align__(128) bf16 As[2][kFM * kFS];
  __shared__ __align__(128) bf16 Bs[2][kFN * kFS];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int tilesX = (W + kFM - 1) / kFM;
  const int bx = blockIdx.x;
  const int x0 = (bx % tilesX) * kFM;
  const int y = (bx / tilesX) % H;
  const int n = bx / (tilesX * H);
  const int co0 = blockIdx.y * kFN;
  const int kcs = Cin / kFK;
  const int steps = 9 * kcs;

  // loader: thread -> (row, 16-byte chunk) of A and of B
  const int lrow = tid >> 1, lch = tid & 1;
  auto load = [&](int stage, int step) {
    const int tap = step / kcs, kc = step - tap * kcs;
    const int dy = tap / 3 - 1, dx = tap % 3 - 1;
    const int yy = y + dy, xx = x0 + lrow + dx;
    const bool va = (yy >= 0 && yy < H && xx >= 0 && xx < W && x0 + lrow < W);
    const bf16 *src = va ? X + ((((size_t)n * H + yy) * W + xx) * Cin + kc * kFK + lch * 8) : X;
    cp_async16(&As[stage][lrow * kFS + lch * 8], src, va);
    const int co = co0 + lrow;
    const bool vb = co < Cout;
    const bf16 *wsrc = vb ? Wt + (((size_t)tap * Cout + co) * Cin + kc * kFK + lch * 8) : Wt;
    cp_async16(&Bs[stage][lrow * kFS + lch * 8], wsrc, vb);
    cp_async_commit();
  };

  float acc[8][4];
#pragma unroll
  for (int j = 0; j < 8; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;

  load(0, 0);
  for (int s = 0; s < steps; s++) {
    if (s + 1 < steps) {
      load((s + 1) & 1, s + 1);
      cp_async_wait1();
    } else {
      cp_async_wait0();
    }
    __syncthreads();
    const bf16 *as = As[s & 1], *bs = Bs[s & 1];
    uint32_t a0, a1, a2, a3;
    ldsm_x4(a0, a1, a2, a3, as + (warp * 16 + (lane & 15)) * kFS + (lane >> 4) * 8);
#pragma unroll
    for (int j = 0; j < 8; j += 2) {
      uint32_t b0, b1, b2, b3;
      ldsm_x4(b0, b1, b2, b3, bs + (j * 8 + (lane & 7) + ((lane >> 4) << 3)) * kFS + ((lane >> 3) & 1) * 8);
      mma_bf16(acc[j], a0, a1, a2, a3, b0, b1);
      mma_bf16(acc[j + 1], a0, a1, a2, a3, b2, b3);
    }
    __syncthreads();
  }

  // epilogue: rows g and g+8 of the warp's 16 pixels, columns 2t, 2t+1 of each n8 tile
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int px = x0 + warp * 16 + g + 8 * h;
    if (px >= W) continue;
    const size_t pix = ((size_t)n * H + y) * W + px;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int co = co0 + j * 8 + 2 * t;
      if (co >= Cout) continue;
      float v0 = acc[j][2 * h], v1 = acc[j][2 * h + 1];
      if (bias) { v0 += bias[co]; v1 += bias[co + 1]; }
      if (relu) { v0 = fmaxf(v0, 0.f); v1 = fmaxf(v1, 0.f); }
      if (outF32) {
        *reinterpret_cast<float2 *>(reinterpret_cast<float *>(Y) + pix * Cout + co) = make_float2(v0, v1);
      } else {
        *reinterpret_cast<__nv_bfloat162 *>(reinterpret_cast<bf16 *>(Y) + pix * Cout + co) = __floats2bfloat162_rn(v0, v1);
      }
    }
  }
}

// ------------------------------------------------------------------ conv3x3 weight gradient
// CTA: one tap, 64 output channels x 64 input channels, a chunk of pixels; 4 warps of 16
// output channels.  K steps of 32 pixels; A = dY^T (ldmatrix.trans), B = shifted X.
constexpr int kWM = 64, kWN = 64, kWK = 32, kWS = 72, kWChunk = 2048;

__global__ void __launch_bounds__(128) conv3x3_wgrad_kernel(const bf16 *__restrict__ X, const bf16 *__restrict__ dY,
                                                            float *dW, int N, int H, int W, int Cin, int Cout) {
  __shared__ __align__(128) bf16 Ds[2][kWK * kWS];   // [pixel][co]
  __shared__ __align__(128) bf16 Xs[2][kWK * kWS];   // [pixel][ci]
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ci0 = blockIdx.x * kWN, co0 = blockIdx.y * kWM;
  const int tap = blockIdx.z % 9, chunk = blockIdx.z / 9;
  const int dy = tap / 3 - 1, dx = tap % 3 - 1;
  const long long P = (long long)N * H * W;
  const long long p0 = (long long)chunk * kWChunk;
  const long long pend = p0 + kWChunk < P ? p0 + kWChunk : P;
  const int steps = (int)((pend - p0 + kWK - 1) / kWK);

  // loader: 32 pixels x 8 chunks of 16 B for each of Ds and Xs = 256 + 256; 2 + 2 per thread
  auto load = [&](int stage, int step) {
#pragma unroll
    for (int r = 0; r < 2; r++) {
      const int idx = tid + r * 128;
      const int row = idx >> 3, ch = idx & 7;
      const long long p = p0 + (long long)step * kWK + row;
      const bool inP = p < pend;
      const int x = inP ? (int)(p % W) : 0;
      const int yy0 = inP ? (int)((p / W) % H) : 0;
      const int nn = inP ? (int)(p / ((long long)W * H)) : 0;
      const int co = co0 + ch * 8;
      const bool vd = inP && co < Cout;
      const bf16 *sd = vd ? dY + (size_t)p * Cout + co : dY;
      cp_async16(&Ds[stage][row * kWS + ch * 8], sd, vd);
      const int ys = yy0 + dy, xs = x + dx, ci = ci0 + ch * 8;
      const bool vx = inP && ys >= 0 && ys < H && xs >= 0 && xs < W && ci < Cin;
      const bf16 *sx = vx ? X + (((size_t)nn * H + ys) * W + xs) * Cin + ci : X;
      cp_async16(&Xs[stage][row * kWS + ch * 8], sx, vx);
    }
    cp_async_commit();
  };

  float acc[8][4];
#pragma unroll
  for (int j = 0; j < 8; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  if (steps > 0) load(0, 0);
  for (int s = 0; s < steps; s++) {
    if (s + 1 < steps) {
      load((s + 1) & 1, s + 1);
      cp_async_wait1();
    } else {
      cp_async_wait0();
    }
    __syncthreads();
    const bf16 *ds = Ds[s & 1], *xs = Xs[s & 1];
#pragma unroll
    for (int kk = 0; kk < kWK; kk += 16) {
      uint32_t a0, a1, a2, a3;
      // A[m = co][k = pixel] from ds[pixel][co]
      ldsm_x4_t(a0, a1, a2, a3, ds + (kk + (lane & 7) + ((lane >> 4) << 3)) * kWS + warp * 16 + ((lane >> 3) & 1) * 8);
#pragma unroll
      for (int j = 0; j < 8; j += 2) {
        uint32_t b0, b1, b2, b3;
        // B[k = pixel][n = ci] from xs[pixel][ci]
        ldsm_x4_t(b0, b1, b2, b3, xs + (kk + (lane & 7) + (((lane >> 3) & 1) << 3)) * kWS + j * 8 + (lane >> 4) * 8);
        mma_bf16(acc[j], a0, a1, a2, a3, b0, b1);
        mma_bf16(acc[j + 1], a0, a1, a2, a3, b2, b3);
      }
    }
    __syncthreads();
  }
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int co = co0 + warp * 16 + g + 8 * h;
    if (co >= Cout) continue;
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int ci = ci0 + j * 8 + 2 * t;
      if (ci >= Cin) continue;
      float *d = dW + ((size_t)tap * Cout + co) * Cin + ci;
      atomicAdd(d, acc[j][2 * h]);
      atomicAdd(d + 1, acc[j][2 * h + 1]);
    }
  }
}

// ------------------------------------------------------------------ elementwise
// Channel counts are multiples of 8: one thread moves 8 channels (16 bytes) at a time.
__device__ __forceinline__ void unpack8(const uint4 &u, float f[8]) {
  const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const float2 t = __bfloat1622float2(h[j]);
    f[2 * j] = t.x;
    f[2 * j + 1] = t.y;
  }
}
__device__ __forceinline__ uint4 pack8(const float f[8]) {
  uint4 u;
  __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
  for (int j = 0; j < 4; j++) h[j] = __floats2bfloat162_rn(f[2 * j], f[2 * j + 1]);
  return u;
}

__global__ void relu_bwd_kernel(bf16 *dY, const bf16 *Y, size_t n8) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n8; i += (size_t)gridDim.x * blockDim.x) {
    const uint4 y = reinterpret_cast<const uint4 *>(Y)[i];
    uint4 d = reinterpret_cast<uint4 *>(dY)[i];
    const uint32_t *yw = &y.x;
    uint32_t *dw = &d.x;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      // keep each BF16 half of d where the matching half of y is > 0: sign clear and the
      // magnitude bits in (0, +inf] (NaN compares false)
      const uint32_t ml = yw[j] & 0xffffu, mh = yw[j] >> 16;
      const uint32_t lo = ml >= 0x0001u && ml <= 0x7f80u ? 0x0000ffffu : 0u;
      const uint32_t hi = mh >= 0x0001u && mh <= 0x7f80u ? 0xffff0000u : 0u;
      dw[j] &= lo | hi;
    }
    reinterpret_cast<uint4 *>(dY)[i] = d;
  }
}

// rows of the output (N x Ho) along grid y, a row's elements (Wo x G uint4) along grid x;
// e / G by a multiply-high with the reciprocal `mg` (exact for e * G < 2^32)
__global__ void avgpool2_kernel(const bf16 *X, bf16 *Y, int N, int H, int W, int C, unsigned mg) {
  const unsigned G = (unsigned)C / 8, Ho = (unsigned)H / 2, Wo = (unsigned)W / 2, perRow = Wo * G;
  const uint4 *src = reinterpret_cast<const uint4 *>(X);
  for (unsigned row = blockIdx.y; row < (unsigned)N * Ho; row += gridDim.y) {
    const unsigned b = row / Ho, yo = row - b * Ho;
    const uint4 *in = src + (size_t)(b * (unsigned)H + 2 * yo) * (unsigned)W * G;
    uint4 *out = reinterpret_cast<uint4 *>(Y) + (size_t)row * perRow;
    for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < perRow; e += gridDim.x * blockDim.x) {
      const unsigned xo = G == 1 ? e : __umulhi(e, mg), g = e - xo * G;
      const size_t base = (size_t)(2 * xo) * G + g;
      float a[8], t[8];
      unpack8(in[base], a);
      unpack8(in[base + G], t);
#pragma unroll
      for (int j = 0; j < 8; j++) a[j] += t[j];
      unpack8(in[base + (size_t)W * G], t);
#pragma unroll
      for (int j = 0; j < 8; j++) a[j] += t[j];
      unpack8(in[base + (size_t)W * G + G], t);
#pragma unroll
      for (int j = 0; j < 8; j++) a[j] = 0.25f * (a[j] + t[j]);
      out[e] = pack8(a);
    }
  }
}

// dX[2y+i][2x+j] = dX[..] + dY[y][x] / 4 (accumulates into the skip's gradient)
__global__ void avgpool2_bwd_add_kernel(const bf16 *dY, bf16 *dX, int N, int H, int W, int C) {
  const int G = C / 8;
  const size_t n = (size_t)N * H * W * G;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int g = (int)(i % G);
    size_t r = i / G;
    const int x = (int)(r % W);
    r /= W;
    const int y = (int)(r % H);
    const int b = (int)(r / H);
    float a[8], t[8];
    unpack8(reinterpret_cast<const uint4 *>(dY)[(((size_t)b * (H / 2) + y / 2) * (W / 2) + x / 2) * G + g], t);
    unpack8(reinterpret_cast<uint4 *>(dX)[i], a);
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = a[j] + 0.25f * t[j];
    reinterpret_cast<uint4 *>(dX)[i] = pack8(a);
  }
}

// out[y][x] = concat(coarse[y/2][x/2] (Cu channels), skip[y][x] (Cs channels))
// rows of the output (N x H) along grid y, a row's elements (W x (Gu + Gs) uint4) along
// grid x; e / G by a multiply-high with the reciprocal `mg`
__global__ void up2_concat_kernel(const bf16 *coarse, const bf16 *skip, bf16 *out, int N, int H, int W, int Cu, int Cs,
                                  unsigned mg) {
  const unsigned Gu = (unsigned)Cu / 8, Gs = (unsigned)Cs / 8, G = Gu + Gs, perRow = (unsigned)W * G;
  const unsigned Hc = (unsigned)H / 2, Wc = (unsigned)W / 2;
  for (unsigned row = blockIdx.y; row < (unsigned)N * (unsigned)H; row += gridDim.y) {
    const unsigned b = row / (unsigned)H, y = row - b * (unsigned)H;
    const uint4 *crow = reinterpret_cast<const uint4 *>(coarse) + (size_t)(b * Hc + y / 2) * Wc * Gu;
    const uint4 *srow = reinterpret_cast<const uint4 *>(skip) + (size_t)row * (unsigned)W * Gs;
    uint4 *orow = reinterpret_cast<uint4 *>(out) + (size_t)row * perRow;
    for (unsigned e = blockIdx.x * blockDim.x + threadIdx.x; e < perRow; e += gridDim.x * blockDim.x) {
      const unsigned x = G == 1 ? e : __umulhi(e, mg), g = e - x * G;
      orow[e] = g < Gu ? crow[(x >> 1) * Gu + g] : srow[x * Gs + (g - Gu)];
    }
  }
}

// backward of up2_concat: dCoarse[Y][X] = sum of the 2x2 block of dOut[.., :Cu];
// dSkip = dOut[.., Cu:]
__global__ void up2_concat_bwd_kernel(const bf16 *dOut, bf16 *dCoarse, bf16 *dSkip, int N, int H, int W, int Cu,
                                      int Cs) {
  const int Gu = Cu / 8, Gs = Cs / 8, G = Gu + Gs;
  const int Hc = H / 2, Wc = W / 2;
  const size_t nc = (size_t)N * Hc * Wc * Gu;
  const size_t ns = (size_t)N * H * W * Gs;
  const uint4 *src = reinterpret_cast<const uint4 *>(dOut);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nc + ns; i += (size_t)gridDim.x * blockDim.x) {
    if (i < nc) {
      const int g = (int)(i % Gu);
      size_t r = i / Gu;
      const int x = (int)(r % Wc);
      r /= Wc;
      const int y = (int)(r % Hc);
      const int b = (int)(r / Hc);
      const size_t base = (((size_t)b * H + 2 * y) * W + 2 * x) * G + g;
      float a[8], t[8];
      unpack8(src[base], a);
      unpack8(src[base + G], t);
#pragma unroll
      for (int j = 0; j < 8; j++) a[j] += t[j];
      unpack8(src[base + (size_t)W * G], t);
#pragma unroll
      for (int j = 0; j < 8; j++) a[j] += t[j];
      unpack8(src[base + (size_t)W * G + G], t);
#pragma unroll
      for (int j = 0; j < 8; j++) a[j] += t[j];
      reinterpret_cast<uint4 *>(dCoarse)[i] = pack8(a);
    } else {
      const size_t j = i - nc;
      const int g = (int)(j % Gs);
      const size_t pix = j / Gs;
      reinterpret_cast<uint4 *>(dSkip)[j] = src[pix * G + Gu + g];
    }
  }
}

__global__ void bias_grad_kernel(const bf16 *dY, float *db, size_t P, int C) {
  // block: 256 threads over (pixel lanes x channels); grid-stride over pixels
  const int c = threadIdx.x % C;
  const int lanes = blockDim.x / C;
  const int l = threadIdx.x / C;
  if (l >= lanes) return;
  float s = 0.f;
  for (size_t p = (size_t)blockIdx.x * lanes + l; p < P; p += (size_t)gridDim.x * lanes) s += __bfloat162float(dY[p * C + c]);
  atomicAdd(db + c, s);
}

// Feature packing: fp32 [N][H][W][16] (tracker features) -> bf16 network input
// [N][Hp][Wp][16], zero outside H x W; one pixel per thread.
__global__ void pack_features_kernel(const float *F, bf16 *X, int N, int H, int W, int Hp, int Wp) {
  for (unsigned row = blockIdx.y; row < (unsigned)N * (unsigned)Hp; row += gridDim.y) {
    const unsigned b = row / (unsigned)Hp, y = row - b * (unsigned)Hp;
    for (unsigned x = blockIdx.x * blockDim.x + threadIdx.x; x < (unsigned)Wp; x += gridDim.x * blockDim.x) {
      const size_t i = (size_t)row * (unsigned)Wp + x;
      float f[16];
      if (y < (unsigned)H && x < (unsigned)W) {
        const float4 *src = reinterpret_cast<const float4 *>(F) + ((size_t)(b * (unsigned)H + y) * (unsigned)W + x) * 4;
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const float4 v = src[j];
          f[4 * j] = v.x; f[4 * j + 1] = v.y; f[4 * j + 2] = v.z; f[4 * j + 3] = v.w;
        }
      } else {
#pragma unroll
        for (int j = 0; j < 16; j++) f[j] = 0.f;
      }
      uint4 *dst = reinterpret_cast<uint4 *>(X) + 2 * i;
      dst[0] = pack8(f);
      dst[1] = pack8(f + 8);
    }
  }
}

// out = features.rgb + net[..., 0:3] over the N x H x W pixels (net padded to Hp x Wp);
// with a target: loss partial sums and the gradient d(loss)/d(net) = 2 (out - target) /
// count on channels 0..2 (dO zeroed by the caller elsewhere).
__global__ void residual_out_kernel(const float *F, const float *O, int Co, float *out4, const float *target4,
                                    bf16 *dO, double *lossSum, int N, int H, int W, int Hp, int Wp, float invCount) {
  double s = 0.0;
  for (unsigned row = blockIdx.y; row < (unsigned)N * (unsigned)H; row += gridDim.y) {
    const unsigned b = row / (unsigned)H, y = row - b * (unsigned)H;
    for (unsigned x = blockIdx.x * blockDim.x + threadIdx.x; x < (unsigned)W; x += gridDim.x * blockDim.x) {
      const size_t p = (size_t)row * (unsigned)W + x;
      const size_t q = (size_t)(b * (unsigned)Hp + y) * (unsigned)Wp + x;
      float o[3];
      for (int k = 0; k < 3; k++) o[k] = F[p * 16 + k] + O[q * Co + k];
      if (out4) *reinterpret_cast<float4 *>(out4 + 4 * p) = make_float4(o[0], o[1], o[2], 1.f);
      if (target4) {
        for (int k = 0; k < 3; k++) {
          const float d = o[k] - target4[4 * p + k];
          s += (double)d * d;
          dO[q * Co + k] = __float2bfloat16(2.f * d * invCount);
        }
      }
    }
  }
  if (lossSum) {
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(lossSum, s);
  }
}

// Adam on the FP32 master weights and bias, then the BF16 copies: forward layout
// Wf[tap][co][ci] and the data-gradient layout Wd[tap'][ci][co] = W[8 - tap'][co][ci].
__global__ void adam_kernel(float *Wm, float *mW, float *vW, const float *gW, bf16 *Wf, bf16 *Wd, int Cin, int Cout,
                            float *b, float *mb, float *vb, const float *gb, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
  const size_t nW = (size_t)9 * Cout * Cin;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nW + Cout; i += (size_t)gridDim.x * blockDim.x) {
    if (i < nW) {
      const float g = gW[i];
      const float m = b1 * mW[i] + (1.f - b1) * g;
      const float v = b2 * vW[i] + (1.f - b2) * g * g;
      mW[i] = m;
      vW[i] = v;
      const float w = Wm[i] - lr * (m / c1) / (sqrtf(v / c2) + eps);
      Wm[i] = w;
      const int ci = (int)(i % Cin);
      const size_t r = i / Cin;
      const int co = (int)(r % Cout);
      const int tap = (int)(r / Cout);
      Wf[i] = __float2bfloat16(w);
      Wd[((size_t)(8 - tap) * Cin + ci) * Cout + co] = __float2bfloat16(w);
    } else {
      const size_t j = i - nW;
      const float g = gb[j];
      const float m = b1 * mb[j] + (1.f - b1) * g;
      const float v = b2 * vb[j] + (1.f - b2) * g * g;
      mb[j] = m;
      vb[j] = v;
      b[j] -= lr * (m / c1) / (sqrtf(v / c2) + eps);
    }
  }
}

// BF16 copies of the master weights without an update.
__global__ void weight_copies_kernel(const float *Wm, bf16 *Wf, bf16 *Wd, int Cin, int Cout) {
  const size_t nW = (size_t)9 * Cout * Cin;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nW; i += (size_t)gridDim.x * blockDim.x) {
    const int ci = (int)(i % Cin);
    const size_t r = i / Cin;
    const int co = (int)(r % Cout);
    const int tap = (int)(r / Cout);
    Wf[i] = __float2bfloat16(Wm[i]);
    Wd[((size_t)(8 - tap) * Cin + ci) * Cout + co] = __float2bfloat16(Wm[i]);
  }
}

// grid of row kernels: blocks along x cover a row of perRow elements (256 threads each),
// grid y takes rows (the kernels loop when there are more than 65535)
inline dim3 row_grid(size_t rows, size_t perRow) {
  size_t gx = (perRow + 255) / 256;
  if (gx > 64) gx = 64;
  size_t gy = rows < 65535 ? rows : 65535;
  return dim3((unsigned)(gx ? gx : 1), (unsigned)(gy ? gy : 1));
}
// reciprocal for e / d as __umulhi(e, m), exact while e * d < 2^32 (d = 1 is handled apart)
inline unsigned div_magic(unsigned d) { return d <= 1 ? 0u : (unsigned)(((1ull << 32) + d - 1) / d); }

inline unsigned grid_for(size_t n, int numSMs) {
  size_t g = (n + 255) / 256;
  const size_t cap = (size_t)numSMs * 16;
  if (g > cap) g = cap;
  return (unsigned)(g ? g : 1);
}

}  // namespace

int conv3x3_fwd(const void *X, const void *Wt, const float *bias, void *Y, int N, int H, int W, int Cin, int Cout,
                int relu, int outF32, void *stream) {
  if (Cin % 16 || Cout % 8 || N <= 0 || H <= 0 || W <= 0) return (int)cudaErrorInvalidValue;
  const int tilesX = (W + kFM - 1) / kFM;
  dim3 grid((unsigned)(N * H * tilesX), (unsigned)((Cout + kFN - 1) / kFN));
  conv3x3_fwd_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>((const bf16 *)X, (const bf16 *)Wt, bias, Y, N, H, W, Cin,
                                                             Cout, relu, outF32);
  return (int)cudaGetLastError();
}

int conv3x3_wgrad(const void *X, const void *dY, float *dW, int N, int H, int W, int Cin, int Cout, void *stream) {
  if (Cin % 8 || Cout % 8) return (int)cudaErrorInvalidValue;
  const long long P = (long long)N * H * W;
  const int chunks = (int)((P + kWChunk - 1) / kWChunk);
  dim3 grid((unsigned)((Cin + kWN - 1) / kWN), (unsigned)((Cout + kWM - 1) / kWM), (unsigned)(9 * chunks));
  conv3x3_wgrad_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>((const bf16 *)X, (const bf16 *)dY, dW, N, H, W, Cin,
                                                               Cout);
  return (int)cudaGetLastError();
}

int relu_bwd(void *dY, const void *Y, size_t n, int numSMs, void *stream) {
  if (n % 8) return (int)cudaErrorInvalidValue;
  relu_bwd_kernel<<<grid_for(n / 8, numSMs), 256, 0, (cudaStream_t)stream>>>((bf16 *)dY, (const bf16 *)Y, n / 8);
  return (int)cudaGetLastError();
}

int avgpool2(const void *X, void *Y, int N, int H, int W, int C, int numSMs, void *stream) {
  (void)numSMs;
  if (C % 8 || (size_t)(W / 2) * (C / 8) * (C / 8) >= (1ull << 32)) return (int)cudaErrorInvalidValue;
  avgpool2_kernel<<<row_grid((size_t)N * (H / 2), (size_t)(W / 2) * (C / 8)), 256, 0, (cudaStream_t)stream>>>(
      (const bf16 *)X, (bf16 *)Y, N, H, W, C, div_magic((unsigned)C / 8));
  return (int)cudaGetLastError();
}

int avgpool2_bwd_add(const void *dY, void *dX, int N, int H, int W, int C, int numSMs, void *stream) {
  if (C % 8) return (int)cudaErrorInvalidValue;
  avgpool2_bwd_add_kernel<<<grid_for((size_t)N * H * W * (C / 8), numSMs), 256, 0, (cudaStream_t)stream>>>(
      (const bf16 *)dY, (bf16 *)dX, N, H, W, C);
  return (int)cudaGetLastError();
}

int up2_concat(const void *coarse, const void *skip, void *out, int N, int H, int W, int Cu, int Cs, int numSMs,
               void *stream) {
  (void)numSMs;
  const size_t G = (size_t)(Cu + Cs) / 8;
  if (Cu % 8 || Cs % 8 || (size_t)W * G * G >= (1ull << 32)) return (int)cudaErrorInvalidValue;
  up2_concat_kernel<<<row_grid((size_t)N * H, (size_t)W * G), 256, 0, (cudaStream_t)stream>>>(
      (const bf16 *)coarse, (const bf16 *)skip, (bf16 *)out, N, H, W, Cu, Cs, div_magic((unsigned)G));
  return (int)cudaGetLastError();
}

int up2_concat_bwd(const void *dOut, void *dCoarse, void *dSkip, int N, int H, int W, int Cu, int Cs, int numSMs,
                   void *stream) {
  if (Cu % 8 || Cs % 8) return (int)cudaErrorInvalidValue;
  const size_t n = (size_t)N * (H / 2) * (W / 2) * (Cu / 8) + (size_t)N * H * W * (Cs / 8);
  up2_concat_bwd_kernel<<<grid_for(n, numSMs), 256, 0, (cudaStream_t)stream>>>((const bf16 *)dOut, (bf16 *)dCoarse,
                                                                               (bf16 *)dSkip, N, H, W, Cu, Cs);
  return (int)cudaGetLastError();
}

int bias_grad(const void *dY, float *db, size_t P, int C, int numSMs, void *stream) {
  if (C > 256) return (int)cudaErrorInvalidValue;
  bias_grad_kernel<<<(unsigned)numSMs * 2, (256 / C) * C, 0, (cudaStream_t)stream>>>((const bf16 *)dY, db, P, C);
  return (int)cudaGetLastError();
}

int pack_features(const float *F, void *X, int N, int H, int W, int Hp, int Wp, int numSMs, void *stream) {
  (void)numSMs;
  pack_features_kernel<<<row_grid((size_t)N * Hp, (size_t)Wp), 256, 0, (cudaStream_t)stream>>>(F, (bf16 *)X, N, H, W, Hp,
                                                                                               Wp);
  return (int)cudaGetLastError();
}

int residual_out(const float *F, const float *O, int Co, float *out4, const float *target4, void *dO, double *lossSum,
                 int N, int H, int W, int Hp, int Wp, float invCount, int numSMs, void *stream) {
  (void)numSMs;
  residual_out_kernel<<<row_grid((size_t)N * H, (size_t)W), 256, 0, (cudaStream_t)stream>>>(
      F, O, Co, out4, target4, (bf16 *)dO, lossSum, N, H, W, Hp, Wp, invCount);
  return (int)cudaGetLastError();
}

int adam(float *Wm, float *mW, float *vW, const float *gW, void *Wf, void *Wd, int Cin, int Cout, float *b, float *mb,
         float *vb, const float *gb, float lr, float b1, float b2, float eps, int step, int numSMs, void *stream) {
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  adam_kernel<<<grid_for((size_t)9 * Cin * Cout + Cout, numSMs), 256, 0, (cudaStream_t)stream>>>(
      Wm, mW, vW, gW, (bf16 *)Wf, (bf16 *)Wd, Cin, Cout, b, mb, vb, gb, lr, b1, b2, eps, c1, c2);
  return (int)cudaGetLastError();
}

int weight_copies(const float *Wm, void *Wf, void *Wd, int Cin, int Cout, int numSMs, void *stream) {
  weight_copies_kernel<<<grid_for((size_t)9 * Cin * Cout, numSMs), 256, 0, (cudaStream_t)stream>>>(
      Wm, (bf16 *)Wf, (bf16 *)Wd, Cin, Cout);
  return (int)cudaGetLastError();
}

}  // namespace nn
}  // namespace mdwt
