// mdwt_nn.h -- launchers of the denoiser kernels (mdwt_nn.cu).  Activations are BF16
// NHWC, weights BF16 [tap][co][ci] (forward) / [tap][ci][co] with flipped taps (data
// gradient), master weights, gradients and optimizer state FP32.  Every launcher returns
// a cudaError_t value.
#pragma once
#include <stddef.h>
#include <stdint.h>

namespace mdwt {
namespace nn {

// Y = act(conv3x3(X, Wt) + bias), zero padding; Cin % 16 == 0, Cout % 8 == 0;
// bias may be null; Y is FP32 when outF32, else BF16.
int conv3x3_fwd(const void *X, const void *Wt, const float *bias, void *Y, int N, int H, int W, int Cin, int Cout,
                int relu, int outF32, void *stream);
// dW[tap][co][ci] += sum over pixels of dY[p][co] * X[p shifted by tap][ci] (dW zeroed by the caller)
int conv3x3_wgrad(const void *X, const void *dY, float *dW, int N, int H, int W, int Cin, int Cout, void *stream);
int relu_bwd(void *dY, const void *Y, size_t n, int numSMs, void *stream);
int avgpool2(const void *X, void *Y, int N, int H, int W, int C, int numSMs, void *stream);
// dX (N x H x W x C) += upsampled dY / 4
int avgpool2_bwd_add(const void *dY, void *dX, int N, int H, int W, int C, int numSMs, void *stream);
// out (N x H x W x (Cu + Cs)) = concat(nearest-2x(coarse), skip)
int up2_concat(const void *coarse, const void *skip, void *out, int N, int H, int W, int Cu, int Cs, int numSMs,
               void *stream);
int up2_concat_bwd(const void *dOut, void *dCoarse, void *dSkip, int N, int H, int W, int Cu, int Cs, int numSMs,
                   void *stream);
// db[c] += sum over P pixels of dY[p][c] (db zeroed by the caller), C <= 256
int bias_grad(const void *dY, float *db, size_t P, int C, int numSMs, void *stream);
// X [N][Hp][Wp][16] bf16 = F [N][H][W][16] fp32, zero outside H x W
int pack_features(const float *F, void *X, int N, int H, int W, int Hp, int Wp, int numSMs, void *stream);
// over the N x H x W pixels (O, dO padded to Hp x Wp): out4 (optional) = F.rgb + O[.., 0:3]
// as RGBA (alpha 1); with target4: *lossSum += sum of squared RGB errors and
// dO[.., 0:3] = 2 (out - target) * invCount (the rest of dO zeroed by the caller)
int residual_out(const float *F, const float *O, int Co, float *out4, const float *target4, void *dO, double *lossSum,
                 int N, int H, int W, int Hp, int Wp, float invCount, int numSMs, void *stream);
int adam(float *Wm, float *mW, float *vW, const float *gW, void *Wf, void *Wd, int Cin, int Cout, float *b, float *mb,
         float *vb, const float *gb, float lr, float b1, float b2, float eps, int step, int numSMs, void *stream);
int weight_copies(const float *Wm, void *Wf, void *Wd, int Cin, int Cout, int numSMs, void *stream);

// tcgen05 path (mdwt_nn_tc.cu): the same convolution with the weights in the operand
// layout Wu[dx][ci / 8][dy][co][8] (umma_weights); *err is set when a bounded wait gave up.
// A tcgen05 convolution tiling: R output rows per tile (x 128 pixels), input channels in
// chunks of KC, SA input stages, AB accumulators in tensor memory (2: the epilogue of one
// tile overlaps the MMAs of the next), NS weight stages (NS >= 9 x chunks keeps all the
// weights resident for the launch).
// ST = 1 stacks the three vertical taps into one MMA (N = 3 Cout; needs 3 Cout <= 256).
struct TcTiling {
  int R = 0, KC = 0, NS = 0, SA = 0, AB = 0, ST = 0;
};
bool conv3x3_tc_supported(int Cin, int Cout);
bool conv3x3_tc_valid(int Cin, int Cout, int H, const TcTiling &t);
int conv3x3_tc_candidates(int Cin, int Cout, int H, TcTiling *out, int maxOut);
// Tiling policy: 1 = two accumulators (default), 0 = one accumulator with the most rows.
void conv3x3_tc_policy(int policy);
// Test hook: the next `launches` tensor-core convolutions issue no input loads, so their
// bounded waits give up and set *err (0 = off).
void conv3x3_tc_stall_test(int launches);
// Weight gradient on the tensor cores (tcgen05, MN-major operands from NHWC by TMA):
// dW[tap][co][ci] += sum_p dY[p][co] X[p + tap][ci], the same contract as conv3x3_wgrad.
// Supported for Cout in 8..128 (multiples of 8) and Cin with a chunk of 16, 32 or 48.
bool conv3x3_wgrad_tc_supported(int Cin, int Cout);
int conv3x3_wgrad_tc(const void *X, const void *dY, float *dW, int N, int H, int W, int Cin, int Cout, int *err,
                     void *stream);
int umma_weights(const void *Wf, void *Wu, int Cin, int Cout, int numSMs, void *stream);
// Residual output fused into the epilogue (the denoiser's last layer, inference): instead of
// storing Y, out4[n][y][x] = (F[n][y][x][0..2] + conv[0..2], 1) for y < H, x < W (F has 16
// floats per pixel; the convolution's H x W may be padded beyond them).
struct TcResidual {
  const float *F = nullptr;
  float *out4 = nullptr;
  int H = 0, W = 0;
};
// tiling: null or R == 0 = the default policy's tiling.  poolOut (optional, BF16 output
// only): also write the 2x2 average pooling of Y there, as avgpool2 would, when the tiling
// allows it (an even row count per tile); *pooled tells whether it did.  X2 (optional): the input
// is the channel concatenation of X (C1 channels, a multiple of 8) and X2 (Cin - C1).  pdl:
// launch as a programmatic dependent of the previous kernel in the stream (its set-up
// overlaps that kernel's tail; it must not write what that kernel reads).
int conv3x3_tc(const void *X, const void *Wu, const float *bias, void *Y, int N, int H, int W, int Cin, int Cout,
               int relu, int outF32, int *err, void *stream, const TcTiling *tiling = nullptr,
               const TcResidual *res = nullptr, void *poolOut = nullptr, bool *pooled = nullptr,
               const void *X2 = nullptr, int C1 = 0, int pdl = 0);

}  // namespace nn
}  // namespace mdwt
