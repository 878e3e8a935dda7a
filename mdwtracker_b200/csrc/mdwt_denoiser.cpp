// mdwt_denoiser.cpp -- the learned denoiser's model: layers, parameters, the forward and
// backward passes as sequences of the kernels in mdwt_nn.cu, Adam, and the C ABI of
// include/mdwt_denoiser.h.
//
// Network (H, W padded to multiples of 4; activations BF16 NHWC):
//   x0 (16)  -> L0a 16->32 -> a1 -> L0b 32->32 -> s0 ------------------------------+
//   pool(s0) -> L1a 32->64 -> a2 -> L1b 64->64 -> s1 ----------------+              |
//   pool(s1) -> L2a 64->128 -> a3 -> L2b 128->128 -> b2              |              |
//   concat(up(b2), s1) (192) -> U1a 192->64 -> a4 -> U1b 64->64 -> b1              |
//   concat(up(b1), s0) (96)  -> U0a 96->32 -> a5 -> U0b 32->16 (FP32, no ReLU) -> o
//   output = x0.rgb + o[0:3]
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mdwt_denoiser.h"
#include "mdwt_nn.h"

namespace {

struct LayerSpec {
  int cin, cout, relu;
};
constexpr int kLayers = 10;
constexpr LayerSpec kSpec[kLayers] = {{16, 32, 1}, {32, 32, 1},  {32, 64, 1},  {64, 64, 1}, {64, 128, 1},
                                      {128, 128, 1}, {192, 64, 1}, {64, 64, 1}, {96, 32, 1}, {32, 16, 0}};

struct Layer {
  int cin = 0, cout = 0, relu = 0;
  float *W = nullptr, *b = nullptr;     // FP32 master
  float *mW = nullptr, *vW = nullptr, *mb = nullptr, *vb = nullptr;
  float *gW = nullptr, *gb = nullptr;   // gradients
  void *Wf = nullptr, *Wd = nullptr;    // BF16 forward / data-gradient weights
  void *Wuf = nullptr, *Wud = nullptr;  // the same in the tensor-core operand layout
  size_t nW() const { return (size_t)9 * cin * cout; }
};

struct Acts {
  int N = 0, Hp = 0, Wp = 0;
  size_t bytes = 0;
  void *base = nullptr;
  // forward
  void *x0, *a1, *s0, *p0, *a2, *s1, *p1, *a3, *b2, *u1, *a4, *b1, *u0, *a5;
  float *o;
  // backward
  void *d_o, *d_a5, *d_u0, *d_b1, *d_s0, *d_a4, *d_u1, *d_b2, *d_s1, *d_a3, *d_p1, *d_a2, *d_p0, *d_a1;
  double *loss;
};

}  // namespace

struct mdwt_denoiser {
  int device = 0;
  int numSMs = 0;
  Layer L[kLayers];
  Acts A;
  int step = 0;
  int useTC = 1;          // tcgen05 convolutions where the shapes allow
  // autotuned tcgen05 tilings per layer (forward, data gradient) for one activation shape
  mdwt::nn::TcTiling tileF[kLayers], tileD[kLayers];
  int tunedN = 0, tunedH = 0, tunedW = 0;
  int *dErr = nullptr;    // set by a tensor-core kernel whose bounded wait gave up
  std::string err;
};

namespace {

mdwt_status fail(mdwt_denoiser *d, mdwt_status s, const std::string &m) {
  if (d) d->err = m;
  return s;
}
#define DCK(call, what)                                                                         \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) return fail(d, MDWT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
  } while (0)
#define DCKI(call, what) DCK((cudaError_t)(call), what)

// splitmix64 -> uniform in [0,1)
struct SplitMix {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  double normal() {   // Box-Muller
    const double u1 = uniform() + 1e-300, u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

size_t act_elems(int N, int H, int W, int C) { return (size_t)N * H * W * C; }

mdwt_status ensure_acts(mdwt_denoiser *d, int N, int Hp, int Wp) {
  Acts &A = d->A;
  if (A.base && A.N == N && A.Hp == Hp && A.Wp == Wp) return MDWT_OK;
  if (A.base) cudaFree(A.base);
  A.base = nullptr;
  const int H1 = Hp / 2, W1 = Wp / 2, H2 = Hp / 4, W2 = Wp / 4;
  struct Item {
    void **p;
    size_t bytes;
  };
  std::vector<Item> items;
  auto bf = [&](void **p, int h, int w, int c) { items.push_back({p, act_elems(N, h, w, c) * 2}); };
  bf(&A.x0, Hp, Wp, 16); bf(&A.a1, Hp, Wp, 32); bf(&A.s0, Hp, Wp, 32); bf(&A.p0, H1, W1, 32);
  bf(&A.a2, H1, W1, 64); bf(&A.s1, H1, W1, 64); bf(&A.p1, H2, W2, 64); bf(&A.a3, H2, W2, 128);
  bf(&A.b2, H2, W2, 128); bf(&A.u1, H1, W1, 192); bf(&A.a4, H1, W1, 64); bf(&A.b1, H1, W1, 64);
  bf(&A.u0, Hp, Wp, 96); bf(&A.a5, Hp, Wp, 32);
  items.push_back({(void **)&A.o, act_elems(N, Hp, Wp, 16) * 4});
  bf(&A.d_o, Hp, Wp, 16); bf(&A.d_a5, Hp, Wp, 32); bf(&A.d_u0, Hp, Wp, 96); bf(&A.d_b1, H1, W1, 64);
  bf(&A.d_s0, Hp, Wp, 32); bf(&A.d_a4, H1, W1, 64); bf(&A.d_u1, H1, W1, 192); bf(&A.d_b2, H2, W2, 128);
  bf(&A.d_s1, H1, W1, 64); bf(&A.d_a3, H2, W2, 128); bf(&A.d_p1, H2, W2, 64); bf(&A.d_a2, H1, W1, 64);
  bf(&A.d_p0, H1, W1, 32); bf(&A.d_a1, Hp, Wp, 32);
  items.push_back({(void **)&A.loss, 256});
  size_t total = 0;
  for (auto &it : items) total += (it.bytes + 255) & ~(size_t)255;
  DCK(cudaMalloc(&A.base, total), "denoiser activations");
  size_t off = 0;
  for (auto &it : items) {
    *it.p = (char *)A.base + off;
    off += (it.bytes + 255) & ~(size_t)255;
  }
  A.N = N; A.Hp = Hp; A.Wp = Wp; A.bytes = total;
  return MDWT_OK;
}

bool tuned_for(const mdwt_denoiser *d) {
  return d->tunedN == d->A.N && d->tunedH == d->A.Hp && d->tunedW == d->A.Wp && d->tunedN > 0;
}

// res (optional): fuse the residual output into the tensor-core epilogue; *fused tells
// whether it was (the mma.sync path stores y and leaves the residual to the caller)
// pool (optional): also the 2x2 average pooling of y, fused into the tensor-core epilogue
// when its tiling allows (*pooled tells; otherwise the caller pools)
// x2 (optional, tensor-core path only): the input is the concatenation of x (c1 channels)
// and x2 (the rest)
mdwt_status conv(mdwt_denoiser *d, const Layer &l, const void *x, void *y, int N, int H, int W, bool f32, void *st,
                 const mdwt::nn::TcResidual *res = nullptr, bool *fused = nullptr, void *pool = nullptr,
                 bool *pooled = nullptr, const void *x2 = nullptr, int c1 = 0, int pdl = 0) {
  const int li = (int)(&l - d->L);
  if (fused) *fused = false;
  if (pooled) *pooled = false;
  if (d->useTC && mdwt::nn::conv3x3_tc_supported(l.cin, l.cout)) {
    DCKI(mdwt::nn::conv3x3_tc(x, l.Wuf, l.b, y, N, H, W, l.cin, l.cout, l.relu, f32 ? 1 : 0, d->dErr, st,
                              tuned_for(d) ? &d->tileF[li] : nullptr, res, pool, pooled, x2, c1, pdl),
         "conv forward (tcgen05)");
    if (fused) *fused = res != nullptr;
  } else
    DCKI(mdwt::nn::conv3x3_fwd(x, l.Wf, l.b, y, N, H, W, l.cin, l.cout, l.relu, f32 ? 1 : 0, st), "conv forward");
  return MDWT_OK;
}

// operand-layout copies of both weight layouts (after every weight change)
mdwt_status umma_copies(mdwt_denoiser *d, const Layer &l, void *st) {
  DCKI(mdwt::nn::umma_weights(l.Wf, l.Wuf, l.cin, l.cout, d->numSMs, st), "operand layout");
  DCKI(mdwt::nn::umma_weights(l.Wd, l.Wud, l.cout, l.cin, d->numSMs, st), "operand layout");
  return MDWT_OK;
}

// out4 (optional, inference): the denoised RGBA, fused into the last layer's epilogue when
// the tensor-core path runs it (*fused then true).  Without out4 (training) the decoder
// inputs u1, u0 are the full concatenations the weight gradients read; with it, where the
// tensor-core path runs the decoder layer, only the upsampled channels are materialised
// (in the same buffer) and the convolution reads the skip channels from the skip tensor.
mdwt_status forward(mdwt_denoiser *d, const float *F, int N, int H, int W, void *st, float *out4 = nullptr,
                    bool *fused = nullptr) {
  const int Hp = (H + 3) & ~3, Wp = (W + 3) & ~3;
  mdwt_status s = ensure_acts(d, N, Hp, Wp);
  if (s) return s;
  Acts &A = d->A;
  const int H1 = Hp / 2, W1 = Wp / 2, H2 = Hp / 4, W2 = Wp / 4, S = d->numSMs;
  DCKI(mdwt::nn::pack_features(F, A.x0, N, H, W, Hp, Wp, S, st), "pack features");
  // inference: each convolution a programmatic dependent of the previous kernel (none writes
  // what its predecessor reads)
  const int pd = out4 ? 1 : 0;
  if ((s = conv(d, d->L[0], A.x0, A.a1, N, Hp, Wp, false, st, nullptr, nullptr, nullptr, nullptr, nullptr, 0, pd))) return s;
  bool pooled = false;
  if ((s = conv(d, d->L[1], A.a1, A.s0, N, Hp, Wp, false, st, nullptr, nullptr, A.p0, &pooled, nullptr, 0, pd))) return s;
  if (!pooled) DCKI(mdwt::nn::avgpool2(A.s0, A.p0, N, Hp, Wp, 32, S, st), "pool");
  if ((s = conv(d, d->L[2], A.p0, A.a2, N, H1, W1, false, st, nullptr, nullptr, nullptr, nullptr, nullptr, 0, pd))) return s;
  if ((s = conv(d, d->L[3], A.a2, A.s1, N, H1, W1, false, st, nullptr, nullptr, A.p1, &pooled, nullptr, 0, pd))) return s;
  if (!pooled) DCKI(mdwt::nn::avgpool2(A.s1, A.p1, N, H1, W1, 64, S, st), "pool");
  if ((s = conv(d, d->L[4], A.p1, A.a3, N, H2, W2, false, st, nullptr, nullptr, nullptr, nullptr, nullptr, 0, pd))) return s;
  if ((s = conv(d, d->L[5], A.a3, A.b2, N, H2, W2, false, st, nullptr, nullptr, nullptr, nullptr, nullptr, 0, pd))) return s;
  const bool split6 = out4 && d->useTC && mdwt::nn::conv3x3_tc_supported(d->L[6].cin, d->L[6].cout);
  if (split6) {
    DCKI(mdwt::nn::up2_concat(A.b2, A.b2, A.u1, N, H1, W1, 128, 0, S, st), "upsample");
    if ((s = conv(d, d->L[6], A.u1, A.a4, N, H1, W1, false, st, nullptr, nullptr, nullptr, nullptr, A.s1, 128, pd))) return s;
  } else {
    DCKI(mdwt::nn::up2_concat(A.b2, A.s1, A.u1, N, H1, W1, 128, 64, S, st), "up+concat");
    if ((s = conv(d, d->L[6], A.u1, A.a4, N, H1, W1, false, st))) return s;
  }
  if ((s = conv(d, d->L[7], A.a4, A.b1, N, H1, W1, false, st, nullptr, nullptr, nullptr, nullptr, nullptr, 0, pd))) return s;
  const bool split8 = out4 && d->useTC && mdwt::nn::conv3x3_tc_supported(d->L[8].cin, d->L[8].cout);
  if (split8) {
    DCKI(mdwt::nn::up2_concat(A.b1, A.b1, A.u0, N, Hp, Wp, 64, 0, S, st), "upsample");
    if ((s = conv(d, d->L[8], A.u0, A.a5, N, Hp, Wp, false, st, nullptr, nullptr, nullptr, nullptr, A.s0, 64, pd))) return s;
  } else {
    DCKI(mdwt::nn::up2_concat(A.b1, A.s0, A.u0, N, Hp, Wp, 64, 32, S, st), "up+concat");
    if ((s = conv(d, d->L[8], A.u0, A.a5, N, Hp, Wp, false, st))) return s;
  }
  mdwt::nn::TcResidual res;
  res.F = F; res.out4 = out4; res.H = H; res.W = W;
  if ((s = conv(d, d->L[9], A.a5, A.o, N, Hp, Wp, true, st, out4 ? &res : nullptr, fused, nullptr, nullptr, nullptr, 0, pd)))
    return s;
  return MDWT_OK;
}

// gradients of layer l from its input x and the (post-ReLU-masked) output gradient dy;
// dx (optional) = data gradient
mdwt_status layer_bwd(mdwt_denoiser *d, const Layer &l, const void *x, const void *dy, void *dx, int N, int H, int W,
                      void *st) {
  if (d->useTC && mdwt::nn::conv3x3_wgrad_tc_supported(l.cin, l.cout))
    DCKI(mdwt::nn::conv3x3_wgrad_tc(x, dy, l.gW, N, H, W, l.cin, l.cout, d->dErr, st), "weight gradient (tcgen05)");
  else
    DCKI(mdwt::nn::conv3x3_wgrad(x, dy, l.gW, N, H, W, l.cin, l.cout, st), "weight gradient");
  DCKI(mdwt::nn::bias_grad(dy, l.gb, (size_t)N * H * W, l.cout, d->numSMs, st), "bias gradient");
  if (dx) {
    const int li = (int)(&l - d->L);
    if (d->useTC && mdwt::nn::conv3x3_tc_supported(l.cout, l.cin))
      DCKI(mdwt::nn::conv3x3_tc(dy, l.Wud, nullptr, dx, N, H, W, l.cout, l.cin, 0, 0, d->dErr, st,
                                tuned_for(d) ? &d->tileD[li] : nullptr),
           "data gradient (tcgen05)");
    else
      DCKI(mdwt::nn::conv3x3_fwd(dy, l.Wd, nullptr, dx, N, H, W, l.cout, l.cin, 0, 0, st), "data gradient");
  }
  return MDWT_OK;
}

mdwt_status backward(mdwt_denoiser *d, const float *F, const float *T, int N, int H, int W, void *st) {
  mdwt_status s = forward(d, F, N, H, W, st);
  if (s) return s;
  Acts &A = d->A;
  const int Hp = A.Hp, Wp = A.Wp, H1 = Hp / 2, W1 = Wp / 2, H2 = Hp / 4, W2 = Wp / 4, S = d->numSMs;
  for (auto &l : d->L) {
    DCK(cudaMemsetAsync(l.gW, 0, l.nW() * 4, (cudaStream_t)st), "zero gradients");
    DCK(cudaMemsetAsync(l.gb, 0, (size_t)l.cout * 4, (cudaStream_t)st), "zero gradients");
  }
  DCK(cudaMemsetAsync(A.d_o, 0, act_elems(N, Hp, Wp, 16) * 2, (cudaStream_t)st), "zero output gradient");
  DCK(cudaMemsetAsync(A.loss, 0, sizeof(double), (cudaStream_t)st), "zero loss");
  const float inv = 1.0f / (float)((double)N * H * W * 3);
  DCKI(mdwt::nn::residual_out(F, A.o, 16, nullptr, T, A.d_o, A.loss, N, H, W, Hp, Wp, inv, S, st), "loss");
  // U0b, U0a
  if ((s = layer_bwd(d, d->L[9], A.a5, A.d_o, A.d_a5, N, Hp, Wp, st))) return s;
  DCKI(mdwt::nn::relu_bwd(A.d_a5, A.a5, act_elems(N, Hp, Wp, 32), S, st), "relu backward");
  if ((s = layer_bwd(d, d->L[8], A.u0, A.d_a5, A.d_u0, N, Hp, Wp, st))) return s;
  DCKI(mdwt::nn::up2_concat_bwd(A.d_u0, A.d_b1, A.d_s0, N, Hp, Wp, 64, 32, S, st), "up+concat backward");
  DCKI(mdwt::nn::relu_bwd(A.d_b1, A.b1, act_elems(N, H1, W1, 64), S, st), "relu backward");
  // U1b, U1a
  if ((s = layer_bwd(d, d->L[7], A.a4, A.d_b1, A.d_a4, N, H1, W1, st))) return s;
  DCKI(mdwt::nn::relu_bwd(A.d_a4, A.a4, act_elems(N, H1, W1, 64), S, st), "relu backward");
  if ((s = layer_bwd(d, d->L[6], A.u1, A.d_a4, A.d_u1, N, H1, W1, st))) return s;
  DCKI(mdwt::nn::up2_concat_bwd(A.d_u1, A.d_b2, A.d_s1, N, H1, W1, 128, 64, S, st), "up+concat backward");
  DCKI(mdwt::nn::relu_bwd(A.d_b2, A.b2, act_elems(N, H2, W2, 128), S, st), "relu backward");
  // L2b, L2a
  if ((s = layer_bwd(d, d->L[5], A.a3, A.d_b2, A.d_a3, N, H2, W2, st))) return s;
  DCKI(mdwt::nn::relu_bwd(A.d_a3, A.a3, act_elems(N, H2, W2, 128), S, st), "relu backward");
  if ((s = layer_bwd(d, d->L[4], A.p1, A.d_a3, A.d_p1, N, H2, W2, st))) return s;
  DCKI(mdwt::nn::avgpool2_bwd_add(A.d_p1, A.d_s1, N, H1, W1, 64, S, st), "pool backward");
  DCKI(mdwt::nn::relu_bwd(A.d_s1, A.s1, act_elems(N, H1, W1, 64), S, st), "relu backward");
  // L1b, L1a
  if ((s = layer_bwd(d, d->L[3], A.a2, A.d_s1, A.d_a2, N, H1, W1, st))) return s;
  DCKI(mdwt::nn::relu_bwd(A.d_a2, A.a2, act_elems(N, H1, W1, 64), S, st), "relu backward");
  if ((s = layer_bwd(d, d->L[2], A.p0, A.d_a2, A.d_p0, N, H1, W1, st))) return s;
  DCKI(mdwt::nn::avgpool2_bwd_add(A.d_p0, A.d_s0, N, Hp, Wp, 32, S, st), "pool backward");
  DCKI(mdwt::nn::relu_bwd(A.d_s0, A.s0, act_elems(N, Hp, Wp, 32), S, st), "relu backward");
  // L0b, L0a
  if ((s = layer_bwd(d, d->L[1], A.a1, A.d_s0, A.d_a1, N, Hp, Wp, st))) return s;
  DCKI(mdwt::nn::relu_bwd(A.d_a1, A.a1, act_elems(N, Hp, Wp, 32), S, st), "relu backward");
  if ((s = layer_bwd(d, d->L[0], A.x0, A.d_a1, nullptr, N, Hp, Wp, st))) return s;
  return MDWT_OK;
}

mdwt_status refresh_copies(mdwt_denoiser *d) {
  for (auto &l : d->L) {
    DCKI(mdwt::nn::weight_copies(l.W, l.Wf, l.Wd, l.cin, l.cout, d->numSMs, nullptr), "weights");
    mdwt_status s = umma_copies(d, l, nullptr);
    if (s) return s;
  }
  DCK(cudaDeviceSynchronize(), "weights");
  return MDWT_OK;
}

bool dims_ok(int n, int h, int w) { return n > 0 && h > 0 && w > 0 && (int64_t)n * h * w < (1ll << 31); }

}  // namespace

extern "C" {

int64_t mdwt_denoiser_num_params(void) {
  int64_t n = 0;
  for (auto &s : kSpec) n += (int64_t)9 * s.cin * s.cout + s.cout;
  return n;
}

mdwt_status mdwt_denoiser_create(mdwt_denoiser **out, int device, uint64_t seed) {
  if (!out) return MDWT_ERR_BAD_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return MDWT_ERR_CUDA;
  if (device < 0 || device >= count) return MDWT_ERR_BAD_ARG;
  mdwt_denoiser *d = new mdwt_denoiser();
  d->device = device;
  if (cudaSetDevice(device) != cudaSuccess) { delete d; return MDWT_ERR_CUDA; }
  cudaDeviceGetAttribute(&d->numSMs, cudaDevAttrMultiProcessorCount, device);
  if (cudaMalloc((void **)&d->dErr, sizeof(int)) != cudaSuccess || cudaMemset(d->dErr, 0, sizeof(int)) != cudaSuccess) {
    delete d;
    return MDWT_ERR_CUDA;
  }
  SplitMix rng{seed};
  for (int i = 0; i < kLayers; i++) {
    Layer &l = d->L[i];
    l.cin = kSpec[i].cin; l.cout = kSpec[i].cout; l.relu = kSpec[i].relu;
    const size_t nW = l.nW();
    float **bufs[8] = {&l.W, &l.mW, &l.vW, &l.gW, &l.b, &l.mb, &l.vb, &l.gb};
    for (int k = 0; k < 8; k++) {
      const size_t bytes = (k < 4 ? nW : (size_t)l.cout) * 4;
      if (cudaMalloc((void **)bufs[k], bytes) != cudaSuccess || cudaMemset(*bufs[k], 0, bytes) != cudaSuccess) {
        mdwt_denoiser_destroy(d);
        return MDWT_ERR_CUDA;
      }
    }
    if (cudaMalloc(&l.Wf, nW * 2) != cudaSuccess || cudaMalloc(&l.Wd, nW * 2) != cudaSuccess ||
        cudaMalloc(&l.Wuf, nW * 2) != cudaSuccess || cudaMalloc(&l.Wud, nW * 2) != cudaSuccess) {
      mdwt_denoiser_destroy(d);
      return MDWT_ERR_CUDA;
    }
    // He normal init over fan-in 9*cin; the output layer starts near zero (residual)
    std::vector<float> w(nW);
    const double sd = std::sqrt(2.0 / (9.0 * l.cin)) * (i == kLayers - 1 ? 0.1 : 1.0);
    for (auto &v : w) v = (float)(sd * rng.normal());
    cudaMemcpy(l.W, w.data(), nW * 4, cudaMemcpyHostToDevice);
  }
  if (refresh_copies(d) != MDWT_OK) {
    mdwt_denoiser_destroy(d);
    return MDWT_ERR_CUDA;
  }
  *out = d;
  return MDWT_OK;
}

mdwt_status mdwt_denoiser_destroy(mdwt_denoiser *d) {
  if (!d) return MDWT_ERR_BAD_ARG;
  cudaSetDevice(d->device);
  for (auto &l : d->L) {
    float *bufs[8] = {l.W, l.mW, l.vW, l.gW, l.b, l.mb, l.vb, l.gb};
    for (auto *b : bufs)
      if (b) cudaFree(b);
    if (l.Wf) cudaFree(l.Wf);
    if (l.Wd) cudaFree(l.Wd);
    if (l.Wuf) cudaFree(l.Wuf);
    if (l.Wud) cudaFree(l.Wud);
  }
  if (d->dErr) cudaFree(d->dErr);
  if (d->A.base) cudaFree(d->A.base);
  delete d;
  return MDWT_OK;
}

const char *mdwt_denoiser_last_error(const mdwt_denoiser *d) { return d ? d->err.c_str() : "null denoiser"; }

mdwt_status mdwt_denoiser_get_params(mdwt_denoiser *d, float *out) {
  if (!d || !out) return MDWT_ERR_BAD_ARG;
  DCK(cudaSetDevice(d->device), "cudaSetDevice");
  DCK(cudaDeviceSynchronize(), "sync");
  for (auto &l : d->L) {
    DCK(cudaMemcpy(out, l.W, l.nW() * 4, cudaMemcpyDeviceToHost), "copy weights");
    out += l.nW();
    DCK(cudaMemcpy(out, l.b, (size_t)l.cout * 4, cudaMemcpyDeviceToHost), "copy bias");
    out += l.cout;
  }
  return MDWT_OK;
}

mdwt_status mdwt_denoiser_set_params(mdwt_denoiser *d, const float *in) {
  if (!d || !in) return MDWT_ERR_BAD_ARG;
  DCK(cudaSetDevice(d->device), "cudaSetDevice");
  DCK(cudaDeviceSynchronize(), "sync");
  for (auto &l : d->L) {
    DCK(cudaMemcpy(l.W, in, l.nW() * 4, cudaMemcpyHostToDevice), "copy weights");
    in += l.nW();
    DCK(cudaMemcpy(l.b, in, (size_t)l.cout * 4, cudaMemcpyHostToDevice), "copy bias");
    in += l.cout;
    DCK(cudaMemset(l.mW, 0, l.nW() * 4), "reset Adam");
    DCK(cudaMemset(l.vW, 0, l.nW() * 4), "reset Adam");
    DCK(cudaMemset(l.mb, 0, (size_t)l.cout * 4), "reset Adam");
    DCK(cudaMemset(l.vb, 0, (size_t)l.cout * 4), "reset Adam");
  }
  d->step = 0;
  return refresh_copies(d);
}

mdwt_status mdwt_denoiser_get_grads(mdwt_denoiser *d, float *out) {
  if (!d || !out) return MDWT_ERR_BAD_ARG;
  DCK(cudaSetDevice(d->device), "cudaSetDevice");
  DCK(cudaDeviceSynchronize(), "sync");
  for (auto &l : d->L) {
    DCK(cudaMemcpy(out, l.gW, l.nW() * 4, cudaMemcpyDeviceToHost), "copy gradients");
    out += l.nW();
    DCK(cudaMemcpy(out, l.gb, (size_t)l.cout * 4, cudaMemcpyDeviceToHost), "copy gradients");
    out += l.cout;
  }
  return MDWT_OK;
}

mdwt_status mdwt_denoiser_infer(mdwt_denoiser *d, const float *F, float *out, int n, int h, int w, void *stream) {
  if (!d || !F || !out || !dims_ok(n, h, w)) return fail(d, MDWT_ERR_BAD_ARG, "bad denoiser arguments");
  DCK(cudaSetDevice(d->device), "cudaSetDevice");
  bool fused = false;
  mdwt_status s = forward(d, F, n, h, w, stream, out, &fused);
  if (s) return s;
  if (!fused)
    DCKI(mdwt::nn::residual_out(F, d->A.o, 16, out, nullptr, nullptr, nullptr, n, h, w, d->A.Hp, d->A.Wp, 0.f,
                                d->numSMs, stream),
         "output");
  return MDWT_OK;
}

mdwt_status mdwt_denoiser_backward(mdwt_denoiser *d, const float *F, const float *T, int n, int h, int w, double *loss,
                                   void *stream) {
  if (!d || !F || !T || !dims_ok(n, h, w)) return fail(d, MDWT_ERR_BAD_ARG, "bad denoiser arguments");
  DCK(cudaSetDevice(d->device), "cudaSetDevice");
  mdwt_status s = backward(d, F, T, n, h, w, stream);
  if (s) return s;
  if (loss) {
    double sum = 0.0;
    DCK(cudaMemcpyAsync(&sum, d->A.loss, sizeof(double), cudaMemcpyDeviceToHost, (cudaStream_t)stream), "loss");
    DCK(cudaStreamSynchronize((cudaStream_t)stream), "loss");
    *loss = sum / ((double)n * h * w * 3);
  }
  return MDWT_OK;
}

// One Adam step of every layer from the gradient buffer, and the BF16 operand copies.
static mdwt_status adam_all(mdwt_denoiser *d, float lr, void *stream) {
  mdwt_status s;
  d->step++;
  for (auto &l : d->L) {
    DCKI(mdwt::nn::adam(l.W, l.mW, l.vW, l.gW, l.Wf, l.Wd, l.cin, l.cout, l.b, l.mb, l.vb, l.gb, lr, 0.9f, 0.999f,
                        1e-8f, d->step, d->numSMs, stream),
         "Adam");
    if (d->useTC && (s = umma_copies(d, l, stream))) return s;
  }
  return MDWT_OK;
}

mdwt_status mdwt_denoiser_train_step(mdwt_denoiser *d, const float *F, const float *T, int n, int h, int w, float lr,
                                     double *loss, void *stream) {
  if (!d) return MDWT_ERR_BAD_ARG;
  if (!(lr > 0.0f) || !std::isfinite(lr)) return fail(d, MDWT_ERR_BAD_ARG, "learning rate");
  mdwt_status s = mdwt_denoiser_backward(d, F, T, n, h, w, loss, stream);
  if (s) return s;
  return adam_all(d, lr, stream);
}

mdwt_status mdwt_denoiser_adam_step(mdwt_denoiser *d, float lr, void *stream) {
  if (!d) return MDWT_ERR_BAD_ARG;
  if (!(lr > 0.0f) || !std::isfinite(lr)) return fail(d, MDWT_ERR_BAD_ARG, "learning rate");
  DCK(cudaSetDevice(d->device), "cudaSetDevice");
  return adam_all(d, lr, stream);
}

mdwt_status mdwt_denoiser_copy_grads(mdwt_denoiser *d, float *out, void *stream) {
  if (!d || !out) return MDWT_ERR_BAD_ARG;
  DCK(cudaSetDevice(d->device), "cudaSetDevice");
  for (auto &l : d->L) {
    DCK(cudaMemcpyAsync(out, l.gW, l.nW() * 4, cudaMemcpyDefault, (cudaStream_t)stream), "copy gradients");
    out += l.nW();
    DCK(cudaMemcpyAsync(out, l.gb, (size_t)l.cout * 4, cudaMemcpyDefault, (cudaStream_t)stream), "copy gradients");
    out += l.cout;
  }
  return MDWT_OK;
}

mdwt_status mdwt_denoiser_load_grads(mdwt_denoiser *d, const float *in, void *stream) {
  if (!d || !in) return MDWT_ERR_BAD_ARG;
  DCK(cudaSetDevice(d->device), "cudaSetDevice");
  for (auto &l : d->L) {
    DCK(cudaMemcpyAsync(l.gW, in, l.nW() * 4, cudaMemcpyDefault, (cudaStream_t)stream), "load gradients");
    in += l.nW();
    DCK(cudaMemcpyAsync(l.gb, in, (size_t)l.cout * 4, cudaMemcpyDefault, (cudaStream_t)stream), "load gradients");
    in += l.cout;
  }
  return MDWT_OK;
}

mdwt_status mdwt_denoiser_set_tensor_cores(mdwt_denoiser *d, int mode) {
  if (!d || mode < 0 || mode > 2) return MDWT_ERR_BAD_ARG;
  if (mode >= 1) mdwt::nn::conv3x3_tc_policy(mode == 1 ? 1 : 0);
  if (mode && !d->useTC) {   // operand copies may be stale after mma.sync-path training
    d->useTC = 1;
    return refresh_copies(d);
  }
  d->useTC = mode ? 1 : 0;
  return MDWT_OK;
}

// Time every candidate tiling of one convolution on its real operands; keep the fastest.
static mdwt_status tune_one(mdwt_denoiser *d, int cin, int cout, const void *x, const void *w, const float *bias, void *y,
                            int N, int H, int W, int relu, int f32, mdwt::nn::TcTiling *best, cudaStream_t st) {
  mdwt::nn::TcTiling cand[64];
  const int nc = mdwt::nn::conv3x3_tc_candidates(cin, cout, H, cand, 64);
  cudaEvent_t e0, e1;
  DCK(cudaEventCreate(&e0), "event");
  DCK(cudaEventCreate(&e1), "event");
  float bestMs = 1e30f;
  *best = mdwt::nn::TcTiling();
  for (int i = 0; i < nc; i++) {
    float ms = 1e30f;
    for (int rep = 0; rep < 3; rep++) {
      cudaEventRecord(e0, st);
      const int rc = mdwt::nn::conv3x3_tc(x, w, bias, y, N, H, W, cin, cout, relu, f32, d->dErr, st, &cand[i]);
      cudaEventRecord(e1, st);
      if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return fail(d, MDWT_ERR_CUDA, "tuning launch"); }
      cudaEventSynchronize(e1);
      float m = 0.f;
      cudaEventElapsedTime(&m, e0, e1);
      if (rep > 0 && m < ms) ms = m;
    }
    if (ms < bestMs) { bestMs = ms; *best = cand[i]; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return MDWT_OK;
}

mdwt_status mdwt_denoiser_autotune(mdwt_denoiser *d, const float *F, int n, int h, int w, int backward) {
  if (!d || !F || !dims_ok(n, h, w)) return MDWT_ERR_BAD_ARG;
  if (!d->useTC) return MDWT_OK;
  DCK(cudaSetDevice(d->device), "cudaSetDevice");
  cudaStream_t st = nullptr;
  d->tunedN = 0;
  mdwt_status s = forward(d, F, n, h, w, st);   // activations of this shape
  if (s) return s;
  DCK(cudaStreamSynchronize(st), "sync");
  Acts &A = d->A;
  const int Hp = A.Hp, Wp = A.Wp, H1 = Hp / 2, W1 = Wp / 2, H2 = Hp / 4, W2 = Wp / 4;
  const void *in[kLayers] = {A.x0, A.a1, A.p0, A.a2, A.p1, A.a3, A.u1, A.a4, A.u0, A.a5};
  void *out[kLayers] = {A.a1, A.s0, A.a2, A.s1, A.a3, A.b2, A.a4, A.b1, A.a5, A.o};
  const int hh[kLayers] = {Hp, Hp, H1, H1, H2, H2, H1, H1, Hp, Hp};
  const int ww[kLayers] = {Wp, Wp, W1, W1, W2, W2, W1, W1, Wp, Wp};
  for (int i = 0; i < kLayers; i++) {
    const Layer &l = d->L[i];
    if (!mdwt::nn::conv3x3_tc_supported(l.cin, l.cout)) continue;
    if ((s = tune_one(d, l.cin, l.cout, in[i], l.Wuf, l.b, out[i], n, hh[i], ww[i], l.relu, i == kLayers - 1, &d->tileF[i],
                      st)))
      return s;
  }
  // data gradients: dy -> dx buffers of the backward pass (contents do not matter for timing)
  void *dyb[kLayers] = {nullptr, A.d_s0, A.d_a2, A.d_s1, A.d_a3, A.d_b2, A.d_a4, A.d_b1, A.d_a5, A.d_o};
  void *dxb[kLayers] = {nullptr, A.d_a1, A.d_p0, A.d_a2, A.d_p1, A.d_a3, A.d_u1, A.d_a4, A.d_u0, A.d_a5};
  for (int i = 1; backward && i < kLayers; i++) {
    const Layer &l = d->L[i];
    if (!mdwt::nn::conv3x3_tc_supported(l.cout, l.cin)) continue;
    if ((s = tune_one(d, l.cout, l.cin, dyb[i], l.Wud, nullptr, dxb[i], n, hh[i], ww[i], 0, 0, &d->tileD[i], st)))
      return s;
  }
  d->tunedN = n; d->tunedH = Hp; d->tunedW = Wp;
  return mdwt_denoiser_check(d);
}

mdwt_status mdwt_denoiser_check(mdwt_denoiser *d) {
  if (!d) return MDWT_ERR_BAD_ARG;
  DCK(cudaSetDevice(d->device), "cudaSetDevice");
  DCK(cudaDeviceSynchronize(), "sync");
  int e = 0;
  DCK(cudaMemcpy(&e, d->dErr, sizeof(int), cudaMemcpyDeviceToHost), "error flag");
  if (e) {
    DCK(cudaMemset(d->dErr, 0, sizeof(int)), "error flag");   // reported once
    return fail(d, MDWT_ERR_TIMEOUT, "a tensor-core convolution gave up waiting for its operands");
  }
  return MDWT_OK;
}

mdwt_status mdwt_denoiser_test_stall(mdwt_denoiser *d, int launches) {
  if (!d || launches < 0) return MDWT_ERR_BAD_ARG;
  mdwt::nn::conv3x3_tc_stall_test(launches);
  return MDWT_OK;
}

}  // extern "C"
