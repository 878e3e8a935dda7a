// mdwt_nn_tc.cu -- the denoiser's 3x3 convolution on the 5th-generation tensor cores.
//
// Implicit GEMM per CTA: D[128 pixels of one image row][Cout] = sum over the 9 taps of
// A_tap[128 pixels][Cin] x B_tap[Cin][Cout].  Per tap:
//   * A: the 128 input pixels (y + dy, x0 + dx .. x0 + dx + 127) x Cin channels, one TMA
//     tile load per group of 8 channels (box 8 channels x 128 pixels from the NHWC tensor
//     map; out-of-image pixels -- padding, row ends -- are zero-filled by the TMA unit);
//   * B: the tap's weights, pre-arranged on the device in the operand layout
//     [ci / 8][co][8], one bulk copy.
// Both land in shared memory in the K-major, no-swizzle core-matrix layout (8 rows x 16
// bytes per core matrix; 8-row groups 128 B apart, K groups LBO apart).  One thread
// issues tcgen05.mma (kind::f16, BF16 inputs, FP32 accumulator in tensor memory, M = 128,
// N = Cout, K = 16 per instruction) and tcgen05.commit to an mbarrier; two stages, the
// loads of tap t + 2 wait for the MMAs of tap t.  Epilogue: each warp reads its 32 TMEM
// lanes (= pixels) with tcgen05.ld, adds the bias, applies ReLU and stores BF16 or FP32.
// Every mbarrier wait is bounded; a wait that gives up sets *err and the CTA skips to
// freeing its tensor memory.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "mdwt_nn.h"

namespace mdwt {
namespace nn {
namespace {

typedef __nv_bfloat16 bf16;

constexpr int kTM = 128;                 // pixels per CTA (MMA M)
constexpr uint32_t kSpinLimit = 1u << 22;   // bounded mbarrier waits (with nanosleep back-off)

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes));
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait: false when it gave up
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  for (uint32_t i = 0; i < kSpinLimit; i++) {
    if (mbar_try_wait(bar, parity)) return true;
    if (i > 64) __nanosleep(64);
  }
  return false;
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// K-major, no-swizzle shared-memory matrix descriptor (tcgen05 format: start >> 4 in
// bits 0-13, leading (K-direction) byte offset >> 4 in bits 16-29, stride (M/N-direction)
// byte offset >> 4 in bits 32-45, descriptor version 1 in bits 46-47, layout 0), as its
// low and high 32-bit words.  Shared-memory addresses are below 256 KB, so adding a byte
// offset >> 4 to the low word moves the start within its 14-bit field without a carry.
__device__ __forceinline__ uint32_t smem_desc_lo(uint32_t addr, uint32_t lbo) {
  return ((addr & 0x3FFFFu) >> 4) | (((lbo & 0x3FFFFu) >> 4) << 16);
}
__device__ __forceinline__ uint32_t smem_desc_hi(uint32_t sbo) { return ((sbo & 0x3FFFFu) >> 4) | (1u << 14); }
// Instruction descriptor, kind::f16: D FP32 (bits 4-5 = 1), A and B BF16 (bits 7-9, 10-12
// = 1), both K-major, N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// One MMA; the descriptors are given as low words plus one shared high word (the same
// stride and version for A and B), so the issuing loop only adds offsets.
__device__ __forceinline__ void umma_f16(uint32_t dtmem, uint32_t alo, uint32_t blo, uint32_t hi, uint32_t idesc,
                                         uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t.reg .b64 a, b;\n\t"
      "setp.ne.b32 p, %5, 0;\n\t"
      "mov.b64 a, {%1, %3};\n\t"
      "mov.b64 b, {%2, %3};\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], a, b, %4, p;\n\t}\n" ::"r"(dtmem),
      "r"(alo), "r"(blo), "r"(hi), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}

constexpr int kMaxStages = 9;     // weight ring depth (runtime NS <= kMaxStages; 9 = a whole chunk's taps)
constexpr uint32_t kSlot = 2176;   // smem slot of one A box (8 channels x 130 pixels = 2080 B), 128-B aligned
constexpr int kHalo = kTM + 2;     // input pixels per row segment (one-pixel halo each side)

// CTA: R output rows x 128 pixels, all Cout channels.  Input channels in chunks of KC;
// per chunk the R + 2 input rows (with a one-pixel halo) are loaded once; the horizontal
// taps are the same rows read from a descriptor start 16 B (one pixel) further.
__global__ void __launch_bounds__(128) conv3x3_tc_kernel(const __grid_constant__ CUtensorMap mapX, const bf16 *Wu,
                                                         const float *bias, void *Y, int N, int H, int W, int Cin,
                                                         int Cout, int relu, int outF32, int tmemCols, int R, int KC,
                                                         int NS, int *err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full[kMaxStages], empty[kMaxStages], fullA, freeA, done;
  __shared__ uint32_t tmemBase;
  uint8_t *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tilesX = (W + kTM - 1) / kTM, tilesY = (H + R - 1) / R;
  const int bx = blockIdx.x;
  const int x0 = (bx % tilesX) * kTM;
  const int y0 = ((bx / tilesX) % tilesY) * R;
  const int n = bx / (tilesX * tilesY);
  const int G = KC / 8;                                   // A boxes per row and chunk
  const uint32_t aRowBytes = (uint32_t)G * kSlot;
  const uint32_t aBytes = (uint32_t)(R + 2) * aRowBytes;  // A buffer
  const uint32_t wBytes = (uint32_t)KC * Cout * 2;        // one tap's weights of a chunk
  uint8_t *bufA = smem;
  uint8_t *wBase = smem + aBytes;          // NS weight stages of wBytes each
  const int chunks = Cin / KC, Q = chunks * 9, Gtot = Cin / 8;

  if (tid == 0) {
    for (int i = 0; i < NS; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(&fullA, 1);
    mbar_init(&freeA, 1);
    mbar_init(&done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmemBase)),
                 "r"(tmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n");
  const uint32_t tmem = tmemBase;

  if (tid == 0) {
    bool ok = true;
    const uint32_t idesc = instr_desc(kTM, Cout);
    auto loadA = [&](int kc) {
      mbar_expect_tx(&fullA, (uint32_t)(R + 2) * G * (kHalo * 16));
      for (int r = 0; r < R + 2; r++)
        for (int g = 0; g < G; g++)
          tma_load_4d(bufA + r * aRowBytes + g * kSlot, &mapX, kc * KC + g * 8, x0 - 1, y0 - 1 + r, n, &fullA);
    };
    auto loadW = [&](int q) {
      const int kc = q / 9, tap = q % 9, st = q % NS;
      mbar_expect_tx(&full[st], wBytes);
      bulk_load(wBase + (size_t)st * wBytes, Wu + ((size_t)tap * Gtot + (size_t)kc * G) * Cout * 8, wBytes, &full[st]);
    };
    loadA(0);
    for (int q = 0; q < NS && q < Q; q++) loadW(q);   // fill the weight ring
    const uint32_t lboB = (uint32_t)Cout * 16;
    // descriptor words: start offsets in 16-byte units are added to the low words
    const uint32_t hi = smem_desc_hi(128);
    const uint32_t aLo0 = smem_desc_lo(smem_u32(bufA), kSlot), bLo0 = smem_desc_lo(smem_u32(wBase), lboB);
    const uint32_t aRowStep = aRowBytes >> 4, aKStep = (2 * kSlot) >> 4, bKStep = (2 * lboB) >> 4;
    const uint32_t wStep = wBytes >> 4;
    const int nk = KC / 16;
    for (int q = 0; q < Q && ok; q++) {
      const int kc = q / 9, t = q % 9, st = q % NS;
      const uint32_t ph = (uint32_t)(q / NS) & 1u;
      if (t == 0 && !mbar_wait(&fullA, (uint32_t)kc & 1u)) { ok = false; break; }
      if (!mbar_wait(&full[st], ph)) { ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;\n");
      const int dy = t / 3 - 1, dx = t % 3 - 1;
      const uint32_t bStep = bLo0 + (uint32_t)st * wStep;
      uint32_t aRow = aLo0 + (uint32_t)(dx + 1) + (uint32_t)(dy + 1) * aRowStep;
      uint32_t d = tmem;
      for (int r = 0; r < R; r++, aRow += aRowStep, d += (uint32_t)Cout) {
        uint32_t a = aRow, b = bStep;
        umma_f16(d, a, b, hi, idesc, q > 0 ? 1u : 0u);
        for (int k = 1; k < nk; k++) {
          a += aKStep;
          b += bKStep;
          umma_f16(d, a, b, hi, idesc, 1u);
        }
      }
      umma_commit(&empty[st]);
      if (t == 8) umma_commit(&freeA);
      // refill the stage of step q - 1 (its MMAs were issued before this step's, which
      // are queued behind them) with step q - 1 + NS
      if (q >= 1 && q - 1 + NS < Q) {
        const int sp = (q - 1) % NS;
        if (!mbar_wait(&empty[sp], (uint32_t)((q - 1) / NS) & 1u)) { ok = false; break; }
        loadW(q - 1 + NS);
      }
      if (t == 8 && kc + 1 < chunks) {
        if (!mbar_wait(&freeA, (uint32_t)kc & 1u)) { ok = false; break; }
        loadA(kc + 1);
      }
    }
    if (ok) {
      umma_commit(&done);
      if (!mbar_wait(&done, 0)) ok = false;
    }
    if (!ok) atomicExch(err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n");
  const bool good = *(volatile int *)err == 0;

  if (good) {
    // epilogue: warp w owns TMEM lanes 32w .. 32w + 31 = pixels x0 + 32w + lane
    const int px = x0 + warp * 32 + lane;
    const bool validX = px < W;
    for (int r = 0; r < R; r++) {
      const int y = y0 + r;
      const bool valid = validX && y < H;
      const size_t pix = (((size_t)n * H + (y < H ? y : 0)) * W + (validX ? px : 0));
      for (int c0 = 0; c0 < Cout; c0 += 16) {
        uint32_t v32[16];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(r * Cout + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
            : "=r"(v32[0]), "=r"(v32[1]), "=r"(v32[2]), "=r"(v32[3]), "=r"(v32[4]), "=r"(v32[5]), "=r"(v32[6]),
              "=r"(v32[7]), "=r"(v32[8]), "=r"(v32[9]), "=r"(v32[10]), "=r"(v32[11]), "=r"(v32[12]), "=r"(v32[13]),
              "=r"(v32[14]), "=r"(v32[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        if (!valid) continue;
        float v[16];
#pragma unroll
        for (int j = 0; j < 16; j++) {
          float f = __uint_as_float(v32[j]);
          if (bias) f += bias[c0 + j];
          if (relu) f = fmaxf(f, 0.f);
          v[j] = f;
        }
        if (outF32) {
          float4 *o = reinterpret_cast<float4 *>(reinterpret_cast<float *>(Y) + pix * Cout + c0);
#pragma unroll
          for (int j = 0; j < 4; j++) o[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
        } else {
          uint4 w[2];
          uint32_t *wp = reinterpret_cast<uint32_t *>(w);
#pragma unroll
          for (int j = 0; j < 8; j++) {
            __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
            wp[j] = *reinterpret_cast<uint32_t *>(&b2);
          }
          uint4 *o = reinterpret_cast<uint4 *>(reinterpret_cast<bf16 *>(Y) + pix * Cout + c0);
          o[0] = w[0];
          o[1] = w[1];
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;\n");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(tmemCols));
  }
}

// weights [tap][co][ci] (forward layout) -> operand layout [tap][ci / 8][co][8]
__global__ void umma_weights_kernel(const bf16 *Wf, bf16 *Wu, int Cin, int Cout) {
  const size_t n = (size_t)9 * Cin * Cout;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int ci = (int)(i % Cin);
    const size_t r = i / Cin;
    const int co = (int)(r % Cout);
    const int tap = (int)(r / Cout);
    Wu[(((size_t)tap * (Cin / 8) + ci / 8) * Cout + co) * 8 + (ci & 7)] = Wf[i];
  }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  });
  return fn;
}

int tmem_cols_for(int cols) {
  int c = 32;
  while (c < cols) c <<= 1;
  return c;
}

constexpr size_t kSmemBudget = 200 * 1024;
constexpr size_t kSmemTwoCtas = 112 * 1024;   // two CTAs per SM

size_t tc_smem(int R, int KC, int Cout, int NS) {
  return (size_t)(R + 2) * (KC / 8) * kSlot + (size_t)NS * KC * Cout * 2;
}

int g_tcPolicy = 1;   // 1: two CTAs per SM where possible (measured faster); 0: most rows per CTA

// Rows per CTA R (<= 8), input-channel chunk KC (a divisor of Cin, multiple of 16) and
// weight stages NS (3, else 2) whose buffers fit the shared-memory budget, R * Cout
// TMEM columns.  Policy 1 first looks for a tiling that fits two CTAs per SM (R >= 2,
// R * Cout <= 256, <= 112 KB).
TcTiling tc_tiling(int Cin, int Cout, int H) {
  TcTiling t;
  t.R = 0;
  auto search = [&](size_t budget, int colsMax, int rmin) {
    int rmax = colsMax / Cout;
    if (rmax > 8) rmax = 8;
    if (rmax > H) rmax = H;
    for (int R = rmax; R >= rmin; R--)
      for (int KC = Cin; KC >= 16; KC -= 16) {
        if (Cin % KC) continue;
        for (int NS = 3; NS >= 2; NS--) {
          const size_t sm = tc_smem(R, KC, Cout, NS);
          if (sm <= budget) {
            t.R = R; t.KC = KC; t.NS = NS;
            return true;
          }
        }
      }
    return false;
  };
  if (g_tcPolicy == 1 && search(kSmemTwoCtas, 256, H >= 2 ? 2 : 1)) return t;
  search(kSmemBudget, 512, 1);
  return t;
}

}  // namespace

bool conv3x3_tc_valid(int Cin, int Cout, int H, const TcTiling &t) {
  return t.R >= 1 && t.R <= 8 && t.R * Cout <= 512 && t.R <= (H > 0 ? H : 1) && t.KC >= 16 && t.KC % 16 == 0 &&
         Cin % t.KC == 0 && t.NS >= 2 && t.NS <= kMaxStages && tc_smem(t.R, t.KC, Cout, t.NS) <= kSmemBudget;
}

// Candidate tilings for the autotuner: for each rows-per-CTA R, the largest channel chunk
// that fits with a 3-stage ring, and with a ring of all of the chunk's 9 taps.
int conv3x3_tc_candidates(int Cin, int Cout, int H, TcTiling *out, int maxOut) {
  int n = 0;
  for (int R = 1; R <= 8 && n < maxOut; R++) {
    if (R * Cout > 512 || R > H) break;
    for (int NS : {3, 9}) {
      for (int KC = Cin; KC >= 16; KC -= 16) {
        if (Cin % KC) continue;
        TcTiling t;
        t.R = R; t.KC = KC; t.NS = NS;
        if (tc_smem(R, KC, Cout, NS) <= kSmemBudget) {
          bool dup = false;
          for (int i = 0; i < n; i++) dup = dup || (out[i].R == R && out[i].KC == KC && out[i].NS == NS);
          if (!dup && n < maxOut) out[n++] = t;
          break;
        }
      }
    }
  }
  return n;
}

bool conv3x3_tc_supported(int Cin, int Cout) {
  return Cin % 16 == 0 && Cin >= 16 && Cout % 16 == 0 && Cout >= 16 && Cout <= 256 && tc_tiling(Cin, Cout, 1).R > 0 &&
         encode_fn() != nullptr;
}

void conv3x3_tc_policy(int policy) { g_tcPolicy = policy == 1 ? 1 : 0; }

int umma_weights(const void *Wf, void *Wu, int Cin, int Cout, int numSMs, void *stream) {
  const size_t n = (size_t)9 * Cin * Cout;
  size_t g = (n + 255) / 256;
  if (g > (size_t)numSMs * 16) g = (size_t)numSMs * 16;
  umma_weights_kernel<<<(unsigned)g, 256, 0, (cudaStream_t)stream>>>((const bf16 *)Wf, (bf16 *)Wu, Cin, Cout);
  return (int)cudaGetLastError();
}

int conv3x3_tc(const void *X, const void *Wu, const float *bias, void *Y, int N, int H, int W, int Cin, int Cout,
               int relu, int outF32, int *err, void *stream, const TcTiling *tiling) {
  if (!conv3x3_tc_supported(Cin, Cout) || N <= 0 || H <= 0 || W <= 0) return (int)cudaErrorInvalidValue;
  if ((reinterpret_cast<uintptr_t>(X) & 15) || (reinterpret_cast<uintptr_t>(Wu) & 15)) return (int)cudaErrorInvalidValue;
  TcTiling tl = tc_tiling(Cin, Cout, H);
  if (tiling && tiling->R > 0) {
    if (!conv3x3_tc_valid(Cin, Cout, H, *tiling)) return (int)cudaErrorInvalidValue;
    tl = *tiling;
  }
  if (tl.R == 0) return (int)cudaErrorInvalidValue;
  CUtensorMap map;
  const cuuint64_t dims[4] = {(cuuint64_t)Cin, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
  const cuuint64_t strides[3] = {(cuuint64_t)Cin * 2, (cuuint64_t)W * Cin * 2, (cuuint64_t)H * W * Cin * 2};
  const cuuint32_t box[4] = {8, (cuuint32_t)kHalo, 1, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  const CUresult cr = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(X), dims, strides, box,
                                  es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (cr != CUDA_SUCCESS) return (int)cudaErrorInvalidValue;
  const size_t smem = tc_smem(tl.R, tl.KC, Cout, tl.NS) + 1024;
  cudaError_t e = cudaFuncSetAttribute(conv3x3_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(kSmemBudget + 1024));
  if (e != cudaSuccess) return (int)e;
  const int tilesX = (W + kTM - 1) / kTM, tilesY = (H + tl.R - 1) / tl.R;
  conv3x3_tc_kernel<<<(unsigned)(N * tilesY * tilesX), 128, smem, (cudaStream_t)stream>>>(
      map, (const bf16 *)Wu, bias, Y, N, H, W, Cin, Cout, relu, outF32, tmem_cols_for(tl.R * Cout), tl.R, tl.KC, tl.NS,
      err);
  return (int)cudaGetLastError();
}

}  // namespace nn
}  // namespace mdwt
