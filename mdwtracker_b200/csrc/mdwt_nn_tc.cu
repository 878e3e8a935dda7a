// mdwt_nn_tc.cu -- the denoiser's 3x3 convolution on the 5th-generation tensor cores.
//
// Implicit GEMM: D[128 pixels of one image row][Cout] = sum over the 9 taps of
// A_tap[128 pixels][Cin] x B_tap[Cin][Cout].
//   * A: the input rows y - 1 .. y + R of a tile, pixels x0 - 1 .. x0 + 128, one TMA load
//     per group of 8 channels (a box of 8 channels x 130 pixels x R + 2 rows of the NHWC
//     tensor map; out-of-image pixels -- padding, row ends -- are zero-filled by the TMA
//     unit); tap (dy, dx) of output row r reads input row r + dy from pixel dx on;
//   * B: the weights, pre-arranged on the device in the operand layout
//     [dx][ci / 8][dy][co][8] and bulk-copied (once per launch when they fit, else per
//     tile and chunk).
// Both sit in shared memory in the K-major, no-swizzle core-matrix layout (8 rows x 16
// bytes per core matrix; 8-row groups 128 B apart, K groups LBO apart).  tcgen05.mma
// kind::f16: BF16 inputs, FP32 accumulator in tensor memory, M = 128 pixels, K = 16, N =
// Cout (or 3 Cout with the vertical taps stacked).  The kernel is persistent and
// warp-specialised (producers, MMA issuer, epilogue warps; see conv3x3_tc_kernel); its
// epilogue can also write the pooled output or the denoiser's residual output.  Every
// mbarrier wait is bounded; a wait that gives up sets *err.
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
constexpr long long kWaitClocks = 1ll << 31;   // bounded mbarrier waits: give up after ~1 s of SM clocks

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
// bounded wait: false when it gave up (after kWaitClocks SM clocks)
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const long long t0 = clock64();
  for (uint32_t i = 0;; i++) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 15u) == 15u && clock64() - t0 > kWaitClocks) return false;
    if (i > 64) __nanosleep(64);
  }
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

// One MMA, issued by one elected lane of a converged warp (all lanes call it); the
// descriptors are given as low words plus one shared high word (the same stride and
// version for A and B), so the issuing loop only adds offsets.
__device__ __forceinline__ void umma_f16(uint32_t dtmem, uint32_t alo, uint32_t blo, uint32_t hi, uint32_t idesc,
                                         uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p, e;\n\t.reg .b64 a, b;\n\t"
      "elect.sync _|e, 0xffffffff;\n\t"
      "setp.ne.b32 p, %5, 0;\n\t"
      "mov.b64 a, {%1, %3};\n\t"
      "mov.b64 b, {%2, %3};\n\t"
      "@e tcgen05.mma.cta_group::1.kind::f16 [%0], a, b, %4, p;\n\t}\n" ::"r"(dtmem),
      "r"(alo), "r"(blo), "r"(hi), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}

// load 16 columns of this warp's 32 TMEM lanes (complete after tcgen05.wait::ld)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}
// store 16 zero columns of this warp's 32 TMEM lanes
__device__ __forceinline__ void tmem_zero16(uint32_t taddr) {
  const uint32_t z = 0;
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};\n" ::"r"(taddr),
      "r"(z)
      : "memory");
}

constexpr int kMaxAStages = 4;            // input (A) ring depth
constexpr int kMaxWStages = 16;           // weight stages (one input-channel chunk x 9 taps each)
constexpr int kEpiWarps = 8;              // epilogue warps (two per TMEM lane quarter)
constexpr int kWarpA = 0;                 // input producer (TMA)
constexpr int kWarpW = 1;                 // weight producer and TMEM allocator
constexpr int kWarpMma = 2;               // MMA issuer
constexpr int kWarpEpi = 3;               // first epilogue warp
constexpr int kThreads = 32 * (3 + kEpiWarps);
constexpr int kHalo = kTM + 2;            // input pixels per row segment (one-pixel halo each side)
constexpr uint32_t kRowBytes = kHalo * 16;   // one row segment of 8 channels: 2080 B

// Shared-memory slot of one channel group of a stage (R + 2 rows x 130 pixels x 8
// channels), 128-B aligned.
__host__ __device__ inline uint32_t a_slot(int R) { return ((uint32_t)(R + 2) * kRowBytes + 127u) & ~127u; }

struct ConvArgs {
  const bf16 *Wu;
  const float *bias;
  void *Y;
  int *err;
  int N, H, W, Cin, Cout, relu, outF32;
  int R, KC, NS, SA, AB, ST, resident, tmemCols, tilesX, tilesY, tiles;
  int stallTest;       // test hook: the input producer issues nothing (every wait then gives up)
  int pdl;             // launched as a programmatic dependent of the previous kernel
  int C1;              // input channels [0, C1) from mapX, [C1, Cin) from mapX2 (C1 = Cin: one tensor)
  const float *resF;   // residual output (TcResidual) when resOut != nullptr
  void *poolOut;       // fused 2x2 average pooling of Y (BF16) when non-null
  float *resOut;
  int resH, resW;
};

// bounded wait that also gives up once another role of the CTA has aborted
__device__ __forceinline__ bool mbar_wait_ab(uint64_t *bar, uint32_t parity, volatile int *abortFlag) {
  const long long t0 = clock64();
  for (uint32_t i = 0;; i++) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 15u) == 15u && (*abortFlag || clock64() - t0 > kWaitClocks)) return false;
    if (i > 64) __nanosleep(32);
  }
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// Persistent, warp-specialised implicit-GEMM convolution.  A tile is R output rows x 128
// pixels of one image, all Cout channels; CTA b takes tiles b, b + grid, ...  Per tile and
// input-channel chunk (KC channels) the R + 2 input rows with a one-pixel halo are staged
// once; the horizontal taps read the same rows from a descriptor start one pixel (16 B)
// further, the vertical taps from the neighbouring rows.
//   warp 0, lane 0: input producer -- per tile and chunk one TMA load per 8-channel group
//     (a box of 8 channels x 130 pixels x R + 2 rows of the NHWC tensor map, zero-filled
//     outside the image; channels from C1 on from a second tensor when the input is the
//     concatenation of two) into a ring of SA stages;
//   warp 1, lane 0: weights -- by bulk copies into stages of one input-channel chunk x 9
//     taps, once for the whole launch (resident) or per tile and chunk through a ring of
//     NS stages;
//   warp 2: MMA issuer -- the warp runs the loops, one elected lane issues tcgen05.mma
//     (M = 128 pixels, K = 16): stacked (ST, Cout <= 85), one MMA per staged input row,
//     horizontal tap and K step covers the three vertical taps (N = 3 Cout, the three
//     output rows' accumulators being adjacent in TMEM), else one MMA per tap (N = Cout); AB
//     accumulators of R x Cout TMEM columns alternate between tiles, so the epilogue of
//     one tile overlaps the MMAs of the next;
//   warps 3-10: epilogue -- tcgen05.ld of their lane quarter (32 pixels), bias, ReLU,
//     BF16 or FP32 stores (or the fused residual output; or also the fused 2x2 average
//     pooling, rows then taken in pairs), then zero the columns read (the MMAs only
//     accumulate); the two warps of a quarter take alternate rows.
// Every wait is bounded; a role that gives up sets *err and the CTA abort flag, the others
// leave their loops, the producers wait for their copies in flight and the MMA issuer for
// its MMAs before the tensor memory is freed.
__global__ void __launch_bounds__(kThreads, 1) conv3x3_tc_kernel(const __grid_constant__ CUtensorMap mapX,
                                                                  const __grid_constant__ CUtensorMap mapX2,
                                                                  const ConvArgs a) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t aFull[kMaxAStages], aEmpty[kMaxAStages], wFull[kMaxWStages], wEmpty[kMaxWStages];
  __shared__ __align__(8) uint64_t wRes, accFull[2], accEmpty[2], mmaDone;
  __shared__ uint32_t tmemBase;
  __shared__ volatile int abortFlag;
  __shared__ float sBias[256];   // the epilogue's bias (Cout <= 256), loaded once
  const bool hasBias = a.bias != nullptr;
  uint8_t *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int R = a.R, Cout = a.Cout, G = a.KC / 8, chunks = a.Cin / a.KC, Gtot = a.Cin / 8;
  const uint32_t slot = a_slot(R), stageA = (uint32_t)G * slot;
  const uint32_t tapChunkBytes = (uint32_t)G * Cout * 16;   // one tap's weights of a chunk
  const uint32_t wStageBytes = 9 * tapChunkBytes;
  const int wStages = a.resident ? chunks : a.NS;
  uint8_t *bufA = smem;
  uint8_t *bufW = smem + (size_t)a.SA * stageA;

  if (threadIdx.x == 0) {
    for (int i = 0; i < a.SA; i++) {
      mbar_init(&aFull[i], 1);
      mbar_init(&aEmpty[i], 1);
    }
    for (int i = 0; i < kMaxWStages; i++) {
      mbar_init(&wFull[i], 1);
      mbar_init(&wEmpty[i], 1);
    }
    mbar_init(&wRes, 1);
    for (int i = 0; i < 2; i++) {
      mbar_init(&accFull[i], 1);
      mbar_init(&accEmpty[i], kEpiWarps);
    }
    mbar_init(&mmaDone, 1);
    abortFlag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (hasBias)   // weights and biases are not written by the kernel this one may overlap
    for (int i = threadIdx.x; i < a.Cout; i += blockDim.x) sBias[i] = a.bias[i];
  if (warp == kWarpW) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmemBase)),
                 "r"(a.tmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n");
  const uint32_t tmem = tmemBase;
  // programmatic dependent launch: the next kernel's CTAs may be scheduled as SMs free up
  // (their set-up overlaps this kernel's tail); only the reads of the previous kernel's
  // output wait for it (griddepcontrol.wait in the input producer)
  if (a.pdl) asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  auto fail = [&]() {
    abortFlag = 1;
    atomicExch(a.err, 1);
  };

  if (warp == kWarpA) {
    if (lane == 0) {
      // ---------------------------------------------------------------- input producer
      // per tile and chunk, one TMA load per 8-channel group: a box of 8 channels x 130
      // pixels x R + 2 rows (zero-filled outside the image) into the group's slot
      bool ok = true;
      uint32_t gA = 0;
      if (a.pdl) asm volatile("griddepcontrol.wait;\n" ::: "memory");   // the input is complete
      for (int t = blockIdx.x; t < a.tiles && ok && !a.stallTest; t += gridDim.x) {
        if (abortFlag) break;
        const int tx = t % a.tilesX, ty = (t / a.tilesX) % a.tilesY, n = t / (a.tilesX * a.tilesY);
        const int x0 = tx * kTM, y0 = ty * R;
        for (int kc = 0; kc < chunks; kc++) {
          const uint32_t s = gA % (uint32_t)a.SA, use = gA / (uint32_t)a.SA;
          if (use > 0 && !mbar_wait_ab(&aEmpty[s], (use - 1) & 1u, &abortFlag)) { ok = false; break; }
          mbar_expect_tx(&aFull[s], (uint32_t)G * (R + 2) * kRowBytes);
          for (int g = 0; g < G; g++)
          {
            const int c = kc * a.KC + g * 8;   // the first tensor's channels, then the second's
            if (c < a.C1) tma_load_4d(bufA + s * stageA + g * slot, &mapX, c, x0 - 1, y0 - 1, n, &aFull[s]);
            else tma_load_4d(bufA + s * stageA + g * slot, &mapX2, c - a.C1, x0 - 1, y0 - 1, n, &aFull[s]);
          }
          gA++;
        }
      }
      if (!ok) fail();
      // wait for every load issued (the last one into each stage may still be in flight)
      for (uint32_t st = 0; st < (uint32_t)a.SA; st++)
        if (gA > st && !mbar_wait(&aFull[st], ((gA - 1 - st) / (uint32_t)a.SA) & 1u)) fail();
    }
    __syncwarp();
  } else if (warp == kWarpW) {
    if (lane == 0) {
      // ---------------------------------------------------------------- weights
      // stage = one input-channel chunk, all 9 taps: [dx][G][dy][Cout][8]; resident weights
      // fill one stage per chunk once, streamed weights cycle NS stages per tile and chunk
      bool ok = true;
      uint32_t gW = 0;
      auto loadChunk = [&](uint32_t st, int kc) {
        mbar_expect_tx(&wFull[st], wStageBytes);
        for (int dx = 0; dx < 3; dx++)
          bulk_load(bufW + (size_t)st * wStageBytes + (size_t)dx * 3 * tapChunkBytes,
                    a.Wu + ((size_t)dx * Gtot + (size_t)kc * G) * 3 * Cout * 8, 3 * tapChunkBytes, &wFull[st]);
      };
      if (a.resident) {
        for (int kc = 0; kc < chunks; kc++) loadChunk((uint32_t)kc, kc);
        gW = (uint32_t)chunks;
      } else {
        for (int t = blockIdx.x; t < a.tiles && ok; t += gridDim.x) {
          if (abortFlag) break;
          for (int kc = 0; kc < chunks; kc++) {
            const uint32_t sw = gW % (uint32_t)wStages, uw = gW / (uint32_t)wStages;
            if (uw > 0 && !mbar_wait_ab(&wEmpty[sw], (uw - 1) & 1u, &abortFlag)) { ok = false; break; }
            loadChunk(sw, kc);
            gW++;
          }
        }
      }
      if (!ok) fail();
      // wait for every copy issued (the last one into each stage may still be in flight)
      for (uint32_t st = 0; st < (uint32_t)wStages; st++)
        if (gW > st && !mbar_wait(&wFull[st], ((gW - 1 - st) / (uint32_t)wStages) & 1u)) fail();
    }
    __syncwarp();
  } else if (warp == kWarpMma) {
    // ------------------------------------------------------------------ MMA issuer
    // The whole warp runs the (uniform) loops; one elected lane issues.  Per chunk and
    // output row the KC / 16 x 9 taps MMAs go to that row's accumulator back to back.
    auto warpWait = [&](uint64_t *bar, uint32_t parity) -> bool {
      int okw = 0;
      if (lane == 0) okw = mbar_wait_ab(bar, parity, &abortFlag) ? 1 : 0;
      return __shfl_sync(0xffffffffu, okw, 0) != 0;
    };
    bool ok = true;
    // Accumulator of output row r: TMEM columns c(r) = (R - 1 - r) Cout of the tile's buffer
    // (descending), zeroed by the epilogue; every MMA accumulates.  Stacked (3 Cout <= 256):
    // staged input row j, horizontal tap dx and K step k feed output rows j - dy for the
    // valid vertical taps dy in [d0, d1] with ONE MMA: B = the weights of (dx, dy = d0..d1)
    // (contiguous rows), N = (d1 - d0 + 1) Cout, D at c(j - d0).  Otherwise one MMA per
    // tap (N = Cout) into c(r).
    const bool stacked = a.ST != 0;
    const uint32_t idesc1 = instr_desc(kTM, Cout), idesc2 = stacked ? instr_desc(kTM, 2 * Cout) : 0u,
                   idesc3 = stacked ? instr_desc(kTM, 3 * Cout) : 0u;
    const uint32_t hi = smem_desc_hi(128);
    // descriptor low words; offsets in 16-byte units are added to them
    const uint32_t aLo0 = smem_desc_lo(smem_u32(bufA), slot);
    const uint32_t bLo0 = smem_desc_lo(smem_u32(bufW), (uint32_t)Cout * 48);   // K groups of [dy][Cout][8]
    const uint32_t rowStep = kRowBytes >> 4, aKStep = (2 * slot) >> 4, bKStep = 6u * Cout;
    const uint32_t stageAU = stageA >> 4, wStageU = wStageBytes >> 4, dxU = (3 * tapChunkBytes) >> 4;
    const uint32_t dyU = (uint32_t)Cout;   // one vertical tap's Cout rows, 16-byte units
    const int nk = a.KC / 16;
    uint32_t gA = 0, gW = 0;
    int it = 0;
    for (int t = blockIdx.x; t < a.tiles && ok; t += gridDim.x, it++) {
      const uint32_t ab = (uint32_t)(it % a.AB), use = (uint32_t)(it / a.AB);
      // the epilogue has read and zeroed this accumulator (phase 0: the initial zeroing)
      if (!warpWait(&accEmpty[ab], use & 1u)) { ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;\n");
      const uint32_t dBase = tmem + ab * (uint32_t)(R * Cout);
      for (int kc = 0; kc < chunks; kc++) {
        const uint32_t s = gA % (uint32_t)a.SA;
        const uint32_t sw = a.resident ? (uint32_t)kc : gW % (uint32_t)wStages;
        const uint32_t pw = a.resident ? 0u : (gW / (uint32_t)wStages) & 1u;
        if (!warpWait(&aFull[s], (gA / (uint32_t)a.SA) & 1u) || !warpWait(&wFull[sw], pw)) { ok = false; break; }
        asm volatile("tcgen05.fence::after_thread_sync;\n");
        const uint32_t aSt = aLo0 + s * stageAU, wSt = bLo0 + sw * wStageU;
        if (stacked) {
          for (int j = 0; j < R + 2; j++) {
            const int d0 = j - R + 1 > 0 ? j - R + 1 : 0, d1 = j < 2 ? j : 2;
            const uint32_t id = d1 == d0 ? idesc1 : (d1 - d0 == 1 ? idesc2 : idesc3);
            const uint32_t d = dBase + (uint32_t)((R - 1 - (j - d0)) * Cout);
            uint32_t aK = aSt + (uint32_t)j * rowStep, bK = wSt + (uint32_t)d0 * dyU;
            for (int k = 0; k < nk; k++, aK += aKStep, bK += bKStep) {
#pragma unroll
              for (int dx = 0; dx < 3; dx++) umma_f16(d, aK + (uint32_t)dx, bK + (uint32_t)dx * dxU, hi, id, 1u);
            }
          }
        } else {
          uint32_t d = dBase + (uint32_t)((R - 1) * Cout), aRow = aSt;
          for (int r = 0; r < R; r++, d -= (uint32_t)Cout, aRow += rowStep) {
            uint32_t aK = aRow, bK = wSt;
            for (int k = 0; k < nk; k++, aK += aKStep, bK += bKStep) {
#pragma unroll
              for (int tap = 0; tap < 9; tap++)
                umma_f16(d, aK + (uint32_t)(tap / 3) * rowStep + (uint32_t)(tap % 3),
                         bK + (uint32_t)(tap % 3) * dxU + (uint32_t)(tap / 3) * dyU, hi, idesc1, 1u);
            }
          }
        }
        if (lane == 0) {
          umma_commit(&aEmpty[s]);
          if (!a.resident) umma_commit(&wEmpty[sw]);
        }
        __syncwarp();
        gA++;
        if (!a.resident) gW++;
      }
      if (!ok) break;
      if (lane == 0) umma_commit(&accFull[ab]);
      __syncwarp();
    }
    if (lane == 0) {
      if (!ok) fail();
      umma_commit(&mmaDone);   // all MMAs issued by this warp have completed
      if (!mbar_wait(&mmaDone, 0)) fail();
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------------ epilogue
    const int qd = warp & 3, half = (warp - kWarpEpi) >> 2;
    bool ok = true;
    int it = 0;
    // zero this warp's rows of every accumulator buffer once, then hand them to the MMA warp
    for (int ab = 0; ab < a.AB; ab++) {
      const uint32_t zBase = tmem + ((uint32_t)(qd * 32) << 16) + (uint32_t)(ab * R * Cout);
      for (int r = half; r < R; r += 2)
        for (int c0 = 0; c0 < Cout; c0 += 16) tmem_zero16(zBase + (uint32_t)(r * Cout + c0));
      asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;\n");
      __syncwarp();
      if (lane == 0) mbar_arrive(&accEmpty[ab]);
    }
    for (int t = blockIdx.x; t < a.tiles; t += gridDim.x, it++) {
      int go = 1;
      const uint32_t ab = (uint32_t)(it % a.AB), use = (uint32_t)(it / a.AB);
      if (lane == 0) go = abortFlag ? 0 : (mbar_wait_ab(&accFull[ab], use & 1u, &abortFlag) ? 1 : 2);
      go = __shfl_sync(0xffffffffu, go, 0);
      if (go != 1) {
        ok = go == 0;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;\n");
      const int tx = t % a.tilesX, ty = (t / a.tilesX) % a.tilesY, n = t / (a.tilesX * a.tilesY);
      const int px = tx * kTM + qd * 32 + lane;
      const bool validX = px < a.W;
      const uint32_t tBase = tmem + ((uint32_t)(qd * 32) << 16) + ab * (uint32_t)(R * Cout);
      if (a.poolOut) {
        // fused 2x2 average pooling (R even, H and W even): rows in pairs (2p, 2p + 1), pair p
        // to warp half p % 2; lanes l and l ^ 1 hold horizontal neighbours.  The pooled value
        // is formed from the BF16-rounded outputs in the order of the separate pooling kernel.
        const int Hq = a.H / 2, Wq = a.W / 2;
        for (int pr = half; pr < R / 2; pr += 2) {
          const int y = ty * R + 2 * pr;
          const bool validP = validX && y < a.H;
          for (int c0 = 0; c0 < Cout; c0 += 16) {
            float v[2][16];
            uint32_t vb[2][16];   // the pair's two rows, loaded together
#pragma unroll
            for (int h2 = 0; h2 < 2; h2++) tmem_ld16(tBase + (uint32_t)((R - 1 - (2 * pr + h2)) * Cout + c0), vb[h2]);
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
            for (int h2 = 0; h2 < 2; h2++)   // ready for the next tile
              tmem_zero16(tBase + (uint32_t)((R - 1 - (2 * pr + h2)) * Cout + c0));
#pragma unroll
            for (int h2 = 0; h2 < 2; h2++) {
              const uint32_t *v32 = vb[h2];
              uint4 w[2];
              uint32_t *wp = reinterpret_cast<uint32_t *>(w);
#pragma unroll
              for (int j = 0; j < 8; j++) {
                float f0 = __uint_as_float(v32[2 * j]), f1 = __uint_as_float(v32[2 * j + 1]);
                if (hasBias) { f0 += sBias[c0 + 2 * j]; f1 += sBias[c0 + 2 * j + 1]; }
                if (a.relu) { f0 = fmaxf(f0, 0.f); f1 = fmaxf(f1, 0.f); }
                __nv_bfloat162 b2 = __floats2bfloat162_rn(f0, f1);
                wp[j] = *reinterpret_cast<uint32_t *>(&b2);
                v[h2][2 * j] = __low2float(b2);
                v[h2][2 * j + 1] = __high2float(b2);
              }
              if (validP) {   // rows y and y + 1 are both inside (H even)
                uint4 *o = reinterpret_cast<uint4 *>(reinterpret_cast<bf16 *>(a.Y) +
                                                     (((size_t)n * a.H + y + h2) * a.W + px) * Cout + c0);
                o[0] = w[0];
                o[1] = w[1];
              }
            }
            float q[16];
#pragma unroll
            for (int j = 0; j < 16; j++) {
              const float x01 = __shfl_xor_sync(0xffffffffu, v[0][j], 1);
              const float x11 = __shfl_xor_sync(0xffffffffu, v[1][j], 1);
              float acc = v[0][j] + x01;
              acc += v[1][j];
              q[j] = 0.25f * (acc + x11);
            }
            if (validP && (lane & 1) == 0) {
              uint4 w[2];
              uint32_t *wp = reinterpret_cast<uint32_t *>(w);
#pragma unroll
              for (int j = 0; j < 8; j++) {
                __nv_bfloat162 b2 = __floats2bfloat162_rn(q[2 * j], q[2 * j + 1]);
                wp[j] = *reinterpret_cast<uint32_t *>(&b2);
              }
              uint4 *o = reinterpret_cast<uint4 *>(reinterpret_cast<bf16 *>(a.poolOut) +
                                                   (((size_t)n * Hq + y / 2) * Wq + px / 2) * Cout + c0);
              o[0] = w[0];
              o[1] = w[1];
            }
          }
        }
      }
      for (int r = half; r < R && !a.poolOut; r += 2) {
        const int y = ty * R + r;
        const bool valid = validX && y < a.H;
        const size_t pix = (((size_t)n * a.H + (y < a.H ? y : 0)) * a.W + (validX ? px : 0));
        // up to 64 columns per tensor-memory wait: the loads of a batch are in flight together
        for (int cb = 0; cb < Cout; cb += 64) {
        uint32_t vb[4][16];
#pragma unroll
        for (int q = 0; q < 4; q++)
          if (cb + 16 * q < Cout) tmem_ld16(tBase + (uint32_t)((R - 1 - r) * Cout + cb + 16 * q), vb[q]);
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
        for (int q = 0; q < 4; q++)
          if (cb + 16 * q < Cout) tmem_zero16(tBase + (uint32_t)((R - 1 - r) * Cout + cb + 16 * q));   // for the next tile
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int c0 = cb + 16 * q;
          if (c0 >= Cout) break;
          const uint32_t *v32 = vb[q];
          if (a.resOut) {   // fused residual output: channels 0..2 of the real image only
            if (c0 == 0 && y < a.resH && px < a.resW) {
              const size_t q = ((size_t)n * a.resH + y) * a.resW + px;
              float o[3];
#pragma unroll
              for (int j = 0; j < 3; j++) {
                float f = __uint_as_float(v32[j]);
                if (hasBias) f += sBias[j];
                if (a.relu) f = fmaxf(f, 0.f);
                o[j] = a.resF[q * 16 + j] + f;
              }
              reinterpret_cast<float4 *>(a.resOut)[q] = make_float4(o[0], o[1], o[2], 1.f);
            }
            continue;
          }
          if (!valid) continue;
          float v[16];
#pragma unroll
          for (int j = 0; j < 16; j++) {
            float f = __uint_as_float(v32[j]);
            if (hasBias) f += sBias[c0 + j];
            if (a.relu) f = fmaxf(f, 0.f);
            v[j] = f;
          }
          if (a.outF32) {
            float4 *o = reinterpret_cast<float4 *>(reinterpret_cast<float *>(a.Y) + pix * Cout + c0);
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
            uint4 *o = reinterpret_cast<uint4 *>(reinterpret_cast<bf16 *>(a.Y) + pix * Cout + c0);
            o[0] = w[0];
            o[1] = w[1];
          }
        }
        }
      }
      asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;\n");
      __syncwarp();
      if (lane == 0) mbar_arrive(&accEmpty[ab]);
    }
    if (!ok && lane == 0) fail();
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  if (warp == kWarpW) {
    asm volatile("tcgen05.fence::after_thread_sync;\n");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(a.tmemCols));
  }
}

// ------------------------------------------------------------------ weight gradient
// dW[tap][co][ci] += sum over pixels p of dY[p][co] X[p + tap][ci] (tap = 3 dy + dx) on the
// tensor cores: per input-channel chunk g of KN channels, a GEMM D_tap[co][ci] with M = 128
// output channels (rows beyond Cout are discarded), N = KN, K = pixels, accumulated in
// tensor memory over the CTA's tiles for all nine taps at once (9 KN <= 432 columns).
//   A = dY of one image row segment (128 pixels), B = X of the three rows y - 1 .. y + 1
//   with a one-pixel halo; both are NHWC in global memory, so the TMA boxes (8 channels x
//   pixels) land as MN-major core matrices (8 pixels x 8 channels, 128 contiguous bytes):
//   the K (pixel) direction steps 128 B, the M / N (channel group) direction a group.
//   Tap (dy, dx) of output pixel p reads staged row dy, pixel p + dx.
//   CTA b takes chunk b mod NG and the row segments of its slice; the epilogue adds its
//   nine accumulators into dW with atomics.
constexpr int kWgEpiWarps = 4;
constexpr int kWgThreads = 32 * (2 + kWgEpiWarps);   // producer, MMA issuer, epilogue
constexpr uint32_t kWgDyGroup = kTM * 16;            // 8 channels of a 128-pixel row segment: 2048 B
constexpr uint32_t kWgXBox = 3 * kRowBytes;          // 8 channels of three 130-pixel rows: 6240 B
constexpr uint32_t kWgXGroup = (kWgXBox + 127u) & ~127u;   // its slot: TMA destinations are 128-byte aligned
constexpr int kWgMaxStages = 4;

struct WgradArgs {
  float *dW;
  int *err;
  int N, H, W, Cin, Cout, KN, NG, SA, tilesX, tiles;
};

// one stage: 16 dY channel groups (M = 128; those at and beyond Cout stay zero) and the
// chunk's KN / 8 X channel groups, every group 128-byte aligned
__host__ __device__ inline uint32_t wg_stage_bytes(int KN) {
  return 16u * kWgDyGroup + (uint32_t)(KN / 8) * kWgXGroup;
}

// One MMA with its own high descriptor word for each operand (their strides differ).
__device__ __forceinline__ void umma_f16_ab(uint32_t dtmem, uint32_t alo, uint32_t ahi, uint32_t blo, uint32_t bhi,
                                            uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p, e;\n\t.reg .b64 a, b;\n\t"
      "elect.sync _|e, 0xffffffff;\n\t"
      "setp.ne.b32 p, %6, 0;\n\t"
      "mov.b64 a, {%1, %2};\n\t"
      "mov.b64 b, {%3, %4};\n\t"
      "@e tcgen05.mma.cta_group::1.kind::f16 [%0], a, b, %5, p;\n\t}\n" ::"r"(dtmem),
      "r"(alo), "r"(ahi), "r"(blo), "r"(bhi), "r"(idesc), "r"(acc));
}

__global__ void __launch_bounds__(kWgThreads, 1) conv3x3_wgrad_tc_kernel(const __grid_constant__ CUtensorMap mapDY,
                                                                         const __grid_constant__ CUtensorMap mapX,
                                                                         const WgradArgs a) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full[kWgMaxStages], empty[kWgMaxStages], done;
  __shared__ uint32_t tmemBase;
  __shared__ volatile int abortFlag;
  uint8_t *smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = (int)blockIdx.x % a.NG, slice = (int)blockIdx.x / a.NG, slices = (int)gridDim.x / a.NG;
  const uint32_t stB = wg_stage_bytes(a.KN);
  const int gDy = a.Cout / 8, gX = a.KN / 8;
  // the dY groups the TMA never writes (channels >= Cout) are zero in every stage
  for (int st = 0; st < a.SA; st++)
    for (uint32_t i = (uint32_t)gDy * kWgDyGroup / 16u + threadIdx.x; i < 16u * kWgDyGroup / 16u; i += kWgThreads)
      reinterpret_cast<uint4 *>(smem + (size_t)st * stB)[i] = make_uint4(0u, 0u, 0u, 0u);
  if (threadIdx.x == 0) {
    for (int i = 0; i < a.SA; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], 1);
    }
    mbar_init(&done, 1);
    abortFlag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmemBase)),
                 "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");   // the zeroed groups, for the tensor cores
  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n");
  const uint32_t tmem = tmemBase;
  auto fail = [&]() {
    abortFlag = 1;
    atomicExch(a.err, 1);
  };

  if (warp == 0) {
    if (lane == 0) {
      // ---------------------------------------------------------------- producer
      bool ok = true;
      uint32_t it = 0;
      for (int t = slice; t < a.tiles && ok; t += slices, it++) {
        if (abortFlag) break;
        const uint32_t s = it % (uint32_t)a.SA, use = it / (uint32_t)a.SA;
        if (use > 0 && !mbar_wait_ab(&empty[s], (use - 1) & 1u, &abortFlag)) { ok = false; break; }
        const int tx = t % a.tilesX, y = (t / a.tilesX) % a.H, n = t / (a.tilesX * a.H);
        const int x0 = tx * kTM;
        uint8_t *st = smem + (size_t)s * stB;
        if ((smem_u32(st) & 127u) != 0u) { ok = false; break; }   // every slot below is then 128-byte aligned
        mbar_expect_tx(&full[s], (uint32_t)gDy * kWgDyGroup + (uint32_t)gX * kWgXBox);
        for (int q = 0; q < gDy; q++) tma_load_4d(st + q * kWgDyGroup, &mapDY, 8 * q, x0, y, n, &full[s]);
        for (int h = 0; h < gX; h++)
          tma_load_4d(st + 16 * kWgDyGroup + h * kWgXGroup, &mapX, g * a.KN + 8 * h, x0 - 1, y - 1, n, &full[s]);
      }
      if (!ok) fail();
      // wait for every load issued (the last one into each stage may still be in flight)
      for (uint32_t st = 0; st < (uint32_t)a.SA; st++)
        if (it > st && !mbar_wait(&full[st], ((it - 1 - st) / (uint32_t)a.SA) & 1u)) fail();
    }
    __syncwarp();
  } else if (warp == 1) {
    // ------------------------------------------------------------------ MMA issuer
    auto warpWait = [&](uint64_t *bar, uint32_t parity) -> bool {
      int okw = 0;
      if (lane == 0) okw = mbar_wait_ab(bar, parity, &abortFlag) ? 1 : 0;
      return __shfl_sync(0xffffffffu, okw, 0) != 0;
    };
    // both operands MN-major (instruction descriptor bits 15 and 16); leading (K) byte
    // offset 128, stride (M / N) byte offsets one channel group
    const uint32_t idesc = instr_desc(kTM, a.KN) | (1u << 15) | (1u << 16);
    const uint32_t aHi = smem_desc_hi(kWgDyGroup), bHi = smem_desc_hi(kWgXGroup);
    const uint32_t aLo0 = smem_desc_lo(smem_u32(smem), 128), bLo0 = smem_desc_lo(smem_u32(smem + 16 * kWgDyGroup), 128);
    const uint32_t stU = stB >> 4;
    bool ok = true;
    uint32_t it = 0;
    for (int t = slice; t < a.tiles && ok; t += slices, it++) {
      const uint32_t s = it % (uint32_t)a.SA;
      if (!warpWait(&full[s], (it / (uint32_t)a.SA) & 1u)) { ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;\n");
      const uint32_t aSt = aLo0 + s * stU, bSt = bLo0 + s * stU;
      for (int k = 0; k < kTM / 16; k++) {
#pragma unroll
        for (int tap = 0; tap < 9; tap++) {
          const uint32_t dy = (uint32_t)(tap / 3), dx = (uint32_t)(tap % 3);
          umma_f16_ab(tmem + (uint32_t)(tap * a.KN), aSt + 16u * (uint32_t)k, aHi,
                      bSt + dy * (kRowBytes >> 4) + 16u * (uint32_t)k + dx, bHi, idesc, (it > 0 || k > 0) ? 1u : 0u);
        }
      }
      if (lane == 0) umma_commit(&empty[s]);
      __syncwarp();
    }
    if (lane == 0) {
      if (!ok) fail();
      umma_commit(&done);   // every MMA issued by this warp has completed
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------------ epilogue
    int go = 1;
    if (lane == 0) go = mbar_wait_ab(&done, 0, &abortFlag) ? 1 : 0;
    go = __shfl_sync(0xffffffffu, go, 0);
    if (go && !abortFlag && slice < a.tiles) {
      asm volatile("tcgen05.fence::after_thread_sync;\n");
      const int qd = warp & 3, co = qd * 32 + lane;
      const uint32_t tBase = tmem + ((uint32_t)(qd * 32) << 16);
      for (int tap = 0; tap < 9; tap++)
        for (int c0 = 0; c0 < a.KN; c0 += 16) {
          uint32_t v32[16];
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
              : "=r"(v32[0]), "=r"(v32[1]), "=r"(v32[2]), "=r"(v32[3]), "=r"(v32[4]), "=r"(v32[5]), "=r"(v32[6]),
                "=r"(v32[7]), "=r"(v32[8]), "=r"(v32[9]), "=r"(v32[10]), "=r"(v32[11]), "=r"(v32[12]), "=r"(v32[13]),
                "=r"(v32[14]), "=r"(v32[15])
              : "r"(tBase + (uint32_t)(tap * a.KN + c0)));
          asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
          if (co < a.Cout) {
            float *d = a.dW + ((size_t)tap * a.Cout + co) * a.Cin + (size_t)g * a.KN + c0;
#pragma unroll
            for (int j = 0; j < 16; j++) atomicAdd(d + j, __uint_as_float(v32[j]));
          }
        }
    } else if (!go && lane == 0) {
      fail();
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  if (warp == 1) {
    asm volatile("tcgen05.fence::after_thread_sync;\n");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(512));
  }
}

// weights [tap][co][ci] (forward layout, tap = 3 dy + dx) -> operand layout
// [dx][ci / 8][dy][co][8]: for one horizontal tap and 8 input channels the three vertical
// taps' Cout rows are contiguous, so one MMA can take all three (N = 3 Cout)
__global__ void umma_weights_kernel(const bf16 *Wf, bf16 *Wu, int Cin, int Cout) {
  const size_t n = (size_t)9 * Cin * Cout;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int ci = (int)(i % Cin);
    const size_t r = i / Cin;
    const int co = (int)(r % Cout);
    const int tap = (int)(r / Cout);
    const int dy = tap / 3, dx = tap % 3;
    Wu[((((size_t)dx * (Cin / 8) + ci / 8) * 3 + dy) * Cout + co) * 8 + (ci & 7)] = Wf[i];
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

constexpr size_t kSmemBudget = 224 * 1024;     // dynamic shared memory of one CTA (one per SM)
constexpr size_t kSmemFloor = 120 * 1024;      // requested at least: keeps a second CTA off the SM
constexpr size_t kResidentMax = 112 * 1024;    // weights kept resident up to this size

int chunks_of(int Cin, const TcTiling &t) { return t.KC > 0 ? Cin / t.KC : 0; }
// weight stages hold one input-channel chunk (all 9 taps); NS >= chunks keeps them resident
bool resident_of(int Cin, const TcTiling &t) { return t.NS >= chunks_of(Cin, t); }

size_t tc_smem(int Cin, int Cout, const TcTiling &t) {
  const int stages = resident_of(Cin, t) ? chunks_of(Cin, t) : t.NS;
  return (size_t)t.SA * (t.KC / 8) * a_slot(t.R) + (size_t)stages * 18 * t.KC * Cout;
}

int g_tcStall = 0;     // launches left that run with the stall test hook
int g_tcPolicy = 1;   // 1: two accumulators (the epilogue overlaps the next tile); 0: one

// Largest input-channel chunk (a divisor of Cin, multiple of 16) that fits the budget with
// SA input stages and the given weight staging (NS = 0: resident); 0 when none does.
int fit_kc(int Cin, int Cout, int R, int SA, int NS, int AB) {
  for (int KC = Cin; KC >= 16; KC -= 16) {
    if (Cin % KC) continue;
    TcTiling t;
    t.R = R; t.KC = KC; t.SA = SA; t.AB = AB;
    t.NS = NS > 0 ? NS : Cin / KC;
    if (Cin / KC > kMaxWStages && NS == 0) continue;
    if (tc_smem(Cin, Cout, t) <= kSmemBudget) return KC;
  }
  return 0;
}

int rows_max(int Cout, int AB, int H) {
  int r = (512 / AB) / Cout;
  if (r > 8) r = 8;
  if (r > H) r = H;
  return r;
}

// Default tiling: the most rows that AB accumulators allow, resident weights when they
// fit kResidentMax (else a ring of 2 chunk stages), the most input stages (4 .. 2) that fit
// with the largest chunk.  Policy 1 uses two accumulators (the epilogue of a tile overlaps
// the MMAs of the next), policy 0 one.
TcTiling tc_tiling(int Cin, int Cout, int H) {
  TcTiling t;
  const int AB = g_tcPolicy == 1 ? 2 : 1;
  const int R = rows_max(Cout, AB, H > 0 ? H : 1);
  if (R < 1) return t;
  const bool res = (size_t)18 * Cin * Cout <= kResidentMax;
  for (int SA = kMaxAStages; SA >= 2; SA--) {
    const int KC = fit_kc(Cin, Cout, R, SA, res ? 0 : 2, AB);
    if (KC) {
      t.R = R; t.KC = KC; t.SA = SA; t.AB = AB;
      t.NS = res ? Cin / KC : 2;
      t.ST = 3 * Cout <= 256 ? 1 : 0;
      return t;
    }
  }
  return t;
}

int num_sms() {
  static int cached[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  if (!cached[dev]) {
    int n = 0;
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = n > 0 ? n : 148;
  }
  return cached[dev];
}

}  // namespace

bool conv3x3_tc_valid(int Cin, int Cout, int H, const TcTiling &t) {
  if (t.R < 1 || t.R > 8 || t.R > (H > 0 ? H : 1) || (t.AB != 1 && t.AB != 2) || t.AB * t.R * Cout > 512) return false;
  if (t.KC < 16 || t.KC % 16 || Cin % t.KC || t.SA < 2 || t.SA > kMaxAStages) return false;
  if (t.ST && 3 * Cout > 256) return false;
  if (resident_of(Cin, t) ? chunks_of(Cin, t) > kMaxWStages : (t.NS < 2 || t.NS > kMaxWStages)) return false;
  return tc_smem(Cin, Cout, t) <= kSmemBudget;
}

// Candidate tilings for the autotuner: stacked vertical taps or not, rows per tile (the
// most, half of it; one or two accumulators), input stages 2..4, weights resident or in a
// ring of 2 or 3 chunk stages, each with the largest chunk that fits.
int conv3x3_tc_candidates(int Cin, int Cout, int H, TcTiling *out, int maxOut) {
  int n = 0;
  auto add = [&](int R, int AB, int SA, int NS, int ST) {
    if (R < 1 || n >= maxOut) return;
    const int KC = fit_kc(Cin, Cout, R, SA, NS, AB);
    if (!KC) return;
    TcTiling t;
    t.R = R; t.KC = KC; t.SA = SA; t.AB = AB; t.ST = ST;
    t.NS = NS > 0 ? NS : Cin / KC;
    if (!conv3x3_tc_valid(Cin, Cout, H, t)) return;
    for (int i = 0; i < n; i++)
      if (out[i].R == t.R && out[i].KC == t.KC && out[i].SA == t.SA && out[i].AB == t.AB && out[i].NS == t.NS &&
          out[i].ST == t.ST)
        return;
    out[n++] = t;
  };
  const int h = H > 0 ? H : 1;
  for (int ST = 3 * Cout <= 256 ? 1 : 0; ST >= 0; ST--)
    for (int AB = 2; AB >= 1; AB--) {
      const int Rm = rows_max(Cout, AB, h);
      for (int R : {Rm, Rm / 2})
        for (int SA = 2; SA <= kMaxAStages; SA++) {
          if ((size_t)18 * Cin * Cout <= kSmemBudget) add(R, AB, SA, 0, ST);
          add(R, AB, SA, 2, ST);
          add(R, AB, SA, 3, ST);
        }
    }
  return n;
}

bool conv3x3_tc_supported(int Cin, int Cout) {
  return Cin % 16 == 0 && Cin >= 16 && Cout % 16 == 0 && Cout >= 16 && Cout <= 256 && tc_tiling(Cin, Cout, 1).R > 0 &&
         encode_fn() != nullptr;
}

void conv3x3_tc_stall_test(int launches) { g_tcStall = launches > 0 ? launches : 0; }

// The weight gradient's input-channel chunk: the largest divisor of Cin that is a multiple
// of 16 and at most 48 (nine taps' accumulators then fit the 512 TMEM columns); 0 if none.
int wgrad_tc_chunk(int Cin) {
  for (int kn = 48; kn >= 16; kn -= 16)
    if (Cin % kn == 0) return kn;
  return 0;
}

bool conv3x3_wgrad_tc_supported(int Cin, int Cout) {
  return Cout % 8 == 0 && Cout >= 8 && Cout <= 128 && wgrad_tc_chunk(Cin) > 0 && encode_fn() != nullptr;
}

int conv3x3_wgrad_tc(const void *X, const void *dY, float *dW, int N, int H, int W, int Cin, int Cout, int *err,
                     void *stream) {
  if (!conv3x3_wgrad_tc_supported(Cin, Cout) || N <= 0 || H <= 0 || W <= 0 || !err) return (int)cudaErrorInvalidValue;
  if ((reinterpret_cast<uintptr_t>(X) & 15) || (reinterpret_cast<uintptr_t>(dY) & 15)) return (int)cudaErrorInvalidValue;
  WgradArgs a;
  a.dW = dW; a.err = err;
  a.N = N; a.H = H; a.W = W; a.Cin = Cin; a.Cout = Cout;
  a.KN = wgrad_tc_chunk(Cin);
  a.NG = Cin / a.KN;
  const uint32_t stB = wg_stage_bytes(a.KN);
  a.SA = (int)(kSmemBudget / stB);
  if (a.SA > kWgMaxStages) a.SA = kWgMaxStages;
  if (a.SA < 2) return (int)cudaErrorInvalidValue;
  a.tilesX = (W + kTM - 1) / kTM;
  a.tiles = N * H * a.tilesX;
  auto encode = [&](CUtensorMap *m, const void *base, int C, int boxW, int boxH) -> bool {
    const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
    const cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
    const cuuint32_t box[4] = {8, (cuuint32_t)boxW, (cuuint32_t)boxH, 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    return encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(base), dims, strides, box, es,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  CUtensorMap mapDY, mapX;
  if (!encode(&mapDY, dY, Cout, kTM, 1) || !encode(&mapX, X, Cin, kHalo, 3)) return (int)cudaErrorInvalidValue;
  const size_t smem = (size_t)a.SA * stB + 1024;
  cudaError_t e = cudaFuncSetAttribute(conv3x3_wgrad_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(kSmemBudget + 1024));
  if (e != cudaSuccess) return (int)e;
  int slices = num_sms() / a.NG;
  if (slices > a.tiles) slices = a.tiles;
  if (slices < 1) slices = 1;
  conv3x3_wgrad_tc_kernel<<<(unsigned)(slices * a.NG), kWgThreads, smem, (cudaStream_t)stream>>>(mapDY, mapX, a);
  return (int)cudaGetLastError();
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
               int relu, int outF32, int *err, void *stream, const TcTiling *tiling, const TcResidual *res,
               void *poolOut, bool *pooled, const void *X2, int C1, int pdl) {
  if (pooled) *pooled = false;
  if (!X2) C1 = Cin;
  if (C1 <= 0 || C1 > Cin || C1 % 8 || (X2 && (reinterpret_cast<uintptr_t>(X2) & 15)))
    return (int)cudaErrorInvalidValue;
  if (!conv3x3_tc_supported(Cin, Cout) || N <= 0 || H <= 0 || W <= 0) return (int)cudaErrorInvalidValue;
  if ((reinterpret_cast<uintptr_t>(X) & 15) || (reinterpret_cast<uintptr_t>(Wu) & 15)) return (int)cudaErrorInvalidValue;
  TcTiling tl = tc_tiling(Cin, Cout, H);
  if (tiling && tiling->R > 0) tl = *tiling;
  if (!conv3x3_tc_valid(Cin, Cout, H, tl)) return (int)cudaErrorInvalidValue;
  // NHWC tensor maps of the input (C1 channels) and, split inputs, of the second input
  // (Cin - C1 channels); box 8 channels x 130 pixels x R + 2 rows
  auto encode = [&](CUtensorMap *m, const void *base, int C) -> bool {
    const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)N};
    const cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
    const cuuint32_t box[4] = {8, (cuuint32_t)kHalo, (cuuint32_t)(tl.R + 2), 1};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    return encode_fn()(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(base), dims, strides, box, es,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  CUtensorMap map, map2;
  if (!encode(&map, X, C1)) return (int)cudaErrorInvalidValue;
  if (X2 ? !encode(&map2, X2, Cin - C1) : false) return (int)cudaErrorInvalidValue;
  if (!X2) map2 = map;
  ConvArgs a;
  a.Wu = (const bf16 *)Wu; a.bias = bias; a.Y = Y; a.err = err;
  a.C1 = C1;
  a.N = N; a.H = H; a.W = W; a.Cin = Cin; a.Cout = Cout; a.relu = relu; a.outF32 = outF32;
  a.R = tl.R; a.KC = tl.KC; a.NS = tl.NS; a.SA = tl.SA; a.AB = tl.AB; a.ST = tl.ST;
  a.stallTest = g_tcStall > 0 ? 1 : 0;
  if (g_tcStall > 0) g_tcStall--;
  a.resF = res ? res->F : nullptr;
  a.resOut = res ? res->out4 : nullptr;
  a.resH = res ? res->H : 0;
  a.resW = res ? res->W : 0;
  if (res && (!res->F || !res->out4 || res->H > H || res->W > W || Cout < 3)) return (int)cudaErrorInvalidValue;
  const bool fusePool = poolOut && !res && !outF32 && tl.R % 2 == 0 && H % 2 == 0 && W % 2 == 0;
  a.poolOut = fusePool ? poolOut : nullptr;
  a.pdl = pdl ? 1 : 0;
  a.resident = resident_of(Cin, tl) ? 1 : 0;
  a.tmemCols = tmem_cols_for(tl.AB * tl.R * Cout);
  a.tilesX = (W + kTM - 1) / kTM;
  a.tilesY = (H + tl.R - 1) / tl.R;
  a.tiles = N * a.tilesX * a.tilesY;
  size_t smem = tc_smem(Cin, Cout, tl) + 1024;
  if (smem < kSmemFloor) smem = kSmemFloor;
  cudaError_t e = cudaFuncSetAttribute(conv3x3_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(kSmemBudget + 1024));
  if (e != cudaSuccess) return (int)e;
  int grid = num_sms();
  if (grid > a.tiles) grid = a.tiles;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = (cudaStream_t)stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaError_t le = cudaLaunchKernelEx(&cfg, conv3x3_tc_kernel, map, map2, a);
  if (le == cudaSuccess) le = cudaGetLastError();
  if (le == cudaSuccess && pooled) *pooled = fusePool;
  return (int)le;
}

}  // namespace nn
}  // namespace mdwt
