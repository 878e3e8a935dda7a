// mdwt_kernels.cu -- sm_100a kernels of the majorant-grid build.
//
// Compiled with --fmad=false: every fused multiply-add below is an explicit fmaf(),
// placed where the reference's expression has the a*b+c form that nvcc contracts
// by default.  Divisions and square roots are IEEE (no fast-math), so the kernels
// reproduce the CPU oracle bit for bit.
//
// Kernels
//   range_xy_kernel / range_z_kernel : per-(cell, channel) value range, the result of
//       rasterElements + rasterBox (renderer.cu:487-519, 835-893) computed as a
//       separable box min/max over voxel intervals (no atomics, volume read once).
//   majorant_kernel : _recalculateDensityRangesMM / _recalculateDensityRanges(float2*)
//       (renderer.cu:111-203): TF-mapped maximum per (cell, channel) or per cell.
// The tracker kernel is in mdwt_track.cu.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <mutex>

#include "../../include/mdwt.h"
#include "mdwt_internal.h"
#include "mdwt_math.cuh"

namespace mdwt {
namespace {

// ------------------------------------------------------------------ value ranges
// Pass 1: per (z, cy, cx), min/max over voxels y in ivy[cy], x in ivx[cx] of slice z.
template <int SK>
__global__ void range_xy_kernel(const void *__restrict__ vol, int X, int Y, int Z,
                                const int *__restrict__ ivx, const int *__restrict__ ivy,
                                int mcx, int mcy, float2 *__restrict__ out) {
  const size_t n = (size_t)Z * mcy * mcx;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int cx = (int)(i % mcx);
    const int cy = (int)((i / mcx) % mcy);
    const int z = (int)(i / ((size_t)mcx * mcy));
    const int x0 = __ldg(ivx + 2 * cx), x1 = __ldg(ivx + 2 * cx + 1);
    const int y0 = __ldg(ivy + 2 * cy), y1 = __ldg(ivy + 2 * cy + 1);
    float mn = __int_as_float(0x7f800000), mx = __int_as_float(0xff800000);
    for (int y = y0; y <= y1; y++) {
      for (int x = x0; x <= x1; x++) {
        const float v = vox<SK>(vol, vidx<SK, size_t>(x, y, z, X, Y));
        if (v < mn) mn = v;   // NaN never enters (atomicMin CAS loop: `while (val < old)`)
        if (v > mx) mx = v;
      }
    }
    out[i] = make_float2(mn, mx);
  }
}

// Float32 voxels, x fastest, into the micro-brick layout (kStoreF32): one thread per
// voxel, reads coalesced along x, writes two floats apart within a brick.
__global__ void brick_f32_kernel(const float *__restrict__ src, float *__restrict__ dst, int X, int Y, int Z) {
  const size_t n = (size_t)X * Y * Z;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(i % (size_t)X);
    const size_t r = i / (size_t)X;
    const int y = (int)(r % (size_t)Y), z = (int)(r / (size_t)Y);
    dst[vidx<kStoreF32, size_t>(x, y, z, X, Y)] = __ldg(src + i);
  }
}

// Pass 2: per (cz, cy, cx), min/max over z in ivz[cz]; merged with the sizeMCs value
// (1e20, -1e20) into ranges[(cell*C + ch)].
__global__ void range_z_kernel(const float2 *__restrict__ in, const int *__restrict__ ivz, int mcx, int mcy, int mcz,
                               int C, int ch, float2 *__restrict__ ranges) {
  const size_t n = (size_t)mcz * mcy * mcx;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t cxy = i % ((size_t)mcx * mcy);
    const int cz = (int)(i / ((size_t)mcx * mcy));
    const int z0 = __ldg(ivz + 2 * cz), z1 = __ldg(ivz + 2 * cz + 1);
    float2 r = ranges[i * C + ch];
    for (int z = z0; z <= z1; z++) {
      const float2 a = in[(size_t)z * mcx * mcy + cxy];
      if (a.x < r.x) r.x = a.x;
      if (a.y > r.y) r.y = a.y;
    }
    ranges[i * C + ch] = r;
  }
}

__global__ void range_init_kernel(float2 *ranges, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    ranges[i] = make_float2(1e20f, -1e20f);
}

// ------------------------------------------------------------------ majorants
__device__ __forceinline__ float tf_probe(const float *A, int n, float u) {
  const Axis a = axis(u, n);
  return lerpf(a.a, __ldg(A + a.i0), __ldg(A + a.i1));
}

__device__ float channel_majorant(const MajorantParams &p, int c, float mn, float mx) {
  if (mx < mn) return 0.f;
  const int n = p.tfN[c];
  if (n <= 0) return 0.f;
  const float *A = p.tfAlpha[c];
  const float os = p.os[c];
  const float v0 = p.vd[c][0], v1 = p.vd[c][1], x0 = p.xd[c][0], x1 = p.xd[c][1];
  const float rmin1 = (mn - v0) / (v1 - v0);
  const float rmin = (rmin1 - x0) / (x1 - x0);
  const float rmax1 = (mx - v0) / (v1 - v0);
  const float rmax = (rmax1 - x0) / (x1 - x0);
  const float addr1 = rmin * (float)n;
  const float addr2 = rmax * (float)n;
  const int aMin = clampi(f2i(fminf(floorf(addr1), floorf(addr2))), 0, n - 1);
  const int aMax = clampi(f2i(fmaxf(ceilf(addr1), ceilf(addr2))), 0, n - 1);
  float m = 0.f;
  for (int i = aMin; i <= aMax; ++i) {
    const float dns = tf_probe(A, n, ((float)i + 0.5f) / (float)n) * os;
    m = (i == aMin) ? dns : fmaxf(m, dns);
  }
  m = fmaxf(m, tf_probe(A, n, (addr1 + 0.5f) / (float)n) * os);
  m = fmaxf(m, tf_probe(A, n, (addr2 + 0.5f) / (float)n) * os);
  return m;
}

// The reciprocal the trackers' table holds beside a majorant: recip_for_div for the exact
// chain's quotients, or 1 / majorant for the fast arithmetic's flights.
__device__ __forceinline__ float table_recip(const MajorantParams &p, float v) {
  if (p.fast) return v != 0.0f ? 1.0f / v : 0.0f;
  return recip_for_div(v);
}

__global__ void majorant_kernel(const __grid_constant__ MajorantParams p) {
  const int C = p.C;
  for (size_t cell = (size_t)blockIdx.x * blockDim.x + threadIdx.x; cell < p.M; cell += (size_t)gridDim.x * blockDim.x) {
    const float2 *r = reinterpret_cast<const float2 *>(p.ranges) + cell * C;
    if (p.mode >= 3) {   // summed majorant: -m 3 and the blending modes -m 4/5 (renderer.cu:250-257)
      float sum = 0.f;
      for (int c = 0; c < C; c++) {
        const float2 rc = r[c];
        if (rc.y < rc.x) continue;
        sum += channel_majorant(p, c, rc.x, rc.y);
      }
      p.majorants[cell] = sum;
      if (p.cellTab) {
        p.cellTab[cell * 2] = make_float2(__uint_as_float(sum != 0.0f ? 1u : 0u), 0.0f);
        p.cellTab[cell * 2 + 1] = make_float2(sum, table_recip(p, sum));
      }
    } else {
      uint32_t m = 0;
      float2 *tab = p.cellTab ? p.cellTab + cell * (C + 1) : nullptr;
      for (int c = 0; c < C; c++) {
        const float2 rc = r[c];
        const float v = channel_majorant(p, c, rc.x, rc.y);
        p.majorants[cell * C + c] = v;
        if (tab) tab[1 + c] = make_float2(v, table_recip(p, v));
        if (v != 0.0f) m |= 1u << c;
      }
      if (tab) tab[0] = make_float2(__uint_as_float(m), 0.0f);
    }
  }
}

inline int grid_for(size_t n, int tpb, int cap) {
  size_t g = (n + tpb - 1) / tpb;
  if (g < 1) g = 1;
  if (g > (size_t)cap) g = cap;
  return (int)g;
}

}  // namespace

// ------------------------------------------------------------------ launchers
int launch_ranges_init(float *ranges, size_t count, void *stream, int *launches) {
  range_init_kernel<<<grid_for(count, 256, 4096), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<float2 *>(ranges), count);
  if (launches) *launches += 1;
  return (int)cudaGetLastError();
}

int launch_ranges(const void *vol, int storeKind, const int dims[3], const uint32_t mc[3],
                  const int *ivx, const int *ivy, const int *ivz, int C, int ch,
                  float *ranges, float *scratchA, float * /*scratchB*/, void *stream, int *launches) {
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n1 = (size_t)dims[2] * mc[1] * mc[0];
  float2 *A = reinterpret_cast<float2 *>(scratchA);
  if (storeKind == kStoreU8)
    range_xy_kernel<kStoreU8><<<grid_for(n1, 256, 148 * 64), 256, 0, st>>>(vol, dims[0], dims[1], dims[2], ivx, ivy, (int)mc[0], (int)mc[1], A);
  else if (storeKind == kStoreF32)
    range_xy_kernel<kStoreF32><<<grid_for(n1, 256, 148 * 64), 256, 0, st>>>(vol, dims[0], dims[1], dims[2], ivx, ivy, (int)mc[0], (int)mc[1], A);
  else
    range_xy_kernel<kStoreF32Lin><<<grid_for(n1, 256, 148 * 64), 256, 0, st>>>(vol, dims[0], dims[1], dims[2], ivx, ivy, (int)mc[0], (int)mc[1], A);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return (int)e;
  const size_t n2 = (size_t)mc[2] * mc[1] * mc[0];
  range_z_kernel<<<grid_for(n2, 256, 148 * 64), 256, 0, st>>>(A, ivz, (int)mc[0], (int)mc[1], (int)mc[2], C, ch,
                                                              reinterpret_cast<float2 *>(ranges));
  if (launches) *launches += 2;
  return (int)cudaGetLastError();
}

size_t stored_voxels(int storeKind, const int64_t dims[3]) {
  if (storeKind == kStoreF32)
    return (size_t)8 * (size_t)((dims[0] + 1) / 2) * (size_t)((dims[1] + 1) / 2) * (size_t)((dims[2] + 1) / 2);
  return (size_t)dims[0] * (size_t)dims[1] * (size_t)dims[2];
}

int launch_brick_f32(const float *src, float *dst, const int dims[3], void *stream, int *launches) {
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t d64[3] = {dims[0], dims[1], dims[2]};
  const size_t nb = stored_voxels(kStoreF32, d64), n = (size_t)dims[0] * dims[1] * dims[2];
  cudaError_t e = cudaSuccess;
  if (nb > n) e = cudaMemsetAsync(dst, 0, nb * sizeof(float), st);   // the padding voxels of odd dims
  if (e != cudaSuccess) return (int)e;
  brick_f32_kernel<<<grid_for(n, 256, 148 * 64), 256, 0, st>>>(src, dst, dims[0], dims[1], dims[2]);
  if (launches) *launches += 1;
  return (int)cudaGetLastError();
}

int launch_majorants(const MajorantParams &p, void *stream, int *launches) {
  majorant_kernel<<<grid_for(p.M, 128, 148 * 32), 128, 0, (cudaStream_t)stream>>>(p);
  if (launches) *launches += 1;
  return (int)cudaGetLastError();
}

// ------------------------------------------------------------------ range build without allocation
// Scratch of mdwt_build_ranges_noalloc: the per-(z, cell-y, cell-x) partial ranges and
// the voxel intervals.  Module globals: every device that loads the library holds them
// (8 MiB + 24 KiB) until the process exits.
namespace {
constexpr size_t kNoAllocPairs = size_t(1) << 20;
constexpr int kNoAllocMaxCells = 1024;
static __device__ __align__(256) float2 g_noalloc_pairs[kNoAllocPairs];
static __device__ __align__(256) int g_noalloc_iv[3 * 2 * kNoAllocMaxCells];

__device__ __forceinline__ int project_d(float f, float lo, float hi, int dim) {
  int v = f2i((float)dim * (f - lo) / (hi - lo));
  v = v < dim - 1 ? v : dim - 1;
  return v > 0 ? v : 0;
}

// Cells [clo, chi] that the 27-neighbour box of voxel p touches on one axis.
__device__ __forceinline__ void voxel_cells(int p, int D, int md, float wlo, float whi, float len, int &clo, int &chi) {
  const float vlo = fmaf((float)p, len, wlo);
  float blo = vlo, bhi = vlo + len;
  if (p - 1 >= 0) { const float nl = fmaf((float)(p - 1), len, wlo); blo = fminf(blo, nl); bhi = fmaxf(bhi, nl); }
  if (p + 1 < D) { const float nl = fmaf((float)(p + 1), len, wlo); blo = fminf(blo, nl); bhi = fmaxf(bhi, nl); }
  clo = project_d(blo, wlo, whi, md);
  const int h = project_d(bhi, wlo, whi, md);
  chi = h < md - 1 ? h : md - 1;
}

// One thread per (axis, cell index): the voxel interval of the separable range build,
// found by binary search (clo and chi are non-decreasing in p for these bounds).
__global__ void noalloc_intervals_kernel(int dx, int dy, int dz, int mx, int my, int mz, float lx, float ly, float lz,
                                         float hx, float hy, float hz, int *iv) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int D, md, off;
  float wlo, whi;
  if (t < mx) { D = dx; md = mx; wlo = lx; whi = hx; off = 0; }
  else if (t < mx + my) { t -= mx; D = dy; md = my; wlo = ly; whi = hy; off = 2 * mx; }
  else if (t < mx + my + mz) { t -= mx + my; D = dz; md = mz; wlo = lz; whi = hz; off = 2 * (mx + my); }
  else return;
  const int k = t;
  const float len = (whi - wlo) / (float)D;
  int lo = 0, hi = D;
  while (lo < hi) {  // first p with chi(p) >= k
    const int mid = (lo + hi) >> 1;
    int cl, ch;
    voxel_cells(mid, D, md, wlo, whi, len, cl, ch);
    if (ch >= k) hi = mid; else lo = mid + 1;
  }
  const int pmin = lo;
  lo = 0; hi = D;
  while (lo < hi) {  // first p with clo(p) > k
    const int mid = (lo + hi) >> 1;
    int cl, ch;
    voxel_cells(mid, D, md, wlo, whi, len, cl, ch);
    if (cl > k) hi = mid; else lo = mid + 1;
  }
  const int pmax = lo - 1;
  if (pmin > pmax) { iv[off + 2 * k] = 1; iv[off + 2 * k + 1] = 0; return; }
  iv[off + 2 * k] = pmin - 1 > 0 ? pmin - 1 : 0;
  iv[off + 2 * k + 1] = pmax + 1 < D - 1 ? pmax + 1 : D - 1;
}

std::mutex g_noalloc_mu;
constexpr int kNoAllocMaxDevices = 64;
void *g_noalloc_pairs_ptr[kNoAllocMaxDevices];
int *g_noalloc_iv_ptr[kNoAllocMaxDevices];
bool g_noalloc_ready[kNoAllocMaxDevices];

int f2i_h(float x) {
  if (!(x == x)) return 0;
  if (x >= 2147483648.0f) return 2147483647;
  if (x <= -2147483648.0f) return (-2147483647 - 1);
  return (int)x;
}

int project_h(float f, float lo, float hi, int dim) {
  int v = f2i_h((float)dim * (f - lo) / (hi - lo));
  v = v < dim - 1 ? v : dim - 1;
  return v > 0 ? v : 0;
}

// The device search of noalloc_intervals_kernel finds, for each cell k, the run of voxels
// whose neighbour boxes reach k.  It gives the voxel set that mdwt_init's scan finds when
// every voxel's neighbour box is non-empty and the cells it touches are non-decreasing
// in the voxel index.  Checked here over every voxel of the axis, with the arithmetic
// of voxel_cells (fmaf corners, IEEE division, truncating conversion).
bool axis_searchable(int64_t D, int md, float wlo, float whi) {
  if (!std::isfinite(wlo) || !std::isfinite(whi) || !(whi > wlo)) return false;
  const float len = (whi - wlo) / (float)D;
  int pclo = 0, pchi = 0;
  for (int64_t p = 0; p < D; p++) {
    const float vlo = std::fma((float)p, len, wlo);
    float blo = vlo, bhi = vlo + len;
    if (p - 1 >= 0) { const float nl = std::fma((float)(p - 1), len, wlo); blo = std::fmin(blo, nl); bhi = std::fmax(bhi, nl); }
    if (p + 1 < D) { const float nl = std::fma((float)(p + 1), len, wlo); blo = std::fmin(blo, nl); bhi = std::fmax(bhi, nl); }
    if (!(blo < bhi)) return false;
    const int clo = project_h(blo, wlo, whi, md);
    const int h = project_h(bhi, wlo, whi, md);
    const int chi = h < md - 1 ? h : md - 1;
    if (clo < pclo || chi < pchi) return false;
    pclo = clo;
    pchi = chi;
  }
  return true;
}
}  // namespace

}  // namespace mdwt

// Value ranges of one channel computed without allocating any memory.  For callers that
// must not allocate device memory: code running inside an application's own memory pool
// or under an allocator that forbids cudaMalloc, or plug-ins that are handed device
// buffers and a stream but no allocation rights.  The scratch is the module-global
// g_noalloc_pairs / g_noalloc_iv; a call outside stream capture looks up their addresses
// on the current device (cudaGetSymbolAddress), and a call under capture reuses the
// addresses of the last call on that device, so make the first call on a device before
// any stream capture.  All calls share the scratch: calls that overlap on the GPU (two
// streams, two threads) race.
extern "C" mdwt_status mdwt_build_ranges_noalloc(const void *d_volume, int format, const int64_t dims[3],
                                                 const uint32_t macrocells[3], const float world_lo[3],
                                                 const float world_hi[3], float *d_ranges_out, void *cuda_stream) {
  using namespace mdwt;
  if (!d_volume || !dims || !macrocells || !world_lo || !world_hi || !d_ranges_out) return MDWT_ERR_BAD_ARG;
  if (format != MDWT_FMT_UINT8 && format != MDWT_FMT_FLOAT32) return MDWT_ERR_UNSUPPORTED;
  for (int a = 0; a < 3; a++) {
    if (dims[a] <= 0 || dims[a] > (1 << 20) || macrocells[a] == 0) return MDWT_ERR_BAD_ARG;
    if (macrocells[a] > (uint32_t)kNoAllocMaxCells) return MDWT_ERR_SCRATCH_LIMIT;
  }
  if ((size_t)dims[2] * macrocells[1] * macrocells[0] > kNoAllocPairs) return MDWT_ERR_SCRATCH_LIMIT;
  for (int a = 0; a < 3; a++)
    if (!axis_searchable(dims[a], (int)macrocells[a], world_lo[a], world_hi[a])) return MDWT_ERR_UNSUPPORTED;
  // an error that earlier work left pending is reported here and left for its owner:
  // nothing is launched, and the check after the launches sees only this call's errors
  if (cudaPeekAtLastError() != cudaSuccess) return MDWT_ERR_CUDA;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) { cudaGetLastError(); return MDWT_ERR_CUDA; }
  cudaStream_t st = (cudaStream_t)cuda_stream;
  {
    // The scratch addresses are looked up on every call outside stream capture (a
    // cudaDeviceReset reloads the module and moves them); under capture the last
    // looked-up address of this device is used.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) { cudaGetLastError(); return MDWT_ERR_CUDA; }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (cap == cudaStreamCaptureStatusNone || !g_noalloc_ready[dev]) {
      if (cap != cudaStreamCaptureStatusNone) return MDWT_ERR_STATE;
      void *p = nullptr, *q = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_pairs) != cudaSuccess ||
          cudaGetSymbolAddress(&q, g_noalloc_iv) != cudaSuccess) {
        cudaGetLastError();
        return MDWT_ERR_CUDA;
      }
      g_noalloc_pairs_ptr[dev] = p;
      g_noalloc_iv_ptr[dev] = (int *)q;
      g_noalloc_ready[dev] = true;
    }
  }
  const int mx = (int)macrocells[0], my = (int)macrocells[1], mz = (int)macrocells[2];
  int *iv = g_noalloc_iv_ptr[dev];
  noalloc_intervals_kernel<<<(mx + my + mz + 127) / 128, 128, 0, st>>>(
      (int)dims[0], (int)dims[1], (int)dims[2], mx, my, mz, world_lo[0], world_lo[1], world_lo[2],
      world_hi[0], world_hi[1], world_hi[2], iv);
  if (cudaGetLastError() != cudaSuccess) return MDWT_ERR_CUDA;
  const size_t M = (size_t)mx * my * mz;
  if (launch_ranges_init(d_ranges_out, M, st, nullptr) != 0) return MDWT_ERR_CUDA;
  const int d3[3] = {(int)dims[0], (int)dims[1], (int)dims[2]};
  const uint32_t mc3[3] = {macrocells[0], macrocells[1], macrocells[2]};
  const int sk = format == MDWT_FMT_UINT8 ? kStoreU8 : kStoreF32Lin;   // the caller's layout: x fastest
  if (launch_ranges(d_volume, sk, d3, mc3, iv, iv + 2 * mx, iv + 2 * (mx + my), 1, 0, d_ranges_out,
                    (float *)g_noalloc_pairs_ptr[dev], nullptr, st, nullptr) != 0)
    return MDWT_ERR_CUDA;
  return MDWT_OK;
}
