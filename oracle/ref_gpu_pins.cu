// TEST INFRASTRUCTURE ONLY.  The reference's own majorant pass and range raster, run on
// the GPU.  The reference's renderer.cu is included unchanged, where it lies, with the
// OWL/umesh stand-ins of ref_shim/ (made host-and-device for nvcc), and compiled by
// oracle/Makefile (`make ref`) with nvcc's default flags, as the reference's CMake
// build compiles it (FMA contraction on).  The entry points below set up the inputs the
// reference's Renderer would hand its kernels and launch them with its launch shapes:
//   refgpu_majorants: RecalculateDensityRanges (renderer.cu:206-274) -- the per-channel
//     _recalculateDensityRangesMM (renderer.cu:159-203) for -m 0..2, the summed
//     _recalculateDensityRanges (renderer.cu:111-157) for -m 3..5 -- on a transfer-function
//     texture made as Renderer::SetXFColormap makes it (renderer.cpp:1094-1165: alpha
//     cubed with powf, a float4 CUDA array, linear filtering, normalized coordinates,
//     clamp), so the texel fetches and the two probes run on the texture unit;
//   refgpu_ranges: the raw branch of buildSpatialMacrocells (renderer.cu:1116-1179) --
//     sizeMCs, then rasterElements per channel (renderer.cu:835-893 with rasterBox and
//     project, renderer.cu:387-403, 487-519).
// The tests compare libmdwt's majorants and ranges with these bit for bit.
#include "renderer.cu"

#include <cstdlib>
#include <vector>

// renderer.cu's host code names these OWL calls; the pins never reach them
OWLBuffer owlDeviceBufferCreate(OWLContext, OWLDataType, size_t, const void *) { std::abort(); }
const void *owlBufferGetPointer(OWLBuffer, int) { std::abort(); }
void owlGroupBuildAccel(OWLGroup) { std::abort(); }

namespace {
int status(cudaError_t e) { return e == cudaSuccess ? 0 : (int)e; }
}  // namespace

// ranges: float2[M * C] (cell-major, channel-minor); tf_rgba: C * n RGBA texels (alpha
// not yet cubed); vol_domain, xf_domain: C (lo, hi) pairs; opacity: C scales.  summed = 0:
// out holds M * C majorants, else M summed ones.
extern "C" int refgpu_majorants(int summed, const float *ranges, int M, int C, const float *tf_rgba, int n,
                                const float *vol_domain, const float *xf_domain, const float *opacity, float *out) {
  std::vector<dtracker::TFData> tf(C);
  std::vector<cudaArray_t> arrays(C, nullptr);
  cudaError_t e = cudaSuccess;
  for (int c = 0; c < C && e == cudaSuccess; c++) {
    std::vector<float4> cm(n);
    for (int i = 0; i < n; i++) {
      const float *t = tf_rgba + ((size_t)c * n + i) * 4;
      cm[i] = make_float4(t[0], t[1], t[2], powf(t[3], 3.f));
    }
    cudaChannelFormatDesc cd = cudaCreateChannelDesc<float4>();
    e = cudaMallocArray(&arrays[c], &cd, n, 1);
    const size_t pitch = (size_t)n * sizeof(float4);
    if (e == cudaSuccess) e = cudaMemcpy2DToArray(arrays[c], 0, 0, cm.data(), pitch, pitch, 1, cudaMemcpyHostToDevice);
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arrays[c];
    cudaTextureDesc td = {};
    td.addressMode[0] = cudaAddressModeClamp;
    td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.normalizedCoords = 1;
    td.maxAnisotropy = 1;
    td.maxMipmapLevelClamp = 99;
    td.minMipmapLevelClamp = 0;
    td.mipmapFilterMode = cudaFilterModePoint;
    td.sRGB = 0;
    if (e == cudaSuccess) e = cudaCreateTextureObject(&tf[c].colorMapTexture, &rd, &td, nullptr);
    tf[c].volDomain = interval<float>(vol_domain[2 * c], vol_domain[2 * c + 1]);
    tf[c].xfDomain = interval<float>(xf_domain[2 * c], xf_domain[2 * c + 1]);
    tf[c].numTexels = n;
    tf[c].opacityScale = opacity[c];
  }
  // the device copy of the TFData array, as the reference's OWL buffer holds it (the
  // host-side members ride along unused)
  dtracker::TFData *dTf = nullptr;
  float2 *dMc = nullptr;
  float *dMax = nullptr;
  const size_t nOut = summed ? (size_t)M : (size_t)M * C;
  if (e == cudaSuccess) e = cudaMalloc(&dTf, sizeof(dtracker::TFData) * C);
  if (e == cudaSuccess) e = cudaMemcpy(dTf, tf.data(), sizeof(dtracker::TFData) * C, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&dMc, sizeof(float2) * (size_t)M * C);
  if (e == cudaSuccess) e = cudaMemcpy(dMc, ranges, sizeof(float2) * (size_t)M * C, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&dMax, sizeof(float) * nOut);
  if (e == cudaSuccess) {
    const dim3 block(32), grid((M + 31) / 32);
    if (summed)
      _recalculateDensityRanges<<<grid, block>>>(M, dMc, dTf, (size_t)C, dMax);
    else
      _recalculateDensityRangesMM<<<grid, block>>>(M, dMc, dTf, (size_t)C, dMax);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(out, dMax, sizeof(float) * nOut, cudaMemcpyDeviceToHost);
  for (int c = 0; c < C; c++) {
    if (tf[c].colorMapTexture) cudaDestroyTextureObject(tf[c].colorMapTexture);
    if (arrays[c]) cudaFreeArray(arrays[c]);
  }
  cudaFree(dTf);
  cudaFree(dMc);
  cudaFree(dMax);
  return status(e);
}

// scalars: C channels of dims[c][0..2] float voxels each (x fastest, the values the
// reference's RawR converts to), one after the other; mc: macrocells per axis; lo, hi:
// the world bounds the reference passes (the channels' cumulative box).  out: float2[M * C].
extern "C" int refgpu_ranges(const float *scalars, const int *dims, int C, const int mc[3], const float lo[3],
                             const float hi[3], float *out) {
  const vec3i mcDims(mc[0], mc[1], mc[2]);
  const box3f bounds(vec3f(lo[0], lo[1], lo[2]), vec3f(hi[0], hi[1], hi[2]));
  const size_t M = (size_t)mc[0] * mc[1] * mc[2];
  float2 *dMc = nullptr;
  float *dS = nullptr;
  cudaError_t e = cudaMalloc(&dMc, sizeof(float2) * M * C);
  if (e == cudaSuccess) {
    const vec3i blockSize = vec3i(4);
    dtracker::sizeMCs<<<dtracker::to_dims(divRoundUp(mcDims, blockSize)), dtracker::to_dims(blockSize)>>>(
        dMc, mcDims, bounds, (size_t)C);
    e = cudaGetLastError();
  }
  size_t off = 0;
  for (int c = 0; c < C && e == cudaSuccess; c++) {
    const vec3i g(dims[3 * c], dims[3 * c + 1], dims[3 * c + 2]);
    const uint64_t count = (uint64_t)g.x * (uint64_t)g.y * (uint64_t)g.z;
    e = cudaMalloc(&dS, sizeof(float) * count);
    if (e == cudaSuccess) e = cudaMemcpy(dS, scalars + off, sizeof(float) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
      const uint64_t blockSize = 32;
      const uint64_t numBlocks = divRoundUp(count, blockSize);
      const vec3i grid((int)std::min(numBlocks, (uint64_t)dtracker::MAX_GRID_SIZE),
                       (int)divRoundUp(numBlocks, (uint64_t)dtracker::MAX_GRID_SIZE), 1);
      dtracker::rasterElements<<<dtracker::to_dims(grid), (unsigned)blockSize>>>(dMc, mcDims, bounds, dS, g, (size_t)c,
                                                                                  (size_t)C);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(dS);
    dS = nullptr;
    off += count;
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dMc, sizeof(float2) * M * C, cudaMemcpyDeviceToHost);
  cudaFree(dMc);
  return status(e);
}

// ---------------------------------------------------------------- the texture unit
// The reference samples its volumes with tex3D<float> on float 3-D arrays (normalized
// coordinates, linear filtering, clamp addressing, element-type reads; renderer.cpp:
// 251-311) and its transfer functions with tex2D<float4> on a float4 N x 1 array
// (renderer.cpp:1094-1165).  These entry points sample such textures at given
// coordinates on the GPU, so that the tests can hold the project's statement of the
// linear filter (8 fractional weight bits, clamp, lerp(a, p, q) = fmaf(a, q, (1 - a) p),
// x then y then z) against the hardware.
namespace {
__global__ void tex3d_probe(cudaTextureObject_t t, const float *xyz, int n, float *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = tex3D<float>(t, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
}
__global__ void tex2d_probe(cudaTextureObject_t t, const float *uv, int n, float4 *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = tex2D<float4>(t, uv[2 * i], uv[2 * i + 1]);
}
}  // namespace

// vol: X * Y * Z floats, x fastest; xyz: n normalized coordinates
extern "C" int refgpu_tex3d(const float *vol, int X, int Y, int Z, const float *xyz, int n, float *out) {
  cudaArray_t arr = nullptr;
  cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
  cudaError_t e = cudaMalloc3DArray(&arr, &cd, make_cudaExtent(X, Y, Z));
  if (e == cudaSuccess) {
    cudaMemcpy3DParms p = {};
    p.srcPtr = make_cudaPitchedPtr(const_cast<float *>(vol), (size_t)X * sizeof(float), X, Y);
    p.dstArray = arr;
    p.extent = make_cudaExtent(X, Y, Z);
    p.kind = cudaMemcpyHostToDevice;
    e = cudaMemcpy3D(&p);
  }
  cudaTextureObject_t t = 0;
  if (e == cudaSuccess) {
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    td.normalizedCoords = true;
    td.filterMode = cudaFilterModeLinear;
    td.addressMode[0] = cudaAddressModeClamp;
    td.addressMode[1] = cudaAddressModeClamp;
    td.addressMode[2] = cudaAddressModeClamp;
    td.readMode = cudaReadModeElementType;
    e = cudaCreateTextureObject(&t, &rd, &td, nullptr);
  }
  float *dIn = nullptr, *dOut = nullptr;
  if (e == cudaSuccess) e = cudaMalloc(&dIn, sizeof(float) * 3 * (size_t)n);
  if (e == cudaSuccess) e = cudaMemcpy(dIn, xyz, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&dOut, sizeof(float) * (size_t)n);
  if (e == cudaSuccess) {
    tex3d_probe<<<(n + 255) / 256, 256>>>(t, dIn, n, dOut);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dOut, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost);
  if (t) cudaDestroyTextureObject(t);
  if (arr) cudaFreeArray(arr);
  cudaFree(dIn);
  cudaFree(dOut);
  return status(e);
}

// rgba: N texels (as uploaded: alpha already cubed); uv: n coordinates; out: n float4
extern "C" int refgpu_tex2d(const float *rgba, int N, const float *uv, int n, float *out) {
  cudaArray_t arr = nullptr;
  cudaChannelFormatDesc cd = cudaCreateChannelDesc<float4>();
  cudaError_t e = cudaMallocArray(&arr, &cd, N, 1);
  const size_t pitch = (size_t)N * sizeof(float4);
  if (e == cudaSuccess) e = cudaMemcpy2DToArray(arr, 0, 0, rgba, pitch, pitch, 1, cudaMemcpyHostToDevice);
  cudaTextureObject_t t = 0;
  if (e == cudaSuccess) {
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td = {};
    td.addressMode[0] = cudaAddressModeClamp;
    td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModeLinear;
    td.normalizedCoords = 1;
    td.maxAnisotropy = 1;
    td.maxMipmapLevelClamp = 99;
    td.mipmapFilterMode = cudaFilterModePoint;
    e = cudaCreateTextureObject(&t, &rd, &td, nullptr);
  }
  float *dIn = nullptr;
  float4 *dOut = nullptr;
  if (e == cudaSuccess) e = cudaMalloc(&dIn, sizeof(float) * 2 * (size_t)n);
  if (e == cudaSuccess) e = cudaMemcpy(dIn, uv, sizeof(float) * 2 * (size_t)n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&dOut, sizeof(float4) * (size_t)n);
  if (e == cudaSuccess) {
    tex2d_probe<<<(n + 255) / 256, 256>>>(t, dIn, n, dOut);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dOut, sizeof(float4) * (size_t)n, cudaMemcpyDeviceToHost);
  if (t) cudaDestroyTextureObject(t);
  if (arr) cudaFreeArray(arr);
  cudaFree(dIn);
  cudaFree(dOut);
  return status(e);
}
