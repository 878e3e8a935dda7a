// TEST INFRASTRUCTURE ONLY: C entry points over the reference's own sources, so that the
// tests can check the oracle's restatement against them.  oracle/Makefile (target `ref`)
// compiles this file together with the reference's dda.h and rawFile.cpp where they lie,
// with the OWL stand-in of oracle/ref_shim, into oracle/_ref/libref_pins.so.  Nothing of
// the reference is copied here; the product never loads this library.
//
// Floating-point contraction follows how the reference builds each part: dda.h is CUDA
// device code (nvcc contracts a*b+c by default), so this file is compiled with FMA
// contraction; rawFile.cpp is host code for the baseline x86-64 target (no FMA), so it is
// compiled without.
#include <cstdint>
#include <cstring>
#include <vector>   // rawFile.h uses std::vector and relies on its includer for it

#include "dda.h"
#include "rawFile.h"

extern "C" {

// dda::dda3 (dda.h:81-202) from org along dir up to tMax over a grid of gs cells: the
// cells visited and each cell's (t0, t1), at most maxOut of them (the callback stops the
// walk there).  Returns the number written.
int ref_dda_trace(const float org[3], const float dir[3], float tMax, const uint32_t gs[3], int maxOut,
                  int32_t *cells, float *t0, float *t1) {
  int n = 0;
  if (maxOut <= 0) return 0;
  auto visit = [&](owl::vec3i c, float a, float b) -> bool {
    cells[3 * n] = c.x;
    cells[3 * n + 1] = c.y;
    cells[3 * n + 2] = c.z;
    t0[n] = a;
    t1[n] = b;
    return ++n < maxOut;
  };
  dda::dda3(owl::vec3f(org[0], org[1], org[2]), owl::vec3f(dir[0], dir[1], dir[2]), tMax,
            owl::vec3ui(gs[0], gs[1], gs[2]), visit, false);
  return n;
}

// raw::RawR::RawR(path, "rb") (rawFile.cpp:31-128): the parsed dims and data format, the
// box4f bounds (getBounds4f: lower xyzw, upper xyzw) and the converted values
// (getDataVector).  Returns the voxel count; the values are written only when `cap`
// holds them all.  The file must exist (the reference reads it unchecked).
int64_t ref_raw_load(const char *path, int64_t dims[3], int *format, float bounds8[8], float *out, int64_t cap) {
  raw::RawR r(path, "rb");
  const raw::Vec3l d = r.getDims();
  dims[0] = d.x;
  dims[1] = d.y;
  dims[2] = d.z;
  *format = (int)r.getDataFormat();
  const owl::box4f b = r.getBounds4f();
  const float v[8] = {b.lower.x, b.lower.y, b.lower.z, b.lower.w, b.upper.x, b.upper.y, b.upper.z, b.upper.w};
  std::memcpy(bounds8, v, sizeof(v));
  const std::vector<float> data = r.getDataVector();
  const int64_t n = (int64_t)data.size();
  if (out && n <= cap) std::memcpy(out, data.data(), (size_t)n * sizeof(float));
  return n;
}

// raw::RawR::reshapeBounds (rawFile.cpp:217-237, the viewer's -cb): the box4f bounds of the
// loaded file after rescaling its xyz bounds by its dims (scale3 == nullptr) or by scale3.
int ref_raw_reshape(const char *path, const float *scale3, float bounds8[8]) {
  raw::RawR r(path, "rb");
  if (scale3) r.reshapeBounds(owl::vec3f(scale3[0], scale3[1], scale3[2]));
  else r.reshapeBounds();
  const owl::box4f b = r.getBounds4f();
  const float v[8] = {b.lower.x, b.lower.y, b.lower.z, b.lower.w, b.upper.x, b.upper.y, b.upper.z, b.upper.w};
  std::memcpy(bounds8, v, sizeof(v));
  return 0;
}

}  // extern "C"
