// TEST INFRASTRUCTURE ONLY.  Stand-in for OWL's LCG<N> random generator
// (owl/common/math/random.h; the submodule is empty and its commit unpinned).  The
// project restates its published method: an N-round TEA hash (Wheeler & Needham 1994,
// delta 0x9E3779B9) of the two seed words with the first four SHA-256 initial hash words
// (FIPS 180-4) as key, feeding a 32-bit LCG with the Numerical Recipes constants
// (1664525, 1013904223); a draw is the top 24 bits of the new state times 2^-24.  This is
// the generator stream the oracle and the kernels use.
#pragma once

#include <cstdint>

namespace owl {
namespace common {

template <int N>
struct LCG {
  uint32_t state = 0;
  LCG() = default;
  SHIM_HD LCG(uint32_t v0, uint32_t v1) { init(v0, v1); }
  SHIM_HD void init(uint32_t v0, uint32_t v1) {
    const uint32_t k0 = 0x6a09e667u, k1 = 0xbb67ae85u, k2 = 0x3c6ef372u, k3 = 0xa54ff53au;
    uint32_t sum = 0;
    for (int n = 0; n < N; n++) {
      sum += 0x9E3779B9u;
      v0 += ((v1 << 4) + k0) ^ (v1 + sum) ^ ((v1 >> 5) + k1);
      v1 += ((v0 << 4) + k2) ^ (v0 + sum) ^ ((v0 >> 5) + k3);
    }
    state = v0;
  }
  SHIM_HD float operator()() {
    state = 1664525u * state + 1013904223u;
    return (float)(state >> 8) * (1.0f / 16777216.0f);
  }
};

}  // namespace common
}  // namespace owl
