// SplitMix64 as java.util.SplittableRandom implements it (the published generator:
// Steele, Lea & Flood, OOPSLA 2014): the k-th nextDouble() (k = 0, 1, ...) of a
// generator seeded with `seed` is a pure function of (seed, k), usable on the host
// and on the device.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define SC_RNG_FN __host__ __device__ __forceinline__
#else
#define SC_RNG_FN inline
#endif

namespace sc {

SC_RNG_FN uint64_t splitmix_mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}
constexpr uint64_t kGoldenGamma = 0x9e3779b97f4a7c15ULL;
SC_RNG_FN double splitmix_double(uint64_t seed, uint64_t k) {
  const uint64_t z = splitmix_mix64(seed + (k + 1ULL) * kGoldenGamma);
  return (double)(z >> 11) * 0x1.0p-53;
}

}  // namespace sc
