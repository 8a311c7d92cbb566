// AXON CPU oracle: the stimulus random stream. TEST INFRASTRUCTURE ONLY.
//
// rakib-nyc/axon draws its stimuli with std::mt19937, std::shuffle and
// std::uniform_real_distribution<double> (src/axon.mm:793-804) built against Apple
// libc++ (Xcode CLT 14.3). mt19937 is fully specified by the C++ standard, so the
// standard library's engine is used as is. shuffle and the distributions are
// implementation-defined, so libc++'s observable algorithms are restated here:
//  - shuffle: forward Fisher-Yates; position p swaps with p + uniform_int(0, n-1-p);
//  - uniform_int(a, b): w = ceil(log2(b-a+1)) low bits of one engine output, redrawn
//    while >= b-a+1 (the __independent_bits_engine path for ranges below 2^32);
//  - generate_canonical<double,53>: (x1 + x2 * 2^32) / 2^64 with the sum rounded once.
#pragma once
#include <cstdint>
#include <random>
#include <utility>
#include <vector>

namespace oracle {

inline uint64_t libcxx_uniform_int(std::mt19937& g, uint64_t a, uint64_t b) {
  const uint64_t range = b - a + 1;
  if (range == 1) return a;
  unsigned w = 63u - (unsigned)__builtin_clzll(range);
  if (range & (~0ull >> (64u - w))) ++w;  // not a power of two: one more bit
  const uint32_t mask = (w >= 32) ? 0xFFFFFFFFu : ((1u << w) - 1u);
  uint64_t u;
  do { u = (uint64_t)((uint32_t)g() & mask); } while (u >= range);
  return a + u;
}

template <class T>
inline void libcxx_shuffle(std::vector<T>& v, std::mt19937& g) {
  int64_t d = (int64_t)v.size();
  if (d <= 1) return;
  size_t first = 0, last = v.size() - 1;
  for (--d; first < last; ++first, --d) {
    uint64_t i = libcxx_uniform_int(g, 0, (uint64_t)d);
    if (i != 0) std::swap(v[first], v[first + i]);
  }
}

inline double libcxx_canonical(std::mt19937& g) {
  double s = (double)(uint32_t)g();
  s += (double)(uint32_t)g() * 4294967296.0;
  return s / 18446744073709551616.0;
}

// Noisy cue (no counterpart in the reference; the engine's axon_noisy_cue is the product
// side): start from the whole pattern clamped on, enumerate its active bits as
// (pattern position p, bit b) -> 32 p + b, and switch off the first round(frac * A)
// elements of a forward Fisher-Yates permutation of 0..A-1 drawn with
// libcxx_uniform_int(g, i, A-1) from mt19937(seed).
inline void noisy_clamp(const std::vector<uint32_t>& cols, double frac, uint32_t seed, std::vector<uint32_t>& stim) {
  std::fill(stim.begin(), stim.end(), 0u);
  for (uint32_t c : cols) stim[c] = 0xFFFFFFFFu;
  const uint64_t A = 32ull * cols.size();
  uint64_t k = (uint64_t)(frac * (double)A + 0.5);
  if (k > A) k = A;
  std::vector<uint64_t> perm(A);
  for (uint64_t i = 0; i < A; ++i) perm[i] = i;
  std::mt19937 g(seed);
  for (uint64_t i = 0; i < k; ++i) {
    std::swap(perm[i], perm[libcxx_uniform_int(g, i, A - 1)]);
    stim[cols[perm[i] / 32]] &= ~(1u << (perm[i] % 32));
  }
}

inline uint32_t noisy_seed(uint32_t q, uint32_t pct, uint32_t draw) { return 90000u + 1000u * pct + 16u * q + draw; }

}  // namespace oracle
