// Host-side stimulus stream of the AXON protocol.
//
// rakib-nyc/axon draws its input patterns with std::mt19937 + std::shuffle and its cue
// masks with std::uniform_real_distribution<double> (src/axon.mm:793-804), compiled
// against Apple libc++. Only mt19937 is pinned by the C++ standard; the other two are
// implementation-defined, so this file implements libc++'s algorithms explicitly and
// the stream is the same on any host library:
//   shuffle        forward Fisher-Yates, element i swapped with i + U[0, n-1-i]
//   U[0, r-1]      the low ceil(log2 r) bits of one mt19937 word, redrawn while >= r
//   uniform [0,1)  (w1 + w2 * 2^32) / 2^64 from two consecutive words
#pragma once
#include <cstdint>
#include <random>
#include <vector>

namespace axon {

class StimulusRng {
 public:
  explicit StimulusRng(uint32_t seed) : mt_(seed) {}

  uint64_t below(uint64_t range) {  // uniform in [0, range), range >= 1
    if (range <= 1) return 0;
    unsigned bits = 64u - (unsigned)__builtin_clzll(range - 1);  // ceil(log2(range))
    const uint64_t mask = (bits >= 64) ? ~0ull : ((1ull << bits) - 1);
    for (;;) {
      const uint64_t v = (uint64_t)(uint32_t)mt_() & mask;
      if (v < range) return v;
    }
  }
  double unit() {
    const double lo = (double)(uint32_t)mt_();
    const double hi = (double)(uint32_t)mt_();
    return (lo + hi * 4294967296.0) * (1.0 / 18446744073709551616.0);
  }
  template <class T>
  void shuffle(std::vector<T>& v) {
    const size_t n = v.size();
    for (size_t i = 0; i + 1 < n; ++i) {
      const size_t j = i + (size_t)below(n - i);
      if (j != i) std::swap(v[i], v[j]);
    }
  }

 private:
  std::mt19937 mt_;
};

// NSTIM patterns of STIM_COLS input columns each (src/axon.mm:793-799)
inline std::vector<std::vector<uint32_t>> make_patterns(uint32_t seed, uint32_t nstim, uint32_t incols,
                                                        uint32_t stimcols) {
  StimulusRng rng(7u + seed * 104729u);
  std::vector<std::vector<uint32_t>> pats(nstim);
  std::vector<uint32_t> order(incols);
  for (auto& p : pats) {
    for (uint32_t i = 0; i < incols; ++i) order[i] = i;
    rng.shuffle(order);
    p.assign(order.begin(), order.begin() + stimcols);
  }
  return pats;
}

// Clamp words for one presentation: each pattern column is kept with probability `keep`,
// tested in pattern order (src/axon.mm:800-804).
inline void make_clamp(const std::vector<uint32_t>& pattern, double keep, uint32_t seed, uint32_t ncol, uint32_t* out) {
  for (uint32_t c = 0; c < ncol; ++c) out[c] = 0u;
  StimulusRng rng(seed);
  for (uint32_t c : pattern)
    if (rng.unit() <= keep) out[c] = 0xFFFFFFFFu;
}

// Noisy cue: the clamp words of the whole pattern (every pattern column on), then
// round(frac * A) of its A = 32 * pattern.size() active bits flipped off. The active bits
// are listed column by column in pattern order, bit 0 first; the flipped ones are the
// first picks of a forward Fisher-Yates over that list driven by mt19937(seed), each pick
// i + U[0, A-1-i] drawn as the shuffle above draws (so the picks for a smaller fraction
// are the first picks for a larger one with the same seed). Pattern columns must be
// distinct and below ncol.
inline void make_noisy_clamp(const std::vector<uint32_t>& pattern, double frac, uint32_t seed, uint32_t ncol,
                             uint32_t* out) {
  for (uint32_t c = 0; c < ncol; ++c) out[c] = 0u;
  for (uint32_t c : pattern) out[c] = 0xFFFFFFFFu;
  const uint64_t A = 32ull * pattern.size();
  uint64_t nflip = (uint64_t)(frac * (double)A + 0.5);
  if (nflip > A) nflip = A;
  std::vector<uint32_t> idx(A);
  for (uint64_t i = 0; i < A; ++i) idx[i] = (uint32_t)i;
  StimulusRng rng(seed);
  for (uint64_t i = 0; i < nflip; ++i) {
    const uint64_t j = i + rng.below(A - i);
    std::swap(idx[i], idx[j]);
    out[pattern[idx[i] >> 5]] &= ~(1u << (idx[i] & 31u));
  }
}

// Seed of noisy-cue draw `draw` of pattern q at `pct` percent of active bits flipped.
inline uint32_t noisy_cue_seed(uint32_t q, uint32_t pct, uint32_t draw) { return 90000u + 1000u * pct + 16u * q + draw; }

}  // namespace axon
