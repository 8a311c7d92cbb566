// Set algebra of the AXON readouts on sorted column / neuron id lists, as the reference's
// host code computes its measurements (src/axon.mm:896-901 and the blocks that use it).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <iterator>
#include <vector>

namespace axon {

using Ids = std::vector<uint32_t>;  // sorted column or neuron ids

inline Ids active_columns(const uint32_t* spk, uint32_t incols, uint32_t ncol) {
  Ids v;
  for (uint32_t c = incols; c < ncol; ++c)
    if (spk[c]) v.push_back(c);
  return v;
}
inline Ids active_neurons(const uint32_t* spk, uint32_t incols, uint32_t ncol) {
  Ids v;
  for (uint32_t c = incols; c < ncol; ++c)
    for (uint32_t b = spk[c]; b; b &= b - 1) v.push_back(c * 32u + (uint32_t)__builtin_ctz(b));  // 32 neurons per column
  return v;
}
inline size_t n_common(const Ids& a, const Ids& b) {
  size_t i = 0, j = 0, k = 0;
  while (i < a.size() && j < b.size()) {
    if (a[i] < b[j]) ++i;
    else if (b[j] < a[i]) ++j;
    else { ++k; ++i; ++j; }
  }
  return k;
}
inline Ids common(const Ids& a, const Ids& b) {
  Ids r;
  std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(r));
  return r;
}
inline Ids minus(const Ids& a, const Ids& b) {
  Ids r;
  std::set_difference(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(r));
  return r;
}
// cosine overlap |A n B| / sqrt(|A||B|), 0 for an empty set (src/axon.mm:896-901)
inline double cos_overlap(const Ids& a, const Ids& b) {
  if (a.empty() || b.empty()) return 0.0;
  return (double)n_common(a, b) / std::sqrt((double)a.size() * b.size());
}
inline double jaccard(const Ids& a, const Ids& b) {
  if (a.empty() || b.empty()) return 0.0;
  const size_t i = n_common(a, b);
  return (double)i / (double)(a.size() + b.size() - i);
}
inline void dedup(Ids& v) {
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
}

}  // namespace axon
