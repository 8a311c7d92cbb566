// Exact column-threshold selection shared by the plain and batched kernels.
#pragma once
#include <cstdint>

#include "axon_device.cuh"

namespace axon {

// Exact selection of the column threshold over recurrent columns [incols, ncol),
// src/axon.mm:301-352 (k_topk_par, default) and :259-292 (k_topk_serial). Both return
// max(v, 1) where v is the need-th largest drive among drives below 2^24 when at least
// `need` such drives exist and need >= 1; with fewer candidates both give 1; with
// need == 0 the parallel form gives 1 and the serial form 0xFFFFFF.
//
// Method: a radix select over the significant bits of the largest candidate, most
// significant digit first, digits of at most 8 bits (two passes for drives below 2^16).
// A pass histograms the candidates that share the prefix selected so far with plain
// shared-memory atomics, then one warp locates the bin where the count from the top
// reaches the remaining rank. Zero drives are left out whenever at least `need` drives
// are positive (they cannot be the answer then); otherwise the answer is 0 and the
// threshold 1. `hint` is a guess of the answer (the previous step's threshold; 0 for
// none): when at least `need` drives reach it (or half of it), only those drives take part,
// which keeps the histogram small. The result does not depend on the hint.
// Every thread of the block calls it; sHist holds 256 words, sRed 96.
static __device__ __noinline__ uint32_t block_theta(const uint32_t* sD, uint32_t incols, uint32_t ncol, uint32_t need,
                                                    uint32_t topkPar, uint32_t* sHist, uint32_t* sRed,
                                                    uint32_t hint) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nw = blockDim.x >> 5;
  const uint32_t h1 = max(hint, 1u), h2 = max(hint >> 1, 1u);
  // largest candidate, number of candidates, of positive candidates, and of candidates
  // reaching the hint and half the hint
  uint32_t mx = 0, cnt = 0, pos = 0, n1 = 0, n2 = 0;
  for (uint32_t c = incols + tid; c < ncol; c += blockDim.x) {
    const uint32_t d = sD[c];
    if (d < (1u << 24)) { mx = max(mx, d); ++cnt; pos += d != 0u; n1 += d >= h1; n2 += d >= h2; }
  }
  mx = __reduce_max_sync(kFull, mx);
  cnt = __reduce_add_sync(kFull, cnt);
  pos = __reduce_add_sync(kFull, pos);
  n1 = __reduce_add_sync(kFull, n1);
  n2 = __reduce_add_sync(kFull, n2);
  if (lane == 0) { sRed[warp] = mx; sRed[32 + warp] = cnt; sRed[64 + warp] = pos; sRed[128 + warp] = n1; sRed[160 + warp] = n2; }
  for (uint32_t i = tid; i < 256u; i += blockDim.x) sHist[i] = 0u;
  __syncthreads();
  uint32_t M, count, npos, lo;
  {
    const bool v = lane < nw;
    M = __reduce_max_sync(kFull, v ? sRed[lane] : 0u);
    count = __reduce_add_sync(kFull, v ? sRed[32 + lane] : 0u);
    npos = __reduce_add_sync(kFull, v ? sRed[64 + lane] : 0u);
    const uint32_t c1 = __reduce_add_sync(kFull, v ? sRed[128 + lane] : 0u);
    const uint32_t c2 = __reduce_add_sync(kFull, v ? sRed[160 + lane] : 0u);
    lo = c1 >= need ? h1 : (c2 >= need ? h2 : 1u);  // every drive below lo ranks below the answer
  }
  if (need == 0u) { __syncthreads(); return topkPar ? 1u : 0xFFFFFFu; }
  if (count < need || npos < need) { __syncthreads(); return 1u; }

  // select the need-th largest x = d - lo over the candidates d in [lo, 2^24)
  const uint32_t nb = 32u - __clz(max(M - lo, 1u));
  uint32_t shift = nb > 8u ? nb - 8u : 0u, hiShift = 32u;
  uint32_t prefix = 0, rem = need;
  for (uint32_t pass = 0;; ++pass) {
    const uint32_t width = (hiShift >= 32u ? nb : hiShift) - shift;  // 1..8
    const uint32_t dmask = (1u << width) - 1u;
    // bins were cleared before the previous sync
    for (uint32_t c = incols + tid; c < ncol; c += blockDim.x) {
      const uint32_t d = sD[c];
      if (d < lo || d >= (1u << 24)) continue;
      const uint32_t x = d - lo;
      if (hiShift < 32u && (x >> hiShift) != (prefix >> hiShift)) continue;
      atomicAdd(&sHist[(x >> shift) & dmask], 1u);
    }
    __syncthreads();
    if (warp == 0) {  // bin where the count from the top reaches rem; then clear the bins
      uint32_t h[8], ls = 0;
#pragma unroll
      for (int i = 0; i < 8; ++i) { h[i] = sHist[lane * 8 + i]; ls += h[i]; }
      uint32_t S = ls;  // inclusive suffix sum over lanes
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t v = __shfl_down_sync(kFull, S, off);
        if (lane + off < 32u) S += v;
      }
      uint32_t Snext = __shfl_down_sync(kFull, S, 1);
      if (lane == 31u) Snext = 0u;
      if (S >= rem && Snext < rem) {
        uint32_t cum = Snext, b = lane * 8u, above = Snext;
#pragma unroll
        for (int i = 7; i >= 0; --i) {
          if (cum + h[i] >= rem) { b = lane * 8u + i; above = cum; break; }
          cum += h[i];
        }
        sRed[94] = b;
        sRed[95] = above;
      }
      __syncwarp();
#pragma unroll
      for (int i = 0; i < 8; ++i) sHist[lane * 8 + i] = 0u;
    }
    __syncthreads();
    prefix |= sRed[94] << shift;
    rem -= sRed[95];
    if (shift == 0u) break;
    hiShift = shift;
    shift = shift >= 8u ? shift - 8u : 0u;
  }
  __syncthreads();
  return max(prefix + lo, 1u);
}

}  // namespace axon
