// Exact column-threshold selection shared by the plain and batched kernels.
#pragma once
#include <cstdint>

#include "axon_device.cuh"

namespace axon {

// Exact selection of the column threshold over recurrent columns [incols, ncol),
// src/axon.mm:301-352 (k_topk_par, default) and :259-292 (k_topk_serial). Both return
// max(v, 1) where v is the need-th largest drive among drives below 2^24 when at least
// `need` such drives exist and need >= 1; with fewer candidates both give 1; with
// need == 0 the parallel form gives 1 and the serial form 0xFFFFFF. The selection here is
// a radix select over the significant bits of the largest candidate; any digit split
// yields the same order statistic.
static __device__ __noinline__ uint32_t block_theta(const uint32_t* sD, uint32_t incols, uint32_t ncol, uint32_t need,
                                       uint32_t topkPar, uint32_t* sHist, uint32_t* sRed) {
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nw = blockDim.x >> 5;
  // block max and count of candidates
  uint32_t mx = 0, cnt = 0;
  for (uint32_t c = incols + tid; c < ncol; c += blockDim.x) {
    const uint32_t d = sD[c];
    if (d < (1u << 24)) { mx = max(mx, d); ++cnt; }
  }
  mx = __reduce_max_sync(kFull, mx);
  cnt = __reduce_add_sync(kFull, cnt);
  if (lane == 0) { sRed[warp] = mx; sRed[32 + warp] = cnt; }
  __syncthreads();
  if (warp == 0) {
    uint32_t m = lane < nw ? sRed[lane] : 0u, n = lane < nw ? sRed[32 + lane] : 0u;
    m = __reduce_max_sync(kFull, m);
    n = __reduce_add_sync(kFull, n);
    if (lane == 0) { sRed[64] = m; sRed[65] = n; }
  }
  __syncthreads();
  const uint32_t M = sRed[64], count = sRed[65];
  if (need == 0u) return topkPar ? 1u : 0xFFFFFFu;
  if (count < need || M == 0u) return 1u;

  const uint32_t nb = 32u - __clz(M);
  uint32_t shift = nb > 8u ? nb - 8u : 0u, hiShift = 32u;
  uint32_t prefix = 0, rem = need;
  const uint32_t iters = (ncol - incols + blockDim.x - 1) / blockDim.x;
  for (;;) {
    for (uint32_t i = tid; i < 256u; i += blockDim.x) sHist[i] = 0u;
    __syncthreads();
    const uint32_t width = (hiShift >= 32u ? nb : hiShift) - shift;  // <= 8
    const uint32_t dmask = (width >= 32u) ? kFull : ((1u << width) - 1u);
    for (uint32_t it = 0; it < iters; ++it) {
      const uint32_t c = incols + tid + it * blockDim.x;
      uint32_t key = kFull;
      if (c < ncol) {
        const uint32_t d = sD[c];
        const bool match = hiShift >= 32u || (d >> hiShift) == (prefix >> hiShift);
        if (d < (1u << 24) && match) key = (d >> shift) & dmask;
      }
      const uint32_t peers = __match_any_sync(kFull, key);
      if (key != kFull && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&sHist[key], (uint32_t)__popc(peers));
    }
    __syncthreads();
    if (warp == 0) {
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
        sRed[66] = b;
        sRed[67] = above;
      }
    }
    __syncthreads();
    prefix |= sRed[66] << shift;
    rem -= sRed[67];
    __syncthreads();  // sRed reused next pass
    if (shift == 0u) break;
    hiShift = shift;
    shift = shift >= 8u ? shift - 8u : 0u;
  }
  return max(prefix, 1u);
}

}  // namespace axon
