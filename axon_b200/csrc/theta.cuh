// Exact column-threshold selection shared by the plain and batched kernels.
#pragma once
#include <cstdint>

#include "axon_device.cuh"

namespace axon {

// The threads that run a threshold select together: the whole block (BlockGrp, synchronised
// by the block barrier), or a set of whole warps with a named barrier of its own (WarpGrp), so
// that several groups of one block can each select for a trajectory of their own at once.
struct BlockGrp {
  __device__ __forceinline__ uint32_t tid() const { return threadIdx.x; }
  __device__ __forceinline__ uint32_t n() const { return blockDim.x; }
  __device__ __forceinline__ void sync() const { __syncthreads(); }
};
struct WarpGrp {
  uint32_t t;    // thread index within the group
  uint32_t nt;   // threads in the group, a multiple of 32
  uint32_t bar;  // named barrier id, 1..15, used by this group alone
  __device__ __forceinline__ uint32_t tid() const { return t; }
  __device__ __forceinline__ uint32_t n() const { return nt; }
  __device__ __forceinline__ void sync() const { asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(nt) : "memory"); }
};

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
// Every thread of the group g calls it; sHist holds 256 words, sRed 192.
template <class G = BlockGrp>
static __device__ __noinline__ uint32_t block_theta(const uint32_t* sD, uint32_t incols, uint32_t ncol, uint32_t need,
                                                    uint32_t topkPar, uint32_t* sHist, uint32_t* sRed,
                                                    uint32_t hint, G g = G{}) {
  const uint32_t tid = g.tid(), lane = tid & 31u, warp = tid >> 5, nw = g.n() >> 5;
  const uint32_t h1 = max(hint, 1u), h2 = max(hint >> 1, 1u);
  // largest candidate, number of candidates, of positive candidates, and of candidates
  // reaching the hint and half the hint
  uint32_t mx = 0, cnt = 0, pos = 0, n1 = 0, n2 = 0;
  for (uint32_t c = incols + tid; c < ncol; c += g.n()) {
    const uint32_t d = sD[c];
    if (d < (1u << 24)) { mx = max(mx, d); ++cnt; pos += d != 0u; n1 += d >= h1; n2 += d >= h2; }
  }
  mx = __reduce_max_sync(kFull, mx);
  cnt = __reduce_add_sync(kFull, cnt);
  pos = __reduce_add_sync(kFull, pos);
  n1 = __reduce_add_sync(kFull, n1);
  n2 = __reduce_add_sync(kFull, n2);
  if (lane == 0) { sRed[warp] = mx; sRed[32 + warp] = cnt; sRed[64 + warp] = pos; sRed[128 + warp] = n1; sRed[160 + warp] = n2; }
  for (uint32_t i = tid; i < 256u; i += g.n()) sHist[i] = 0u;
  g.sync();
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
  if (need == 0u) { g.sync(); return topkPar ? 1u : 0xFFFFFFu; }
  if (count < need || npos < need) { g.sync(); return 1u; }

  // select the need-th largest x = d - lo over the candidates d in [lo, 2^24)
  const uint32_t nb = 32u - __clz(max(M - lo, 1u));
  uint32_t shift = nb > 8u ? nb - 8u : 0u, hiShift = 32u;
  uint32_t prefix = 0, rem = need;
  for (uint32_t pass = 0;; ++pass) {
    const uint32_t width = (hiShift >= 32u ? nb : hiShift) - shift;  // 1..8
    const uint32_t dmask = (1u << width) - 1u;
    // bins were cleared before the previous sync
    for (uint32_t c = incols + tid; c < ncol; c += g.n()) {
      const uint32_t d = sD[c];
      if (d < lo || d >= (1u << 24)) continue;
      const uint32_t x = d - lo;
      if (hiShift < 32u && (x >> hiShift) != (prefix >> hiShift)) continue;
      atomicAdd(&sHist[(x >> shift) & dmask], 1u);
    }
    g.sync();
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
    g.sync();
    prefix |= sRed[94] << shift;
    rem -= sRed[95];
    if (shift == 0u) break;
    hiShift = shift;
    shift = shift >= 8u ? shift - 8u : 0u;
  }
  g.sync();
  return max(prefix + lo, 1u);
}

// Bin of a column drive d < 2^24 in the threshold histogram: monotone in d, the drive
// itself below 64, and above that the octave with the five bits after the leading one
// (32 bins per octave, 640 bins in all). Bin k >= 64 holds the drives
// [(32 | (k & 31)) << b, ((32 | (k & 31)) + 1) << b) with b = (k >> 5) - 1.
__device__ __forceinline__ uint32_t theta_key(uint32_t d) {
  if (d < 64u) return d;
  const uint32_t e = 31u - __clz(d);  // 6..23
  return ((e - 4u) << 5) | ((d >> (e - 5u)) & 31u);
}

// The smallest drive of theta_key bin k.
__device__ __forceinline__ uint32_t theta_bin_lo(uint32_t k) { return k < 64u ? k : (32u | (k & 31u)) << ((k >> 5) - 1u); }

// The same threshold as block_theta (src/axon.mm:301-352 and :259-292) when every
// recurrent drive below 2^24 has been recorded in sH as it was published: per theta_key
// bin the count (sH[0, 640)), the largest drive (sH[640, 1280)) and the complement of the
// smallest (sH[1280, 1920)). Warp 0 scans the counts from the top to the bin that holds
// the need-th largest drive. That drive is the bin itself below 64, and the bin's largest
// or smallest drive when it ranks first or last in its bin; otherwise the block collects
// the bin's drives (usually a few) into sCand and warp 0 resolves the rank bit by bit, most
// significant first. sCtl[0] is the candidate counter and must be zero on entry;
// sCtl[2..5] is scratch. Every thread of the group g calls it. The histogram must be in shared
// memory on entry; the drives are read only after the scan, so with kDrivesGroup >= 0 they may
// still be arriving by asynchronous copy: each thread then waits until at most kDrivesGroup of
// its copy groups are pending before the group barrier that precedes the first read.
template <int kDrivesGroup = -1, class G = BlockGrp>
static __device__ __forceinline__ uint32_t hist_theta(const uint32_t* sD, const uint32_t* sH, uint32_t* sCand,
                                                   uint32_t* sCtl, uint32_t incols, uint32_t ncol, uint32_t need,
                                                   uint32_t topkPar, G g = G{}) {
  constexpr uint32_t kPer = 20;  // bins per lane (640 / 32)
  constexpr uint32_t kThetaBinCount = 32u * kPer;
  const uint32_t lane = g.tid() & 31u, warp = g.tid() >> 5;
  if (warp == 0u) {
    uint32_t h[kPer], ls = 0;
    const uint4* h4 = reinterpret_cast<const uint4*>(sH + lane * kPer);
#pragma unroll
    for (int i = 0; i < (int)kPer / 4; ++i) {
      const uint4 v = h4[i];
      h[4 * i] = v.x; h[4 * i + 1] = v.y; h[4 * i + 2] = v.z; h[4 * i + 3] = v.w;
      ls += v.x + v.y + v.z + v.w;
    }
    uint32_t S = ls;  // drives in the bins of this lane and the lanes above
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t v = __shfl_down_sync(kFull, S, off);
      if (lane + off < 32u) S += v;
    }
    const uint32_t count = __shfl_sync(kFull, S, 0), zeros = __shfl_sync(kFull, h[0], 0);
    uint32_t res = 0;  // the threshold when it is known without candidates (always >= 1), else 0
    uint32_t b = 0, above = 0, inBin = 0;
    if (need == 0u) {
      res = topkPar ? 1u : 0xFFFFFFu;
    } else if (count < need || count - zeros < need) {
      res = 1u;
    } else {
      uint32_t Snext = __shfl_down_sync(kFull, S, 1);
      if (lane == 31u) Snext = 0u;
      const bool mine = S >= need && Snext < need;
      if (mine) {
        uint32_t cum = Snext;
#pragma unroll
        for (int i = (int)kPer - 1; i >= 0; --i) {
          if (cum + h[i] >= need) { b = lane * kPer + (uint32_t)i; above = cum; inBin = h[i]; break; }
          cum += h[i];
        }
      }
      const uint32_t src = (uint32_t)__ffs(__ballot_sync(kFull, mine)) - 1u;
      b = __shfl_sync(kFull, b, src);
      above = __shfl_sync(kFull, above, src);
      inBin = __shfl_sync(kFull, inBin, src);
      if (b < 64u) res = b;  // one drive per bin; b >= 1 because at least `need` drives are positive
      else if (need - above == 1u) res = sH[kThetaBinCount + b];
      else if (need - above == inBin) res = ~sH[2u * kThetaBinCount + b];
    }
    if (lane == 0u) { sCtl[2] = res; sCtl[3] = b; sCtl[4] = need - above; sCtl[5] = inBin; }
  }
  if constexpr (kDrivesGroup >= 0) cp_async_wait<kDrivesGroup>();
  g.sync();
  const uint32_t res = sCtl[2];
  if (res != 0u) return res;
  const uint32_t b = sCtl[3];
  const uint32_t bits = (b >> 5) - 1u, lo = (32u | (b & 31u)) << bits;
  for (uint32_t c = incols + g.tid(); c < ncol; c += g.n()) {
    const uint32_t d = sD[c];
    if (d < (1u << 24) && theta_key(d) == b) sCand[atomicAdd(sCtl, 1u)] = d - lo;
  }
  g.sync();
  if (warp == 0u) {
    uint32_t rem = sCtl[4];  // rank of the answer among the drives of bin b, from the top
    const uint32_t inBin = sCtl[5];
    uint32_t prefix = 0;
    if (inBin <= 64u) {
      const bool v0 = lane < inBin, v1 = lane + 32u < inBin;
      const uint32_t x0 = v0 ? sCand[lane] : 0u, x1 = v1 ? sCand[lane + 32u] : 0u;
      for (int bit = (int)bits - 1; bit >= 0; --bit) {
        const uint32_t want = (prefix >> bit) | 1u;
        const uint32_t c1 = (uint32_t)__popc(__ballot_sync(kFull, v0 && (x0 >> bit) == want)) +
                            (uint32_t)__popc(__ballot_sync(kFull, v1 && (x1 >> bit) == want));
        if (c1 >= rem) prefix |= 1u << bit; else rem -= c1;
      }
    } else {
      for (int bit = (int)bits - 1; bit >= 0; --bit) {
        const uint32_t want = (prefix >> bit) | 1u;
        uint32_t c1 = 0;
        for (uint32_t i = lane; i < inBin; i += 32u) c1 += (sCand[i] >> bit) == want;
        c1 = __reduce_add_sync(kFull, c1);
        if (c1 >= rem) prefix |= 1u << bit; else rem -= c1;
      }
    }
    if (lane == 0u) sCtl[2] = lo + prefix;
  }
  g.sync();
  return sCtl[2];
}

}  // namespace axon
