// Batched recall: B trajectories of one trained network share every read of W3.
//
// Readout presentations of rakib-nyc/axon (present() with learn=false, src/axon.mm:815-888)
// change no weight, so any number of them can run together. One cooperative launch runs
// T steps for all B trajectories, two grid barriers per step.
//
//   phase 2 (end of step t-1) publishes, for every presynaptic group g, the list of
//            trajectories in which g spiked, each entry carrying that trajectory's nonzero
//            spike words of g (one 16-byte record; most groups have one or two).
//   phase 1  work items are pairs of columns, claimed dynamically. The item's 64 W3 tiles
//            (64 KiB, laid out [branch][row][word]) arrive by bulk TMA copies into shared
//            memory, double-buffered so the next item loads while this one computes. The
//            item's (branch, entry) pairs are flattened and dealt 32 per warp, one per lane:
//            a lane pops AND-counts of its entry's words against all 32 rows of the tile
//            and adds the dendritic terms into per-(trajectory, neuron) counters in shared
//            memory (two 16-bit sums per 32-bit atomic). Silent (branch, trajectory) pairs
//            cost nothing. The counters then become the per-neuron and column drives, and
//            the write-back that reads them clears them. One CTA barrier per item separates
//            its units from its write-back; with two counter buffers nothing else does.
//            The write-back also counts every recurrent column drive at or above the
//            trajectory's floor into its drive histogram for the step (count, largest and
//            smallest drive per bin), and stores the per-neuron drives of those columns.
//   phase 2  per trajectory, by groups of warps that each take trajectories of their own:
//            the column threshold from that histogram (hist_theta, or a sorting select when
//            too few drives reached the floor), the exact k-of-32 ballot only for columns
//            that pass the gate, the new spike vector, and its group lists. The tiles of
//            the next step's first item are requested before the grid barrier.
#include <cstdint>

#include "axon_device.cuh"
#include "batch.cuh"
#include "batch_common.cuh"
#include "plain.cuh"
#include "theta.cuh"

namespace axon {

__global__ void k_make_w3r(const uint4* __restrict__ W3, uint32_t* __restrict__ W3R, uint64_t ntile) {
  // one thread per (tile, row): scatters the row's 8 words
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ntile * 32) return;
  const uint64_t tile = i >> 5;
  const uint32_t row = (uint32_t)(i & 31u);
  const uint4 a = W3[tile * kTileU4 + row], b = W3[tile * kTileU4 + 32 + row];
  uint32_t* o = W3R + tile * 256;
  o[w3r_pos(row, 0)] = a.x; o[w3r_pos(row, 1)] = a.y; o[w3r_pos(row, 2)] = a.z; o[w3r_pos(row, 3)] = a.w;
  o[w3r_pos(row, 4)] = b.x; o[w3r_pos(row, 5)] = b.y; o[w3r_pos(row, 6)] = b.z; o[w3r_pos(row, 7)] = b.w;
}

cudaError_t launch_make_w3r(const uint4* W3, uint32_t* W3R, uint32_t ncol, cudaStream_t st) {
  const uint64_t ntile = (uint64_t)ncol * kNslot;
  k_make_w3r<<<(unsigned)((ntile * 32 + 255) / 256), 256, 0, st>>>(W3, W3R, ntile);
  return cudaGetLastError();
}

// Row rr (= column-in-item * B + trajectory) of a counter buffer. Packed rows are 16 words
// (32 neurons in 16-bit pairs) at a stride of 17 (32-bit rows at 33): the odd stride
// spreads the rows of different trajectories over all 32 banks. (Rows aligned to even words
// for 8-byte accesses leave only 16 starting banks: measured slower, as was adding four rows
// by one 64-bit shared atomic, 9.76 ms per benchmark batch against 7.01 ms.)
template <bool PACK>
__device__ __forceinline__ uint32_t* acc_row(uint32_t* accB, uint32_t rr) {
  return accB + rr * (PACK ? 17u : 33u);
}

// One m16n8k256 binary MMA: d = c + popcount(a AND b) over 256 bits, a 16 x 256 bit rows
// (row-major fragment), b 256 x 8 bit columns, c/d 16 x 8 int32.
__device__ __forceinline__ void mma_b1_and(uint32_t (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k256.row.col.s32.b1.b1.s32.and.popc {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Phase-1 entry units of one work item on the tensor cores. A unit is a chunk of 8 entries
// of one branch (the branch's single-word entries first, then its multi-word ones); the
// warp's lanes hold the fragments of m16n8k256: lane = 4 * g + q holds rows g, g+8 (and
// g+16, g+24 in the second MMA) of the tile at 32-bit words q and q+4, and entry g's spike
// words q and q+4. The counts come back as rows g, g+8 for entries 2q, 2q+1; each count
// becomes its dendritic term and is added into the entry's trajectory row, packed in pairs
// of rows with the lane that holds the neighbouring row (lane ^ 4).
template <bool PACK, bool LIN>
__device__ __forceinline__ void mma_units(const uint32_t* cPC, const uint32_t* cP1, const uint32_t* cPM,
                                          const uint32_t* cConn, const uint32_t* tileBase, uint32_t* accB,
                                          uint32_t accStride, uint32_t* unitCtr, const uint2* e1In, const uint4* eMIn,
                                          const uint32_t* spkIn, uint32_t B, uint32_t ncol, uint32_t dthr,
                                          uint32_t bst, uint32_t lane) {
  const uint32_t nchunks = cPC[64];
  const uint32_t g4 = lane >> 2, q = lane & 3u;
  constexpr uint32_t kNone = 0xFFFFFFFFu;
  for (;;) {
    uint32_t u = 0;
    if (lane == 0) u = atomicAdd(unitCtr, 1u);
    u = __shfl_sync(kFull, u, 0);
    if (u >= nchunks) break;
    // the chunk's branch: how many branches end at or before chunk u
    const uint32_t sp = (uint32_t)__popc(__ballot_sync(kFull, cPC[lane + 1] <= u)) +
                        (uint32_t)__popc(__ballot_sync(kFull, cPC[lane + 33] <= u));
    const uint32_t G = cConn[sp];
    const uint32_t n1 = cP1[sp + 1] - cP1[sp], nE = n1 + (cPM[sp + 1] - cPM[sp]);
    const uint32_t e = 8u * (u - cPC[sp]) + g4;
    uint32_t bq = kNone, b0 = 0u, b1 = 0u;
    if (e < n1) {
      const uint2 en = __ldcg(e1In + (size_t)G * B + e);
      const uint32_t w = en.x >> 16;
      bq = en.x & 0xFFFFu;
      b0 = w == q ? en.y : 0u;
      b1 = w == q + 4u ? en.y : 0u;
    } else if (e < nE) {
      const uint4 en = __ldcg(eMIn + (size_t)G * B + (e - n1));
      const uint32_t nz = (en.x >> 16) & 0xFFu;
      bq = en.x & 0xFFFFu;
      const uint32_t* sw = spkIn + (size_t)bq * ncol + 8u * G;
      b0 = ((nz >> q) & 1u) ? __ldcg(sw + q) : 0u;
      b1 = ((nz >> (q + 4u)) & 1u) ? __ldcg(sw + q + 4u) : 0u;
    }
    const uint32_t* tile = tileBase + (sp >> 5) * kColWords + (sp & 31u) * 256u;
    uint32_t a[4], a2[4], c0[4] = {0u, 0u, 0u, 0u}, c1[4] = {0u, 0u, 0u, 0u};
    a[0] = tile[w3r_pos(g4, q)];
    a[1] = tile[w3r_pos(g4 + 8u, q)];
    a[2] = tile[w3r_pos(g4, q + 4u)];
    a[3] = tile[w3r_pos(g4 + 8u, q + 4u)];
    a2[0] = tile[w3r_pos(g4 + 16u, q)];
    a2[1] = tile[w3r_pos(g4 + 24u, q)];
    a2[2] = tile[w3r_pos(g4 + 16u, q + 4u)];
    a2[3] = tile[w3r_pos(g4 + 24u, q + 4u)];
    __syncwarp();
    mma_b1_and(c0, a, b0, b1);
    mma_b1_and(c1, a2, b0, b1);
    // the trajectories of entries 2q and 2q+1 (held by lanes 8q and 8q + 4)
    const uint32_t bA = __shfl_sync(kFull, bq, 8u * q), bB = __shfl_sync(kFull, bq, 8u * q + 4u);
    // counts by row block k (rows g4 + 8k): cA for entry 2q, cB for entry 2q+1
    const uint32_t cA[4] = {c0[0], c0[2], c1[0], c1[2]}, cB[4] = {c0[1], c0[3], c1[1], c1[3]};
    uint32_t* rowA = bA != kNone ? acc_row<PACK>(accB, (sp >> 5) * B + bA) : nullptr;
    uint32_t* rowB = bB != kNone ? acc_row<PACK>(accB, (sp >> 5) * B + bB) : nullptr;
    if (PACK) {
      // rows g4 and g4 ^ 1 share a counter word: the even lane adds entry 2q's pair, the odd
      // lane entry 2q+1's; both terms of a word at once (see acc_add4c)
      const bool ev = (g4 & 1u) == 0u;
      const uint32_t kk = (0x8000u - min(dthr, 0x8000u)) * 0x00010001u;
      uint32_t* row = ev ? rowA : rowB;
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k) {
        const uint32_t x = __shfl_xor_sync(kFull, ev ? cB[k] : cA[k], 4);
        const uint32_t P = ev ? (cA[k] | (x << 16)) : (x | (cB[k] << 16));
        const uint32_t N = ((P + kk) >> 15) & 0x00010001u;
        if (row) atomicAdd(row + (((g4 & ~1u) + 8u * k) >> 1), LIN ? P + bst * N : N);
      }
    } else {
#pragma unroll
      for (uint32_t k = 0; k < 4; ++k) {
        if (rowA) atomicAdd(rowA + g4 + 8u * k, branch_term<LIN>(cA[k], dthr, bst));
        if (rowB) atomicAdd(rowB + g4 + 8u * k, branch_term<LIN>(cB[k], dthr, bst));
      }
    }
  }
}

// The smallest drive a trajectory's histogram records in a step: the lower edge of the bin
// of half the threshold of its previous step (at least 1), so every bin is recorded whole or
// not at all. The threshold is the target-th largest recurrent drive, so when at least
// `target` drives reach the floor the histogram holds every drive that can be the answer,
// and each of their bins completely; otherwise phase 2 falls back to sorting all drives.
// Counting only these columns keeps the write-back's atomics few and off the crowded low
// bins.
__device__ __forceinline__ uint32_t hist_floor(const uint32_t* thPrev) {
  return theta_bin_lo(theta_key(min(max(__ldcg(thPrev) >> 1, 1u), (1u << 24) - 1u)));
}

// One recurrent column drive into a threshold histogram (theta_key bins: count, largest
// drive, complement of the smallest), as the plain path's phase A counts them.
__device__ __forceinline__ void count_drive(uint32_t* h, uint32_t drv) {
  if (drv >= (1u << 24)) return;  // never a threshold candidate (src/axon.mm:276)
  h += theta_key(drv);
  atomicAdd(h, 1u);
  atomicMax(h + kThetaBins, drv);
  atomicMax(h + 2u * kThetaBins, ~drv);
}

// The threshold select of phase 2, kept out of line so that its registers do not add to
// phase 1's.
static __device__ __noinline__ uint32_t recall_theta(const uint32_t* sD, const uint32_t* sH, uint32_t* sCand,
                                                     uint32_t* sCtl, uint32_t incols, uint32_t ncol, uint32_t need,
                                                     uint32_t topkPar, WarpGrp g) {
  return hist_theta<-1>(sD, sH, sCand, sCtl, incols, ncol, need, topkPar, g);
}

// The per-neuron drives of column cc for one trajectory, recomputed from that trajectory's
// spike vector of the previous step (spkB, ncol words), for a gated column whose entry the
// write-back did not store. Lane = branch: its group's nonzero spike words AND-counted
// against the branch's 32 tile rows give its 32 dendritic terms, none for a silent group
// (src/axon.mm:166-178, the terms the phase-1 units add); the lanes add them into the
// warp's 32 row sums in shared memory (scr, zero on entry and on return), and lane r
// returns neuron r's drive. Loops over rows are not unrolled: the path is rare, and its
// registers count against the whole kernel's.
template <bool LIN>
__device__ __forceinline__ uint32_t recompute_drive(const uint32_t* W3R, const uint32_t* conn, const uint32_t* spkB,
                                                    uint32_t cc, uint32_t dthr, uint32_t bst, uint32_t lane,
                                                    uint32_t* scr) {
  const uint32_t g = __ldg(conn + cc * kNslot + lane);
  const uint4 p = __ldcg(reinterpret_cast<const uint4*>(spkB + 8u * g));
  const uint4 q = __ldcg(reinterpret_cast<const uint4*>(spkB + 8u * g) + 1);
  const uint32_t S[8] = {p.x, p.y, p.z, p.w, q.x, q.y, q.z, q.w};
  if ((p.x | p.y | p.z | p.w | q.x | q.y | q.z | q.w) != 0u) {
    const uint32_t* tile = W3R + (size_t)cc * kColWords + lane * 256u;
#pragma unroll 1
    for (uint32_t r = 0; r < 32u; r += 4) {
      uint32_t c0 = 0u, c1 = 0u, c2 = 0u, c3 = 0u;
#pragma unroll
      for (uint32_t w = 0; w < 8u; ++w) {
        if (S[w] == 0u) continue;
        const uint4 a = __ldg(reinterpret_cast<const uint4*>(tile + w3r_pos(r, w)));
        c0 += __popc(a.x & S[w]); c1 += __popc(a.y & S[w]);
        c2 += __popc(a.z & S[w]); c3 += __popc(a.w & S[w]);
      }
      atomicAdd(scr + r, branch_term<LIN>(c0, dthr, bst));
      atomicAdd(scr + r + 1u, branch_term<LIN>(c1, dthr, bst));
      atomicAdd(scr + r + 2u, branch_term<LIN>(c2, dthr, bst));
      atomicAdd(scr + r + 3u, branch_term<LIN>(c3, dthr, bst));
    }
  }
  __syncwarp();
  const uint32_t a = scr[lane];
  scr[lane] = 0u;
  __syncwarp();
  return a;
}

// MMA: the AND-popcount contraction of phase 1 on the tensor cores (mma.sync b1 and.popc,
// m16n8k256: 16 tile rows x 8 entries x the group's 256 spike bits per instruction) instead
// of __popc on the CUDA cores; the dendritic terms, counters and everything else are shared.
template <bool PACK, bool LIN, bool MMA>
__global__ void __launch_bounds__(896, 1) k_recall(RecallDev d, RecallCfg c) {
  extern __shared__ __align__(128) uint32_t sm[];
  const uint32_t ncol = c.ncol, incols = c.incols, B = c.B, ngrp = ncol / 8u;
  const uint32_t dthr = c.dthr, bst = c.bst;
  constexpr uint32_t accStride = PACK ? 17u : 33u;  // padded: distinct trajectories hit distinct banks
  uint32_t* sTile = sm;                                  // [2][kItemWords]
  const uint32_t accWords = kRecallCpi * B * accStride;
  uint32_t* sAcc = sTile + 2 * kItemWords;               // [1 or 2][kRecallCpi][B][accStride]
  uint32_t* sConn = sAcc + (c.dacc ? 2u : 1u) * accWords;  // [2][64] groups of the item's branches
  uint32_t* sP1 = sConn + 2 * 64;                        // [2][68] single-word entries: prefix over 64 branches
  uint32_t* sPM = sP1 + 2 * 68;                          // [2][68] multi-word entries
  uint32_t* sPC = sPM + 2 * 68;                          // [2][68] MMA: chunks of 8 entries, prefix over branches
  uint32_t* sMisc = sPC + 2 * 68;  // [16]: grid barrier flag, first item, -, -, -, -, unit counters [2], next items [2]
  uint64_t* sBar = reinterpret_cast<uint64_t*>(sMisc + 16);  // [2]
  uint32_t* sFloor = sMisc + 20;  // [B] each trajectory's histogram floor for this step
  uint32_t* sUT = sFloor + B;     // [2][kUnitTab] first branch of each list per unit (prep)

  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nw = blockDim.x >> 5;
  const uint32_t nitems = (ncol + kRecallCpi - 1) / kRecallCpi;
  if (tid == 0) {
    mbar_init(&sBar[0], 1);
    mbar_init(&sBar[1], 1);
    fence_proxy_async_smem();
  }
  // the counters start at zero; each item's write-back clears what it read
  for (uint32_t i = tid; i < (c.dacc ? 2u : 1u) * accWords; i += blockDim.x) sAcc[i] = 0u;
  __syncthreads();
  uint32_t uses0 = 0, uses1 = 0;  // completed phases per buffer
  uint32_t kbuf = 0;              // buffer of the next item
  uint32_t epoch = 0;
  uint32_t claim = 0;             // thread 0: the item claimed one ahead
  bool pre = false;               // the step's first item was claimed and its tiles issued already

  auto issue = [&](uint32_t item, uint32_t buf) {  // thread 0 only
    const uint32_t c0 = item * kRecallCpi;
    const uint32_t ncols = min(kRecallCpi, ncol - c0);
    fence_proxy_async_smem();
    mbar_expect_tx(&sBar[buf], ncols * kColWords * 4u);
    for (uint32_t k = 0; k < ncols; ++k)
      bulk_g2s(sTile + buf * kItemWords + k * kColWords, d.W3R + (size_t)(c0 + k) * kColWords, kColWords * 4u, &sBar[buf]);
  };
  // warp 0: the item's branch groups and the prefixes of its 64 entry-list lengths, single-
  // word and multi-word, into buffer buf
  // groups below skipGroups contribute nothing this step: their entries are left out (the
  // clamped input groups while their contribution comes from the afferent cache)
  uint32_t skipGroups = 0;
  auto prep = [&](uint32_t item, uint32_t buf, const uint32_t* c1In, const uint32_t* cMIn) {
    const uint32_t c0 = item * kRecallCpi;
    const bool v1 = c0 + 1 < ncol;
    const uint32_t g0 = __ldg(d.conn + c0 * kNslot + lane), g1 = v1 ? __ldg(d.conn + (c0 + 1) * kNslot + lane) : 0u;
    sConn[buf * 64u + lane] = g0;
    sConn[buf * 64u + 32u + lane] = g1;
    const bool u0 = g0 >= skipGroups, u1 = v1 && g1 >= skipGroups;
    uint32_t a0 = u0 ? __ldcg(c1In + g0) : 0u, a1 = u1 ? __ldcg(c1In + g1) : 0u;
    uint32_t m0 = u0 ? __ldcg(cMIn + g0) : 0u, m1 = u1 ? __ldcg(cMIn + g1) : 0u;
    uint32_t k0 = (a0 + m0 + 7u) >> 3, k1 = (a1 + m1 + 7u) >> 3;  // MMA chunks of the branch
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t x0 = __shfl_up_sync(kFull, a0, off), x1 = __shfl_up_sync(kFull, a1, off);
      const uint32_t y0 = __shfl_up_sync(kFull, m0, off), y1 = __shfl_up_sync(kFull, m1, off);
      if (lane >= (uint32_t)off) { a0 += x0; a1 += x1; m0 += y0; m1 += y1; }
      if (MMA) {
        const uint32_t z0 = __shfl_up_sync(kFull, k0, off), z1 = __shfl_up_sync(kFull, k1, off);
        if (lane >= (uint32_t)off) { k0 += z0; k1 += z1; }
      }
    }
    if (MMA) {
      const uint32_t totK = __shfl_sync(kFull, k0, 31);
      uint32_t* PC = sPC + buf * 68u;
      PC[1 + lane] = k0;
      PC[33 + lane] = totK + k1;
      if (lane == 0) PC[0] = 0u;
    }
    const uint32_t totA = __shfl_sync(kFull, a0, 31), totM = __shfl_sync(kFull, m0, 31);
    uint32_t* P1 = sP1 + buf * 68u;
    uint32_t* PM = sPM + buf * 68u;
    P1[1 + lane] = a0;
    P1[33 + lane] = totA + a1;
    PM[1 + lane] = m0;
    PM[33 + lane] = totM + m1;
    if (lane == 0) P1[0] = PM[0] = 0u;
    // Unit table: for unit u < kUnitTab, the number of branches of each list that end at or
    // before the unit's first entry of that list (multi-word in the low half, single-word in
    // the high half), which the units would otherwise count with four ballots each. A branch
    // ending at prefix e is counted from unit ceil(e / 32) on (single-word entries follow
    // all EM multi-word ones): a histogram over units, then a prefix sum. Where a unit
    // straddles the two lists the single-word count is a lower bound, which the units' step
    // over branch boundaries completes.
    uint32_t* UT = sUT + buf * kUnitTab;
    for (uint32_t u = lane; u < kUnitTab; u += 32u) UT[u] = 0u;
    __syncwarp();
    const uint32_t EMt = __shfl_sync(kFull, totM + m1, 31);
    const uint32_t uM0 = (m0 + 31u) >> 5, uM1 = (totM + m1 + 31u) >> 5;
    const uint32_t uS0 = (a0 + EMt + 31u) >> 5, uS1 = (totA + a1 + EMt + 31u) >> 5;
    if (uM0 < kUnitTab) atomicAdd(UT + uM0, 1u);
    if (uM1 < kUnitTab) atomicAdd(UT + uM1, 1u);
    if (uS0 < kUnitTab) atomicAdd(UT + uS0, 1u << 16);
    if (uS1 < kUnitTab) atomicAdd(UT + uS1, 1u << 16);
    __syncwarp();
    {  // inclusive prefix over the kUnitTab units, kUnitTab / 32 per lane (counts <= 64 per half)
      constexpr uint32_t kPerLane = kUnitTab / 32u;
      uint32_t v[kPerLane], sum = 0u;
#pragma unroll
      for (uint32_t j = 0; j < kPerLane; ++j) { sum += UT[lane * kPerLane + j]; v[j] = sum; }
      uint32_t before = sum;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t x = __shfl_up_sync(kFull, before, off);
        if (lane >= (uint32_t)off) before += x;
      }
      before -= sum;
#pragma unroll
      for (uint32_t j = 0; j < kPerLane; ++j) UT[lane * kPerLane + j] = v[j] + before;
    }
  };

  for (uint32_t t = 0; t < c.T; ++t) {
    const uint32_t par = t & 1u;
    const uint32_t* spkIn = d.spk + (size_t)par * B * ncol;
    uint32_t* spkOut = d.spk + (size_t)(par ^ 1u) * B * ncol;
    const uint2* e1In = d.ent1 + (size_t)par * ngrp * B;
    const uint4* eMIn = d.entM + (size_t)par * ngrp * B;
    uint2* e1Out = d.ent1 + (size_t)(par ^ 1u) * ngrp * B;
    uint4* eMOut = d.entM + (size_t)(par ^ 1u) * ngrp * B;
    const uint32_t* c1In = d.ecnt + (size_t)par * 2 * ngrp;
    const uint32_t* cMIn = c1In + ngrp;
    uint32_t* c1Out = d.ecnt + (size_t)(par ^ 1u) * 2 * ngrp;
    uint32_t* cMOut = c1Out + ngrp;
    const bool clamp = t < c.clampSteps;
    // Afferent cache. While the inputs are clamped their spike words are the cue in every
    // step, so the input groups' dendritic terms are the same at steps 1..clampSteps: step 1
    // (whose drives come from the input groups alone, every recurrent column being silent at
    // step 0) stores its per-neuron counters, and steps 2..clampSteps leave the input groups'
    // entries out and add the stored counters in the write-back.
    const bool affStore = d.aff != nullptr && t == 1u;
    const bool affAdd = d.aff != nullptr && t >= 2u && t <= c.clampSteps;
    skipGroups = affAdd ? incols / 8u : 0u;
    // Sparse drive slab (packed path without bias, facilitation or drive log): the write-back
    // stores a (column, trajectory) entry only when the column drive reaches the trajectory's
    // histogram floor. A threshold selected from the histogram is at least the floor, so every
    // gated column has its entry; after a sorting fallback, phase 2 recomputes the gated
    // columns below the floor. At the first step after the clamp the drives fall below the
    // floor for almost every trajectory, so the host has that step store every entry
    // (slabAllStep), or every step (slabFull).
    const bool fast = PACK && !c.useBias && c.facil == 0u && d.refBall == nullptr;
    const bool storeAll = c.slabFull != 0u || t == c.slabAllStep;

    // next step's list lengths start at zero (last read in phase 1 of step t-1)
    if (blockIdx.x == 0)
      for (uint32_t g = tid; g < 2 * ngrp; g += blockDim.x) c1Out[g] = 0u;
    for (uint32_t b = tid; b < B; b += blockDim.x) sFloor[b] = hist_floor(d.thPrev + b);  // read after the sync below

    // ---------------- phase 1
    // thread 0 claims one item ahead: the claim's round trip overlaps the current item. After
    // the first step the first item was claimed, and its tiles requested, before the grid
    // barrier that ended the previous step.
    if (tid == 0) {
      if (!pre) {
        const uint32_t it0 = atomicAdd(d.work + t, 1u);
        sMisc[1] = it0;
        claim = nitems;
        if (it0 < nitems) {
          issue(it0, kbuf);
          claim = atomicAdd(d.work + t, 1u);
        }
      }
      sMisc[6] = sMisc[7] = MMA ? 0u : nw - 1u;  // unit counters (see the unit loop)
    }
    pre = false;
    __syncthreads();
    uint32_t item = sMisc[1];
    if (warp == 0 && item < nitems) prep(item, kbuf, c1In, cMIn);
    __syncthreads();
    // One CTA barrier per item, between its entry units and its write-back. With two counter
    // buffers a warp goes from the write-back of one item straight to the units of the next;
    // with one, a second barrier keeps them apart. Tiles, groups, prefixes, unit counters
    // and next-item slots alternate by item, so each is rewritten only after the barrier
    // that follows its last reader.
    while (item < nitems) {
      const uint32_t bcur = kbuf;
      if (!c.dacc) __syncthreads();
      uint32_t nx = nitems;
      if (tid == 0) {
        nx = claim;
        sMisc[8 + bcur] = nx;
        if (nx < nitems) {
          issue(nx, bcur ^ 1u);
          claim = atomicAdd(d.work + t, 1u);
        }
      }
      // warp 0 loads the next item's groups and prefixes, then joins the entry units
      // (claimed dynamically)
      if (warp == 0) {
        nx = __shfl_sync(kFull, nx, 0);
        if (nx < nitems) prep(nx, bcur ^ 1u, c1In, cMIn);
      }
      const uint32_t c0 = item * kRecallCpi;
      const uint32_t parCur = (bcur ? uses1 : uses0) & 1u;
      // on a timeout the units below run on whatever the buffer holds (in bounds) and the
      // barrier after them ends the launch
      const bool ok = mbar_wait(&sBar[bcur], parCur, c.waitNs);
      if (bcur) ++uses1; else ++uses0;
      uint32_t* accB = sAcc + (c.dacc ? bcur * accWords : 0u);
      const uint32_t* cConn = sConn + bcur * 64u;
      const uint32_t* cP1 = sP1 + bcur * 68u;
      const uint32_t* cPM = sPM + bcur * 68u;
      // multi-word entries (the costlier ones) are dealt first, so the units that finish
      // last are single-word ones
      const uint32_t E1 = cP1[64], EM = cPM[64], E = E1 + EM, units = (E + 31u) >> 5;
      const uint32_t* tileBase = sTile + bcur * kItemWords;
      if (MMA) {
        mma_units<PACK, LIN>(sPC + bcur * 68u, cP1, cPM, cConn, tileBase, accB, accStride, sMisc + 6 + bcur, e1In,
                             eMIn, spkIn, B, ncol, dthr, bst, lane);
      } else
      // the first unit of warps 1.. is fixed (unit warp - 1, no claim round trip); later units,
      // and all of warp 0's (it joins after its look-ahead), are claimed from the counter,
      // which starts at nw - 1
      for (bool first = warp != 0u;; first = false) {
        uint32_t u = warp - 1u;
        if (!first) {
          u = 0;
          if (lane == 0) u = atomicAdd(sMisc + 6 + bcur, 1u);
          u = __shfl_sync(kFull, u, 0);
        }
        if (u >= units) break;
        // the branch of each list (multi-word, single-word) that holds the unit's first entry
        // of that list: the number of branches ending at or before it; a lane then steps over
        // the few branch boundaries between that entry and its own
        const uint32_t f0 = u * 32u, fM = min(f0, EM), f1 = f0 > EM ? f0 - EM : 0u;
        uint32_t spM, sp1;
        if (u < kUnitTab) {  // from the item's unit table
          const uint32_t ut = sUT[bcur * kUnitTab + u];
          spM = ut & 0xFFFFu;
          sp1 = ut >> 16;
        } else {
          spM = (uint32_t)__popc(__ballot_sync(kFull, cPM[lane + 1] <= fM)) +
                (uint32_t)__popc(__ballot_sync(kFull, cPM[lane + 33] <= fM));
          sp1 = (uint32_t)__popc(__ballot_sync(kFull, cP1[lane + 1] <= f1)) +
                (uint32_t)__popc(__ballot_sync(kFull, cP1[lane + 33] <= f1));
        }
        uint32_t flat = f0 + lane;
        if (flat >= E) continue;
        const bool single = flat >= EM;
        const uint32_t* P = single ? cP1 : cPM;
        if (single) flat -= EM;
        uint32_t sp = single ? sp1 : spM;
        while (P[sp + 1] <= flat) ++sp;
        const uint32_t e = flat - P[sp];
        const uint32_t g = cConn[sp];
        const uint32_t* tile = tileBase + (sp >> 5) * kColWords + (sp & 31u) * 256u;
        if (single) {  // one nonzero word: 32 AND-counts
          const uint2 en = __ldcg(e1In + (size_t)g * B + e);
          const uint32_t b = en.x & 0xFFFFu, w = en.x >> 16, S = en.y;
          uint32_t* accb = acc_row<PACK>(accB, (sp >> 5) * B + b);
#pragma unroll
          for (uint32_t r = 0; r < 32u; r += 4) {
            const uint4 a = *reinterpret_cast<const uint4*>(tile + w3r_pos(r, w));
            acc_add4c<PACK, LIN>(accb, r, __popc(a.x & S), __popc(a.y & S), __popc(a.z & S), __popc(a.w & S), dthr,
                                 bst);
          }
        } else {  // several nonzero words: counts in registers (words past the third from the spikes)
          const uint4 en = __ldcg(eMIn + (size_t)g * B + e);
          const uint32_t b = en.x & 0xFFFFu, nz = (en.x >> 16) & 0xFFu;
          uint32_t* accb = acc_row<PACK>(accB, (sp >> 5) * B + b);
          uint32_t cnt[32];
#pragma unroll
          for (int r = 0; r < 32; ++r) cnt[r] = 0u;
          uint32_t m = nz, k = 0;
          while (m) {
            const uint32_t w = (uint32_t)__ffs(m) - 1u;
            m &= m - 1u;
            const uint32_t S = k == 0 ? en.y : k == 1 ? en.z : k == 2 ? en.w : __ldcg(spkIn + (size_t)b * ncol + 8u * g + w);
            ++k;
#pragma unroll
            for (int r = 0; r < 32; r += 4) {
              const uint4 a = *reinterpret_cast<const uint4*>(tile + w3r_pos(r, w));
              cnt[r] += __popc(a.x & S); cnt[r + 1] += __popc(a.y & S);
              cnt[r + 2] += __popc(a.z & S); cnt[r + 3] += __popc(a.w & S);
            }
          }
#pragma unroll
          for (int r = 0; r < 32; r += 4)
            acc_add4c<PACK, LIN>(accb, r, cnt[r], cnt[r + 1], cnt[r + 2], cnt[r + 3], dthr, bst);
        }
      }
      if (__syncthreads_or(!ok)) {
        if (tid == 0) {
          atomicCAS(d.err, 0u, kErrTimeout);
          // the copies this CTA issued must land before its shared memory is released:
          // wait for both buffers' outstanding copies, with a bound of its own
          const uint64_t drain = c.waitNs > kDrainNs ? c.waitNs : kDrainNs;
          mbar_wait(&sBar[bcur], parCur, drain);
          if (nx < nitems) mbar_wait(&sBar[bcur ^ 1u], (bcur ? uses0 : uses1) & 1u, drain);
        }
        __syncthreads();
        return;
      }
      if (tid == 0) sMisc[6 + bcur] = MMA ? 0u : nw - 1u;  // every warp has claimed its units of this item
      // per-neuron and column drives of the item's columns for every trajectory
      if (fast) {
        // the packed counters already are the u16 drive slab. One (column, trajectory) pair
        // per thread, pairs in column-major order: its 16 counter words are read and cleared
        // with scalar shared accesses (rows are 17 words apart, so 32 consecutive rows fall
        // on 32 banks), summed in registers and stored as 64 contiguous bytes
        const uint32_t np = min(kRecallCpi, ncol - c0) * B;
        for (uint32_t p = tid; p < np; p += blockDim.x) {
          const uint32_t colL = p / B, b = p - colL * B, col = c0 + colL;
          uint32_t* src = acc_row<PACK>(accB, p);
          uint32_t w[16];
#pragma unroll
          for (int i = 0; i < 16; ++i) w[i] = src[i];
#pragma unroll
          for (int i = 0; i < 16; ++i) src[i] = 0u;
          if (affStore || affAdd) {  // the afferent cache (halves add without carry: drives stay below 2^16)
            // laid out [column][quad][trajectory]: consecutive threads touch consecutive quads
            uint4* ap = reinterpret_cast<uint4*>(d.aff) + (size_t)col * 4u * B + b;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              if (affStore) {
                __stcg(ap + (size_t)j * B, make_uint4(w[4 * j], w[4 * j + 1], w[4 * j + 2], w[4 * j + 3]));
              } else {
                const uint4 a = __ldcg(ap + (size_t)j * B);
                w[4 * j] += a.x; w[4 * j + 1] += a.y; w[4 * j + 2] += a.z; w[4 * j + 3] += a.w;
              }
            }
          }
          // sum of the 32 per-neuron drives: each word is lo + 65536 hi, so lo + hi is the
          // word minus 65535 hi
          uint32_t s = 0u;
#pragma unroll
          for (int i = 0; i < 16; ++i) s += w[i] - 65535u * (w[i] >> 16);
          const uint32_t fl = sFloor[b];
          if (storeAll || s >= fl) {  // laid out [column][quad][trajectory], like the afferent cache
            uint4* dst = reinterpret_cast<uint4*>(d.acc) + (size_t)col * 4u * B + b;
#pragma unroll
            for (int j = 0; j < 4; ++j) dst[(size_t)j * B] = make_uint4(w[4 * j], w[4 * j + 1], w[4 * j + 2], w[4 * j + 3]);
          }
          __stcg(d.drv + (size_t)b * ncol + col, s);
          if (col >= incols && s >= fl) count_drive(d.thHist + ((size_t)(t % 3u) * B + b) * kHistWords, s);
        }
      } else {
        for (uint32_t pp = warp; pp < kRecallCpi * B; pp += nw) {
          const uint32_t colL = pp / B, b = pp - colL * B, col = c0 + colL;
          if (col >= ncol) continue;
          uint32_t* ab = acc_row<PACK>(accB, colL * B + b);
          uint32_t a = PACK ? ((ab[lane >> 1] >> (16u * (lane & 1u))) & 0xFFFFu) : ab[lane];
          __syncwarp();
          if (lane < (PACK ? 16u : 32u)) ab[lane] = 0u;
          if (c.facil != 0u && ((__ldcg(spkIn + (size_t)b * ncol + col) >> lane) & 1u)) a += c.facil;
          const uint32_t biasL = c.useBias ? (__ldg(d.bias + col * 32u + lane) >> c.biasShift) : 0u;
          a = a > biasL ? a - biasL : 0u;
          if (c.acc32) reinterpret_cast<uint32_t*>(d.acc)[((size_t)b * ncol + col) * 32u + lane] = a;
          else reinterpret_cast<uint16_t*>(d.acc)[((size_t)b * ncol + col) * 32u + lane] = (uint16_t)a;
          const uint32_t dsum = __reduce_add_sync(kFull, a);
          if (lane == 0) {
            __stcg(d.drv + (size_t)b * ncol + col, dsum);
            if (col >= incols && dsum >= sFloor[b])
              count_drive(d.thHist + ((size_t)(t % 3u) * B + b) * kHistWords, dsum);
          }
          if (d.refBall != nullptr && col >= incols) {  // driveLog of k_emit, src/axon.mm:216-220
            const uint32_t rb = __ldg(d.refBall + (size_t)b * ncol + col);
            if (rb) {
              const bool member = (rb >> lane) & 1u, shared = __ldg(d.mult + col * 32u + lane) > 1u;
              const uint32_t mS = __ballot_sync(kFull, member && shared), mE = __ballot_sync(kFull, member && !shared);
              const uint32_t sumS = __reduce_add_sync(kFull, (member && shared) ? a : 0u);
              const uint32_t sumE = __reduce_add_sync(kFull, (member && !shared) ? a : 0u);
              if (lane == 0) {
                uint32_t* dl = d.driveLog + (size_t)b * 256u + t * 4u;
                if (mS) { atomicAdd(dl + 0, sumS); atomicAdd(dl + 1, (uint32_t)__popc(mS)); }
                if (mE) { atomicAdd(dl + 2, sumE); atomicAdd(dl + 3, (uint32_t)__popc(mE)); }
              }
            }
          }
        }
      }
      item = sMisc[8 + bcur];
      kbuf ^= 1u;
    }
    if (!grid_barrier(d.bar, d.err, gridDim.x, epoch++, c.waitNs, sMisc)) return;

    // ---------------- phase 2: threshold, gated k-of-32 ballots, next spike vectors and lists
    // The CTA works as NG groups of whole warps, each on trajectories of its own, so that their
    // latency chains (drive copies, threshold select, per-neuron drive loads, ballots, list
    // appends) overlap: up to three groups, as many as the tile and counter regions (one
    // contiguous range, both idle in phase 2) hold. A group's buffers: the trajectory's drives,
    // its spike vector and the gated (or candidate) columns (ncol words each), the select
    // scratch (512), the drive histogram and each warp's recompute sums. With second drive
    // buffers after all groups' buffers, the next trajectory's drives and histogram are in
    // flight while the current one runs. Whatever of the counter region this uses is zeroed
    // again before phase 1.
    const uint32_t gWords = 3u * ncol + 512u + kHistWords;
    const uint32_t avail = 2u * kItemWords + (c.dacc ? 2u : 1u) * accWords;
    const uint32_t NG = nw >= 3u && 3u * gWords + 32u * nw <= avail ? 3u : nw >= 2u && 2u * gWords + 32u * nw <= avail ? 2u : 1u;
    // group gi has warps [w0, w0 + gnw): the first nw % NG groups one warp more
    const uint32_t gq = nw / NG, gx = nw % NG;
    const uint32_t gi = warp < gx * (gq + 1u) ? warp / (gq + 1u) : gx + (warp - gx * (gq + 1u)) / gq;
    const uint32_t gnw = gq + (gi < gx ? 1u : 0u), w0 = gi * gq + min(gi, gx), gw = warp - w0;
    const WarpGrp grp{tid - 32u * w0, 32u * gnw, 1u + gi};
    const uint32_t usedG = NG * gWords + 32u * nw;  // all groups' buffers
    uint32_t* const sD0 = sTile + gi * gWords + 32u * w0;
    uint32_t* const sSpk = sD0 + ncol;
    uint32_t* const sList = sD0 + 2u * ncol;
    uint32_t* const sRed = sD0 + 3u * ncol;  // 192 words and
    uint32_t* const sHist = sRed + 192u;      // 256 words of the sorting threshold select
    uint32_t* const sCtl = sHist + 256u;      // 64 words: select control, gated count
    uint32_t* const sH0 = sCtl + 64u;         // the drive histogram
    uint32_t* const sScr = sH0 + kHistWords + 32u * gw;  // this warp's drive recompute sums
    const bool dbuf = usedG + NG * (ncol + kHistWords) <= avail;
    const uint32_t usedEnd = usedG + (dbuf ? NG * (ncol + kHistWords) : 0u);
    uint32_t* const sD1 = sTile + usedG + gi * (ncol + kHistWords);
    uint32_t* const sH1 = sD1 + ncol;
    const uint32_t* hStep = d.thHist + (size_t)(t % 3u) * B * kHistWords;
    auto load_drv = [&](uint32_t b, uint32_t slot) {
      const uint4* src = reinterpret_cast<const uint4*>(d.drv + (size_t)b * ncol);
      uint4* dst = reinterpret_cast<uint4*>(slot ? sD1 : sD0);
      for (uint32_t i = grp.t; i < ncol / 4u; i += grp.nt) cp_async16(dst + i, src + i);
      const uint4* hs = reinterpret_cast<const uint4*>(hStep + (size_t)b * kHistWords);
      uint4* hd = reinterpret_cast<uint4*>(slot ? sH1 : sH0);
      for (uint32_t i = grp.t; i < kHistWords / 4u; i += grp.nt) cp_async16(hd + i, hs + i);
    };
    // Tasks. A worker is one group; workers are numbered group-major (wid = gi * G + CTA), so
    // whole trajectories spread evenly over the CTAs. A part is a range of whole groups (8
    // columns) of one trajectory: every part selects the same threshold, then gates, ballots,
    // writes and lists only its own columns, so a split trajectory costs each of its workers
    // about one threshold select.
    // * When the CTAs' groups outnumber B / G whole trajectories each, groups gi < B / G take
    //   trajectory gi * G + CTA, and the B mod G remaining trajectories are split over the
    //   other groups (P parts each), which run beside the whole ones.
    // * Otherwise worker wid takes trajectories wid + k * W for the full rounds k < B / W, and
    //   the remaining R < W are split into P = W / R parts when P >= 2, else taken whole.
    const uint32_t G = gridDim.x, W = G * NG, perCta = B / G;
    const bool spare = perCta < NG && B % G != 0u;
    uint32_t nfull, fb0, fstep, pb = 0u, ppi = 0u, pnp = 1u;
    bool hasPart = false;
    if (spare) {
      const uint32_t v = (gi - min(gi, perCta)) * G + blockIdx.x, V = (NG - perCta) * G, R = B - perCta * G;
      const uint32_t P = V / R;
      fstep = 0u;
      if (gi < perCta) {
        nfull = 1u;
        fb0 = gi * G + blockIdx.x;
      } else if (P >= 2u) {
        nfull = 0u;
        fb0 = 0u;
        hasPart = v < R * P;
        pb = perCta * G + v / P; ppi = v % P; pnp = P;
      } else {
        nfull = v < R ? 1u : 0u;
        fb0 = perCta * G + v;
      }
    } else {
      const uint32_t wid = gi * G + blockIdx.x, F = B / W, R = B - F * W;
      const uint32_t P = R ? W / R : 0u;
      fb0 = wid;
      fstep = W;
      nfull = F + (R != 0u && P < 2u && wid < R ? 1u : 0u);
      hasPart = P >= 2u && wid < R * P;
      pb = F * W + (P ? wid / P : 0u); ppi = P ? wid % P : 0u; pnp = P ? P : 1u;
    }
    const uint32_t ntask = nfull + (hasPart ? 1u : 0u);
    auto task_b = [&](uint32_t k) { return k < nfull ? fb0 + k * fstep : pb; };
    if (ntask) load_drv(task_b(0), 0);
    cp_async_commit();
    for (uint32_t k = 0; k < ntask; ++k) {
      const uint32_t b = task_b(k);
      const bool part = k >= nfull;
      const uint32_t pi = part ? ppi : 0u, np = part ? pnp : 1u;
      const uint32_t gLo = pi * ngrp / np, gHi = (pi + 1u) * ngrp / np, cLo = 8u * gLo, cHi = 8u * gHi;
      const uint32_t slot = dbuf ? (k & 1u) : 0u;
      uint32_t* sD = slot ? sD1 : sD0;
      const uint32_t* sH = slot ? sH1 : sH0;
      const bool hasNext = k + 1u < ntask;
      if (dbuf && hasNext) load_drv(task_b(k + 1u), slot ^ 1u);
      cp_async_commit();
      if (dbuf) cp_async_wait<1>();  // all but the copies just issued: this trajectory's
      else cp_async_wait<0>();
      if (grp.t == 0) { sCtl[9] = 0u; sCtl[0] = 0u; }
      grp.sync();  // every thread's copies have landed
      if (gw == 0) {  // drives the histogram holds
        uint32_t n = 0;
        for (uint32_t i = lane; i < kThetaBins; i += 32u) n += sH[i];
        n = __reduce_add_sync(kFull, n);
        if (lane == 0) sCtl[8] = n;
      }
      grp.sync();
      // gated columns whose drive is below reFloor have no slab entry (a fallback select)
      const uint32_t reFloor = fast && !storeAll && sCtl[8] < c.targetCols ? sFloor[b] : 0u;
      const uint32_t theta = sCtl[8] >= c.targetCols
                                 ? recall_theta(sD, sH, sList, sCtl, incols, ncol, c.targetCols, c.topkPar, grp)
                                 : block_theta(sD, incols, ncol, c.targetCols, c.topkPar, sHist, sRed,
                                               __ldcg(d.thPrev + b), grp);
      // this trajectory's histogram of step t+1 mod 3, last read two steps ago, is cleared
      // for phase 1 of the next step
      if (pi == 0u) {
        uint4* hz = reinterpret_cast<uint4*>(d.thHist + ((size_t)((t + 1u) % 3u) * B + b) * kHistWords);
        for (uint32_t i = grp.t; i < kHistWords / 4u; i += grp.nt) __stcg(hz + i, make_uint4(0u, 0u, 0u, 0u));
      }
      const uint32_t gate = max(theta, 1u);
      const uint32_t* stimb = d.stims + (size_t)b * ncol;
      for (uint32_t cc = cLo + grp.t; cc < cHi; cc += grp.nt) {
        uint32_t v = 0u;
        if (clamp && cc < incols) v = __ldg(stimb + cc);
        else if (sD[cc] >= gate) sList[atomicAdd(sCtl + 9, 1u)] = cc;
        sSpk[cc] = v;
      }
      grp.sync();
      const uint32_t npend = sCtl[9];
      // k-of-32 of one gated column from its per-neuron drive a (one per lane)
      auto emit_col = [&](uint32_t cc, uint32_t a) {
        uint32_t vk, vk1;
        const uint32_t ball = warp_kwta(a, lane, c.k, vk, vk1);
        if (lane == 0) {
          sSpk[cc] = ball;
          if (d.stats && ball != 0u && cc >= incols) {  // k_emit counters, src/axon.mm:225-234
            uint32_t* st = d.stats + (size_t)b * 1024u;
            const uint32_t sb = 64u + t * 8u;
            atomicAdd(st + 0, 1u);
            atomicAdd(st + 1, (uint32_t)__popc(ball));
            atomicAdd(st + sb + 0u, vk - vk1);
            atomicAdd(st + sb + 1u, vk);
            atomicAdd(st + sb + 2u, 1u);
            if (vk == vk1) atomicAdd(st + sb + 3u, 1u);
            if (vk == 0u) atomicAdd(st + sb + 4u, 1u);
          }
        }
      };
      // gated columns without a slab entry: drives recomputed, one column per warp
      if (reFloor != 0u) {
        sScr[lane] = 0u;
        __syncwarp();
        for (uint32_t e = gw; e < npend; e += gnw) {
          const uint32_t cc = sList[e];
          if (sD[cc] < reFloor)
            emit_col(cc, recompute_drive<LIN>(d.W3R, d.conn, spkIn + (size_t)b * ncol, cc, dthr, bst, lane, sScr));
        }
      }
      // the others from the slab, a warp's gated columns kPend at a time: their per-neuron
      // drives load together
      constexpr uint32_t kPend = 4;
      for (uint32_t e0 = gw; e0 < npend; e0 += kPend * gnw) {
        uint32_t av[kPend];
#pragma unroll
        for (uint32_t u = 0; u < kPend; ++u) {
          const uint32_t e = e0 + u * gnw;
          av[u] = 0u;
          if (e < npend && sD[sList[e]] >= reFloor) {
            // the fast write-back's layout: neuron n of (column cc, trajectory b) is 16-bit
            // element n % 8 of quad ((cc * 4 + n / 8) * B + b); the others [b][cc][neuron]
            const size_t o = fast ? (((size_t)sList[e] * 4u + (lane >> 3)) * B + b) * 8u + (lane & 7u)
                                  : ((size_t)b * ncol + sList[e]) * 32u + lane;
            av[u] = c.acc32 ? __ldcg(reinterpret_cast<const uint32_t*>(d.acc) + o)
                            : (uint32_t)__ldcg(reinterpret_cast<const uint16_t*>(d.acc) + o);
          }
        }
#pragma unroll
        for (uint32_t u = 0; u < kPend; ++u) {
          const uint32_t e = e0 + u * gnw;
          if (e >= npend) break;  // warp-uniform
          const uint32_t cc = sList[e];
          if (sD[cc] >= reFloor) emit_col(cc, av[u]);
        }
      }
      grp.sync();
      uint32_t* outb = spkOut + (size_t)b * ncol;
      for (uint32_t i = cLo / 4u + grp.t; i < cHi / 4u; i += grp.nt) {
        const uint4 v = reinterpret_cast<const uint4*>(sSpk)[i];
        __stcg(reinterpret_cast<uint4*>(outb) + i, v);
        if (d.hist) reinterpret_cast<uint4*>(d.hist + ((size_t)b * c.T + t) * ncol)[i] = v;
        if (d.finalOut && t + 1u == c.T) reinterpret_cast<uint4*>(d.finalOut + (size_t)b * ncol)[i] = v;
      }
      if (t + 1u < c.T) {  // group lists for the next step
        for (uint32_t g = gLo + grp.t; g < gHi; g += grp.nt) {
          const uint4 p = reinterpret_cast<const uint4*>(sSpk)[2 * g], q = reinterpret_cast<const uint4*>(sSpk)[2 * g + 1];
          const uint32_t w[8] = {p.x, p.y, p.z, p.w, q.x, q.y, q.z, q.w};
          uint32_t nz = 0, S0 = 0u, S1 = 0u, S2 = 0u, k = 0, w0 = 0;
#pragma unroll
          for (int i = 0; i < 8; ++i)
            if (w[i]) {
              nz |= 1u << i;
              if (k == 0) { S0 = w[i]; w0 = (uint32_t)i; }
              else if (k == 1) S1 = w[i];
              else if (k == 2) S2 = w[i];
              ++k;
            }
          if (k == 1) {
            const uint32_t slot = atomicAdd(c1Out + g, 1u);
            __stcg(e1Out + (size_t)g * B + slot, make_uint2(b | (w0 << 16), S0));
          } else if (k > 1) {
            const uint32_t slot = atomicAdd(cMOut + g, 1u);
            __stcg(eMOut + (size_t)g * B + slot, make_uint4(b | (nz << 16), S0, S1, S2));
          }
        }
      }
      if (grp.t == 0 && pi == 0u) {
        __stcg(d.thPrev + b, theta);
        if (d.theta && t + 1u == c.T) d.theta[b] = theta;
      }
      grp.sync();
      if (!dbuf && hasNext) load_drv(task_b(k + 1u), 0);  // committed at the next task's start
    }
    cp_async_wait<0>();
    if (t + 1u == c.T) break;
    // the part of the counter region that phase 2 used: zero again before the next phase 1
    __syncthreads();
    for (uint32_t i = tid; i + 2u * kItemWords < usedEnd; i += blockDim.x) sAcc[i] = 0u;
    // The tiles of the next step's first item do not depend on this step's spikes: claim it
    // and request them now (the phase-2 buffers over the tile region are free after the
    // barrier above), so that the copy runs while the grid barrier waits.
    if (tid == 0) {
      const uint32_t it0 = atomicAdd(d.work + t + 1u, 1u);
      sMisc[1] = it0;
      claim = nitems;
      if (it0 < nitems) {
        issue(it0, kbuf);
        claim = atomicAdd(d.work + t + 1u, 1u);
      }
    }
    pre = true;
    if (!grid_barrier(d.bar, d.err, gridDim.x, epoch++, c.waitNs, sMisc)) {
      // the copy requested above must land before the CTA's shared memory is released
      if (tid == 0 && sMisc[1] < nitems)
        mbar_wait(&sBar[kbuf], (kbuf ? uses1 : uses0) & 1u, c.waitNs > kDrainNs ? c.waitNs : kDrainNs);
      __syncthreads();
      return;
    }
  }
}

size_t recall_smem_bytes(uint32_t ncol, uint32_t B, uint32_t acc32, uint32_t dacc) {
  (void)ncol;
  const size_t stride = acc32 ? 33 : 17;
  return (2ull * kItemWords + (dacc ? 2 : 1) * kRecallCpi * (size_t)B * stride + 2 * (64 + 68 + 68 + 68) + 16 + 4 + B +
          2 * kUnitTab) *
         4;
}

namespace {
template <bool PACK, bool LIN>
const void* recall_fn_m(uint32_t mma) {
  return mma ? (const void*)k_recall<PACK, LIN, true> : (const void*)k_recall<PACK, LIN, false>;
}
const void* recall_fn(uint32_t acc32, uint32_t lin, uint32_t mma) {
  if (acc32) return lin ? recall_fn_m<false, true>(mma) : recall_fn_m<false, false>(mma);
  return lin ? recall_fn_m<true, true>(mma) : recall_fn_m<true, false>(mma);
}
}  // namespace

cudaError_t recall_max_blocks_per_sm(int acc32, int threads, size_t smem, int* out) {
  for (uint32_t lin = 0; lin < 2; ++lin)
    for (uint32_t mma = 0; mma < 2; ++mma) {
      cudaError_t e = cudaFuncSetAttribute(recall_fn(acc32, lin, mma), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
      if (e != cudaSuccess) return e;
    }
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, recall_fn(acc32, 1, 0), threads, smem);
}

cudaError_t launch_recall(const RecallDev& d, const RecallCfg& c, const RecallShape& s, cudaStream_t st) {
  void* args[] = {(void*)&d, (void*)&c};
  return cudaLaunchCooperativeKernel(recall_fn(c.acc32, c.mode != 2u, c.mma), dim3(s.grid), dim3(s.threads), args,
                                     s.smem, st);
}

}  // namespace axon
