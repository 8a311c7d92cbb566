// Batched drive of the recall server: one tick's drive step for every trajectory of the
// networks that have many trajectories in flight (k_drive, src/axon.mm:150-190, learn = 0).
//
// Work items are (network, column pair) claimed dynamically by every CTA. An item's 64
// W3 tiles (64 KiB, batched layout) arrive by TMA bulk copies into shared memory,
// double-buffered across items, so each tile is read once per tick for all of the
// network's trajectories. The per-group entry lists written by the previous tick's emit
// kernel name, for each presynaptic group, the trajectories whose group spiked and their
// nonzero spike words; lanes take (branch, entry) pairs and AND-popcount the entry's
// words against all 32 rows of the tile into per-(trajectory, neuron) counters in shared
// memory (two 16-bit sums per 32-bit atomic when they fit). The counters become each
// trajectory's per-neuron drives and column drives in its slot. Trajectories are
// independent, so this kernel needs no grid barrier: the emit kernel that follows in the
// stream finishes the step.
#include <cstdint>

#include "axon_device.cuh"
#include "batch_common.cuh"
#include "serve.cuh"

namespace axon {

namespace {
template <bool PACK>
__host__ __device__ constexpr uint32_t sb_stride() { return PACK ? 17u : 33u; }
template <bool PACK>
__host__ __device__ constexpr uint32_t sb_maxb() { return PACK ? kServeMaxB : kServeMaxB32; }
// two counter buffers of this many trajectories take about the shared memory one buffer of
// sb_maxb takes plus what is left of the 227 KiB
template <bool PACK>
__host__ __device__ constexpr uint32_t sb_daccb() { return PACK ? 366u : 188u; }
template <bool PACK>
__host__ __device__ constexpr uint32_t sb_acc_words() {
  return 2u * kRecallCpi * sb_daccb<PACK>() * sb_stride<PACK>() > kRecallCpi * sb_maxb<PACK>() * sb_stride<PACK>()
             ? 2u * kRecallCpi * sb_daccb<PACK>() * sb_stride<PACK>()
             : kRecallCpi * sb_maxb<PACK>() * sb_stride<PACK>();
}
}  // namespace

template <bool PACK, bool LIN>
__global__ void __launch_bounds__(896, 1) k_serve_batched(ServeDev d, ServeCfg c) {
  extern __shared__ __align__(128) uint32_t sm[];
  const uint32_t ncol = c.ncol, ngrp = ncol / 8u, dthr = c.dthr, bst = c.bst;
  constexpr uint32_t accStride = sb_stride<PACK>();
  uint32_t* sTile = sm;                                     // [2][kItemWords]
  // counters: one buffer [kRecallCpi][B][accStride], or two of sb_daccb trajectories
  uint32_t* sAcc = sTile + 2 * kItemWords;
  uint32_t* sConn = sAcc + sb_acc_words<PACK>();            // [2][64] groups of the item's branches
  uint32_t* sP1 = sConn + 2 * 64;                           // [2][68] single-word entries: prefix over 64 branches
  uint32_t* sPM = sP1 + 2 * 68;                             // [2][68] multi-word entries
  uint32_t* sMisc = sPM + 2 * 68;  // [16]: -, first item, -, -, -, -, unit counters [2], next items [2]
  uint64_t* sBar = reinterpret_cast<uint64_t*>(sMisc + 16);  // [2]
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nw = blockDim.x >> 5;
  const uint32_t nip = (ncol + kRecallCpi - 1) / kRecallCpi;  // work items per network
  const uint32_t nitems = d.counts[3];
  if (nitems == 0u) return;
  if (tid == 0) {
    mbar_init(&sBar[0], 1);
    mbar_init(&sBar[1], 1);
    fence_proxy_async_smem();
  }
  // the counters start at zero; each item's write-back clears what it read
  for (uint32_t i = tid; i < sb_acc_words<PACK>(); i += blockDim.x) sAcc[i] = 0u;
  __syncthreads();
  uint32_t uses0 = 0, uses1 = 0, kbuf = 0;

  auto issue = [&](uint32_t it, uint32_t buf) {  // thread 0 only
    const uint32_t* W3R = d.nets[d.bnets[it / nip].net].W3R;
    const uint32_t c0 = (it % nip) * kRecallCpi;
    const uint32_t ncols = min(kRecallCpi, ncol - c0);
    fence_proxy_async_smem();
    mbar_expect_tx(&sBar[buf], ncols * kColWords * 4u);
    for (uint32_t k = 0; k < ncols; ++k)
      bulk_g2s(sTile + buf * kItemWords + k * kColWords, W3R + (size_t)(c0 + k) * kColWords, kColWords * 4u, &sBar[buf]);
  };
  // warp 0: the item's branch groups and the prefixes of its 64 entry-list lengths, single-
  // word and multi-word, into buffer buf
  auto prep = [&](uint32_t it, uint32_t buf) {
    const ServeBNet pn = d.bnets[it / nip];
    const uint32_t* conn = d.nets[pn.net].conn;
    const uint32_t* c1 = d.nets[pn.net].ecnt + (size_t)d.par * 2 * ngrp;
    const uint32_t* cM = c1 + ngrp;
    const uint32_t c0 = (it % nip) * kRecallCpi;
    const bool v1 = c0 + 1 < ncol;
    const uint32_t g0 = __ldg(conn + c0 * kNslot + lane), g1 = v1 ? __ldg(conn + (c0 + 1) * kNslot + lane) : 0u;
    sConn[buf * 64u + lane] = g0;
    sConn[buf * 64u + 32u + lane] = g1;
    uint32_t a0 = __ldcg(c1 + g0), a1 = v1 ? __ldcg(c1 + g1) : 0u;
    uint32_t m0 = __ldcg(cM + g0), m1 = v1 ? __ldcg(cM + g1) : 0u;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t x0 = __shfl_up_sync(kFull, a0, off), x1 = __shfl_up_sync(kFull, a1, off);
      const uint32_t y0 = __shfl_up_sync(kFull, m0, off), y1 = __shfl_up_sync(kFull, m1, off);
      if (lane >= (uint32_t)off) { a0 += x0; a1 += x1; m0 += y0; m1 += y1; }
    }
    const uint32_t totA = __shfl_sync(kFull, a0, 31), totM = __shfl_sync(kFull, m0, 31);
    uint32_t* P1 = sP1 + buf * 68u;
    uint32_t* PM = sPM + buf * 68u;
    P1[1 + lane] = a0;
    P1[33 + lane] = totA + a1;
    PM[1 + lane] = m0;
    PM[33 + lane] = totM + m1;
    if (lane == 0) P1[0] = PM[0] = 0u;
  };
  auto spk_prev = [&](uint32_t tabOff, uint32_t b) -> const uint32_t* {  // spk(t-1) of batch index b
    const uint2 st = __ldg(d.btab + tabOff + b);
    return d.slots + (size_t)st.x * d.slotWords + ((st.y - 1u) & 1u) * ncol;
  };

  // thread 0 claims one item ahead: the claim's round trip overlaps the current item
  uint32_t claim = nitems;
  if (tid == 0) {
    const uint32_t it0 = atomicAdd(d.work, 1u);
    sMisc[1] = it0;
    sMisc[6] = sMisc[7] = 0u;
    if (it0 < nitems) {
      issue(it0, kbuf);
      claim = atomicAdd(d.work, 1u);
    }
  }
  __syncthreads();
  uint32_t item = sMisc[1];
  if (warp == 0 && item < nitems) prep(item, kbuf);
  __syncthreads();
  // One CTA barrier per item, between its entry units and its write-back. With two counter
  // buffers a warp goes from the write-back of one item straight to the units of the next;
  // with one, a second barrier keeps them apart. Tiles, groups, prefixes, unit counters and
  // next-item slots alternate by item, so each is rewritten only after the barrier that
  // follows its last reader.
  while (item < nitems) {
    const uint32_t bcur = kbuf;
    if (!d.dacc) __syncthreads();
    uint32_t nx = nitems;
    if (tid == 0) {
      nx = claim;
      sMisc[8 + bcur] = nx;
      if (nx < nitems) {
        issue(nx, bcur ^ 1u);
        claim = atomicAdd(d.work, 1u);
      }
    }
    // warp 0 loads the next item's groups and prefixes, then joins the entry units (claimed
    // dynamically)
    if (warp == 0) {
      nx = __shfl_sync(kFull, nx, 0);
      if (nx < nitems) prep(nx, bcur ^ 1u);
    }
    const ServeBNet bn = d.bnets[item / nip];
    const uint2* e1In = d.nets[bn.net].ent1 + (size_t)d.par * ngrp * kServeMaxB;
    const uint4* eMIn = d.nets[bn.net].entM + (size_t)d.par * ngrp * kServeMaxB;
    const uint32_t B = bn.B;
    const uint32_t c0 = (item % nip) * kRecallCpi;
    const uint32_t parCur = (bcur ? uses1 : uses0) & 1u;
    // on a timeout the units below run on whatever the buffer holds (in bounds) and the
    // barrier after them ends the launch
    const bool ok = mbar_wait(&sBar[bcur], parCur, d.waitNs);
    if (bcur) ++uses1; else ++uses0;
    uint32_t* accB = sAcc + (d.dacc ? bcur * (kRecallCpi * sb_daccb<PACK>() * accStride) : 0u);
    const uint32_t* cConn = sConn + bcur * 64u;
    const uint32_t* cP1 = sP1 + bcur * 68u;
    const uint32_t* cPM = sPM + bcur * 68u;
    // multi-word entries (the costlier ones) are dealt first, so the units that finish last
    // are single-word ones
    const uint32_t E1 = cP1[64], EM = cPM[64], E = E1 + EM, units = (E + 31u) >> 5;
    const uint32_t* tileBase = sTile + bcur * kItemWords;
    for (;;) {
      uint32_t u = 0;
      if (lane == 0) u = atomicAdd(sMisc + 6 + bcur, 1u);
      u = __shfl_sync(kFull, u, 0);
      if (u >= units) break;
      uint32_t flat = u * 32u + lane;
      if (flat >= E) continue;
      const bool single = flat >= EM;
      const uint32_t* P = single ? cP1 : cPM;
      if (single) flat -= EM;
      uint32_t sp = 0;
#pragma unroll
      for (uint32_t step = 32; step; step >>= 1)
        if (sp + step < 64u && P[sp + step] <= flat) sp += step;
      const uint32_t e = flat - P[sp];
      const uint32_t g = cConn[sp];
      const uint32_t* tile = tileBase + (sp >> 5) * kColWords + (sp & 31u) * 256u;
      if (single) {  // one nonzero word: 32 AND-counts
        const uint2 en = __ldcg(e1In + (size_t)g * kServeMaxB + e);
        const uint32_t b = en.x & 0xFFFFu, w = en.x >> 16, S = en.y;
        uint32_t* accb = accB + ((sp >> 5) * B + b) * accStride;
#pragma unroll
        for (uint32_t r = 0; r < 32u; r += 4) {
          const uint4 a = *reinterpret_cast<const uint4*>(tile + w3r_pos(r, w));
          acc_add4c<PACK, LIN>(accb, r, __popc(a.x & S), __popc(a.y & S), __popc(a.z & S), __popc(a.w & S), dthr,
                               bst);
        }
      } else {  // several nonzero words: counts in registers (words past the third from the spikes)
        const uint4 en = __ldcg(eMIn + (size_t)g * kServeMaxB + e);
        const uint32_t b = en.x & 0xFFFFu, nz = (en.x >> 16) & 0xFFu;
        uint32_t* accb = accB + ((sp >> 5) * B + b) * accStride;
        uint32_t cnt[32];
#pragma unroll
        for (int r = 0; r < 32; ++r) cnt[r] = 0u;
        uint32_t m = nz, k = 0;
        while (m) {
          const uint32_t w = (uint32_t)__ffs(m) - 1u;
          m &= m - 1u;
          const uint32_t S = k == 0 ? en.y : k == 1 ? en.z : k == 2 ? en.w : __ldcg(spk_prev(bn.tabOff, b) + 8u * g + w);
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
        // the copies this CTA issued must land before its shared memory is released
        const uint64_t drain = d.waitNs > kDrainNs ? d.waitNs : kDrainNs;
        mbar_wait(&sBar[bcur], parCur, drain);
        if (nx < nitems) mbar_wait(&sBar[bcur ^ 1u], (bcur ? uses0 : uses1) & 1u, drain);
      }
      __syncthreads();
      return;
    }
    if (tid == 0) sMisc[6 + bcur] = 0u;  // every warp has claimed its units of this item
    // per-neuron and column drives of the item's columns into every trajectory's slot
    const uint32_t accOff = serve_acc_off(ncol), xOff = 2u * ncol + 2u * d.nactw;
    if (PACK) {  // the packed counters are the u16 drives: four lanes per (column, trajectory),
                 // each storing 4 of its 16 words as one 16-byte vector
      const uint32_t q = lane & 3u, grp = lane >> 2;
      const uint32_t gmask = 0xFu << (grp * 4u);
      for (uint32_t pp = warp * 8u + grp; pp < kRecallCpi * B; pp += nw * 8u) {
        const uint32_t colL = pp / B, b = pp - colL * B, col = c0 + colL;
        if (col >= ncol) continue;  // uniform over the four lanes
        uint32_t* base = d.slots + (size_t)__ldg(d.btab + bn.tabOff + b).x * d.slotWords;
        uint32_t* src = accB + (colL * B + b) * accStride + q * 4u;
        const uint4 w = make_uint4(src[0], src[1], src[2], src[3]);
        src[0] = src[1] = src[2] = src[3] = 0u;
        __stcg(reinterpret_cast<uint4*>(base + accOff + col * 16u) + q, w);
        uint32_t s = (w.x & 0xFFFFu) + (w.x >> 16) + (w.y & 0xFFFFu) + (w.y >> 16) + (w.z & 0xFFFFu) + (w.z >> 16) +
                     (w.w & 0xFFFFu) + (w.w >> 16);
        s += __shfl_xor_sync(gmask, s, 1);
        s += __shfl_xor_sync(gmask, s, 2);
        if (q == 0) __stcg(base + xOff + col, s);
      }
    } else {
      for (uint32_t pp = warp; pp < kRecallCpi * B; pp += nw) {
        const uint32_t colL = pp / B, b = pp - colL * B, col = c0 + colL;
        if (col >= ncol) continue;
        const uint2 st = __ldg(d.btab + bn.tabOff + b);
        uint32_t* base = d.slots + (size_t)st.x * d.slotWords;
        uint32_t a = accB[(colL * B + b) * accStride + lane];
        accB[(colL * B + b) * accStride + lane] = 0u;  // one lane per word
        if (c.facil != 0u && st.y > 0u && ((__ldcg(base + ((st.y - 1u) & 1u) * ncol + col) >> lane) & 1u)) a += c.facil;
        if (c.acc32) __stcg(base + accOff + col * 32u + lane, a);
        else __stcg(reinterpret_cast<unsigned short*>(base + accOff) + col * 32u + lane, (unsigned short)a);
        const uint32_t dsum = __reduce_add_sync(kFull, a);
        if (lane == 0) __stcg(base + xOff + col, dsum);
      }
    }
    item = sMisc[8 + bcur];
    kbuf ^= 1u;
  }
}

size_t serve_batched_smem_bytes(uint32_t packed) {
  const size_t acc = packed ? sb_acc_words<true>() : sb_acc_words<false>();
  return (2ull * kItemWords + acc + 2 * (64 + 68 + 68) + 16 + 4) * 4;
}

uint32_t serve_batched_dacc_maxb(uint32_t packed) { return packed ? sb_daccb<true>() : sb_daccb<false>(); }

namespace {
const void* sb_fn(uint32_t packed, uint32_t lin) {
  if (packed) return lin ? (const void*)k_serve_batched<true, true> : (const void*)k_serve_batched<true, false>;
  return lin ? (const void*)k_serve_batched<false, true> : (const void*)k_serve_batched<false, false>;
}
}  // namespace

cudaError_t serve_batched_prepare(uint32_t packed) {
  for (uint32_t lin = 0; lin < 2; ++lin) {
    const cudaError_t e =
        cudaFuncSetAttribute(sb_fn(packed, lin), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)serve_batched_smem_bytes(packed));
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_serve_batched(const ServeDev& d, const ServeCfg& c, int sms, cudaStream_t st) {
  const uint32_t packed = (!c.acc32 && c.facil == 0u) ? 1u : 0u;
  void* args[] = {(void*)&d, (void*)&c};
  return cudaLaunchKernel(sb_fn(packed, c.mode != 2u), dim3(sms), dim3(896), args, serve_batched_smem_bytes(packed), st);
}

}  // namespace axon
