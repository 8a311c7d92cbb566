// Batched recall: B trajectories of one trained network share every read of W3.
//
// Readout presentations of rakib-nyc/axon (present() with learn=false, src/axon.mm:815-888)
// change no weight, so any number of them can run together. One cooperative launch runs
// T steps for all B trajectories, two grid barriers per step:
//
//   phase 1  work items are columns (dynamically claimed). For its column, a warp per
//            trajectory computes every neuron's drive over the branches whose presynaptic
//            group is active in that trajectory: the warp gathers the spike words of up to
//            four active branches in one coalesced load, ballots which are nonzero, and
//            pops AND-counts only for nonzero words against W3 words that all B
//            trajectories of the item read through L1. Per-neuron drive goes to a u16 (or
//            u32) slab, the column drive to a [B][ncol] table.
//   phase 2  per trajectory: the column threshold (block_theta), then the exact k-of-32
//            ballot only for columns that pass the gate - a few dozen of 4096 - from the
//            stored per-neuron drives; the new spike vector and its group-activity bits.
//
// W3 is re-laid out once per trained network as [col][branch][word][lane] so that a
// warp's 32 lanes read one word of a tile from 128 contiguous bytes.
#include <cstdint>

#include "axon_device.cuh"
#include "batch.cuh"
#include "theta.cuh"

namespace axon {

__global__ void k_make_w3b(const uint4* __restrict__ W3, uint32_t* __restrict__ W3B, uint64_t ntile) {
  // one thread per (tile, lane): reads 2 uint4, writes 8 words strided by 32
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ntile * 32) return;
  const uint64_t tile = i >> 5;
  const uint32_t lane = (uint32_t)(i & 31u);
  const uint4 a = W3[tile * kTileU4 + lane], b = W3[tile * kTileU4 + 32 + lane];
  uint32_t* o = W3B + tile * 256 + lane;
  o[0 * 32] = a.x; o[1 * 32] = a.y; o[2 * 32] = a.z; o[3 * 32] = a.w;
  o[4 * 32] = b.x; o[5 * 32] = b.y; o[6 * 32] = b.z; o[7 * 32] = b.w;
}

cudaError_t launch_make_w3b(const uint4* W3, uint32_t* W3B, uint32_t ncol, cudaStream_t st) {
  const uint64_t ntile = (uint64_t)ncol * kNslot;
  k_make_w3b<<<(unsigned)((ntile * 32 + 255) / 256), 256, 0, st>>>(W3, W3B, ntile);
  return cudaGetLastError();
}

// dendritic nonlinearity of k_drive, src/axon.mm:174-178
__device__ __forceinline__ uint32_t branch_term(uint32_t cnt, const RecallCfg& c) {
  const bool nmda = cnt >= c.dthr;
  if (c.mode == 0u) return cnt;
  if (c.mode == 1u) return nmda ? cnt + c.boost : cnt;
  return nmda ? 1u : 0u;
}

template <typename AccT>
__global__ void __launch_bounds__(1024, 1) k_recall(RecallDev d, RecallCfg c) {
  extern __shared__ __align__(16) uint32_t sm[];
  const uint32_t ncol = c.ncol, incols = c.incols, B = c.B;
  const uint32_t ngrp = ncol / 8u, nactw = (((ngrp + 31u) / 32u) + 3u) & ~3u;
  uint32_t* sD = sm;               // drives of one trajectory
  uint32_t* sSpk = sD + ncol;      // its new spike vector
  uint32_t* sList = sSpk + ncol;   // columns that need the k-of-32 ballot
  uint32_t* sHist = sList + ncol;  // 256
  uint32_t* sRed = sHist + 256;    // 96
  uint32_t* sMisc = sRed + 96;     // [0] barrier flag, [1] work item, [2] list length

  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nw = blockDim.x >> 5;
  const uint32_t cpi = c.cpi, nitems = (ncol + cpi - 1) / cpi;
  const uint32_t wsub = warp % cpi, bstart = warp / cpi, bstep = nw / cpi;
  AccT* accv = reinterpret_cast<AccT*>(d.acc);
  uint32_t epoch = 0;

  for (uint32_t t = 0; t < c.T; ++t) {
    const uint32_t par = t & 1u;
    const uint32_t* spkIn = d.spk + (size_t)par * B * ncol;
    uint32_t* spkOut = d.spk + (size_t)(par ^ 1u) * B * ncol;
    const uint32_t* actIn = d.act + (size_t)par * B * nactw;
    uint32_t* actOut = d.act + (size_t)(par ^ 1u) * B * nactw;
    const bool clamp = t < c.clampSteps;

    // ---------------- phase 1: drives of every (column, trajectory)
    for (;;) {
      if (tid == 0) sMisc[1] = atomicAdd(d.work + t, 1u);
      __syncthreads();
      const uint32_t item = sMisc[1];
      __syncthreads();
      if (item >= nitems) break;
      const uint32_t cc = item * cpi + wsub;
      if (cc >= ncol || bstart >= B) continue;
      const uint32_t gS = __ldg(d.conn + cc * kNslot + lane);  // lane = branch
      const uint32_t biasL = c.useBias ? (__ldg(d.bias + cc * 32u + lane) >> c.biasShift) : 0u;
      const bool logCol = d.refBall != nullptr && cc >= incols;
      const uint32_t multL = logCol ? __ldg(d.mult + cc * 32u + lane) : 0u;
      const uint32_t* wcol = d.W3B + (size_t)cc * (kNslot * 256u) + lane;
      for (uint32_t b = bstart; b < B; b += bstep) {
        const uint32_t* inb = spkIn + (size_t)b * ncol;
        const uint32_t aw = __ldcg(actIn + (size_t)b * nactw + (gS >> 5));
        uint32_t amask = __ballot_sync(kFull, (aw >> (gS & 31u)) & 1u);
        uint32_t a = 0;
        while (amask) {
          uint32_t s4[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            s4[u] = amask ? (uint32_t)(__ffs(amask) - 1) : 32u;
            amask &= amask - 1u;
          }
          const uint32_t slot = lane >> 3, wd = lane & 7u;
          const uint32_t mys = slot == 0 ? s4[0] : slot == 1 ? s4[1] : slot == 2 ? s4[2] : s4[3];
          const uint32_t g = __shfl_sync(kFull, gS, mys & 31u);
          const uint32_t word = mys < 32u ? __ldcg(inb + 8u * g + wd) : 0u;
          const uint32_t nz = __ballot_sync(kFull, word != 0u);
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (s4[u] >= 32u) break;
            uint32_t m = (nz >> (8 * u)) & 0xFFu, cnt = 0;
            const uint32_t* wt = wcol + s4[u] * 256u;
            while (m) {
              const uint32_t w2 = (uint32_t)(__ffs(m) - 1);
              m &= m - 1u;
              const uint32_t S = __shfl_sync(kFull, word, 8u * u + w2);
              cnt += __popc(__ldg(wt + w2 * 32u) & S);
            }
            a += branch_term(cnt, c);
          }
        }
        if (c.facil != 0u && ((__ldcg(inb + cc) >> lane) & 1u)) a += c.facil;
        a = a > biasL ? a - biasL : 0u;
        accv[((size_t)b * ncol + cc) * 32u + lane] = (AccT)a;
        const uint32_t dsum = __reduce_add_sync(kFull, a);
        if (lane == 0) __stcg(d.drv + (size_t)b * ncol + cc, dsum);
        if (logCol) {  // driveLog of k_emit, src/axon.mm:216-220
          const uint32_t rb = __ldg(d.refBall + (size_t)b * ncol + cc);
          if (rb) {
            const bool member = (rb >> lane) & 1u, shared = multL > 1u;
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
    if (!grid_barrier(d.bar, d.err, gridDim.x, epoch++, c.waitNs, sMisc)) return;

    // ---------------- phase 2: threshold, gated k-of-32 ballots, next spike vectors
    for (uint32_t b = blockIdx.x; b < B; b += gridDim.x) {
      const uint32_t* drvb = d.drv + (size_t)b * ncol;
      for (uint32_t i = tid; i < ncol / 4u; i += blockDim.x)
        reinterpret_cast<uint4*>(sD)[i] = __ldcg(reinterpret_cast<const uint4*>(drvb) + i);
      if (tid == 0) sMisc[2] = 0u;
      __syncthreads();
      const uint32_t theta = block_theta(sD, incols, ncol, c.targetCols, c.topkPar, sHist, sRed);
      const uint32_t gate = max(theta, 1u);
      const uint32_t* stimb = d.stims + (size_t)b * ncol;
      for (uint32_t cc = tid; cc < ncol; cc += blockDim.x) {
        uint32_t v = 0u;
        if (clamp && cc < incols) v = __ldg(stimb + cc);
        else if (sD[cc] >= gate) sList[atomicAdd(sMisc + 2, 1u)] = cc;
        sSpk[cc] = v;
      }
      __syncthreads();
      const uint32_t npend = sMisc[2];
      for (uint32_t e = warp; e < npend; e += nw) {
        const uint32_t cc = sList[e];
        const uint32_t a = (uint32_t)__ldcg(accv + ((size_t)b * ncol + cc) * 32u + lane);
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
      }
      __syncthreads();
      uint32_t* outb = spkOut + (size_t)b * ncol;
      for (uint32_t i = tid; i < ncol / 4u; i += blockDim.x) {
        const uint4 v = reinterpret_cast<const uint4*>(sSpk)[i];
        __stcg(reinterpret_cast<uint4*>(outb) + i, v);
        if (d.hist) reinterpret_cast<uint4*>(d.hist + ((size_t)b * c.T + t) * ncol)[i] = v;
        if (d.finalOut && t + 1u == c.T) reinterpret_cast<uint4*>(d.finalOut + (size_t)b * ncol)[i] = v;
      }
      for (uint32_t gb = warp * 32u; gb < nactw * 32u; gb += nw * 32u) {
        const uint32_t g = gb + lane;
        bool any = false;
        if (g < ngrp) {
          const uint4 p = reinterpret_cast<const uint4*>(sSpk)[2 * g], q = reinterpret_cast<const uint4*>(sSpk)[2 * g + 1];
          any = (p.x | p.y | p.z | p.w | q.x | q.y | q.z | q.w) != 0u;
        }
        const uint32_t wv = __ballot_sync(kFull, any);
        if (lane == 0) __stcg(actOut + (size_t)b * nactw + (gb >> 5), wv);
      }
      if (tid == 0 && d.theta && t + 1u == c.T) d.theta[b] = theta;
      __syncthreads();
    }
    if (t + 1u < c.T && !grid_barrier(d.bar, d.err, gridDim.x, epoch++, c.waitNs, sMisc)) return;
  }
}

size_t recall_smem_bytes(uint32_t ncol) { return (3ull * ncol + 256 + 96 + 4) * 4; }

cudaError_t recall_max_blocks_per_sm(int acc32, int threads, size_t smem, int* out) {
  const void* fn = acc32 ? (const void*)k_recall<uint32_t> : (const void*)k_recall<uint16_t>;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, fn, threads, smem);
}

cudaError_t launch_recall(const RecallDev& d, const RecallCfg& c, const RecallShape& s, cudaStream_t st) {
  void* args[] = {(void*)&d, (void*)&c};
  const void* fn = c.acc32 ? (const void*)k_recall<uint32_t> : (const void*)k_recall<uint16_t>;
  return cudaLaunchCooperativeKernel(fn, dim3(s.grid), dim3(s.threads), args, s.smem, st);
}

}  // namespace axon
