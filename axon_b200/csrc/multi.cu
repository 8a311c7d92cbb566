// Many independent AXON networks in one persistent cooperative launch.
//
// The grid is cut into slots of consecutive CTAs. A slot runs a queue of networks, one
// after the other, and each network runs its own program of presentations (training
// presents, then readouts) - the step loop of present(), src/axon.mm:815-888, for every
// entry. Within a slot the step is the plain kernel's: phase A (drive + ungated k-WTA of
// the owned columns, published), one slot-wide barrier, phase B (every CTA selects the
// column threshold and rebuilds the spike vector in shared memory), phase C (records,
// bias, learning of the owned columns).
//
// Unlike the plain kernel, a slot may be a handful of CTAs, so a warp can own tens of
// columns: per-column state lives in global memory (acc, bbits, bias: L2-resident, each
// word touched only by its owner lane) and in shared memory (k-WTA values), and learning
// runs in chunks of at most kChunk columns. A column's W tiles are read and written only
// by its owner CTA, so slots and CTAs share no weights; the exchange slots alternate by a
// slot-wide step counter, so consecutive presentations need no extra barrier.
#include <cstdint>

#include "axon_device.cuh"
#include "emit.cuh"
#include "learn.cuh"
#include "multi.cuh"
#include "theta.cuh"

namespace axon {

namespace {
constexpr uint32_t kChunk = 64;  // learning columns per chunk

struct MultiSmem {  // offsets (in words) of the shared-memory arrays
  uint32_t spk0, spk1, act0, act1, d, b, stim, hist, red, flag, vk, vk1, lcol, task, bbl, ltp, ltd, colc, total;
};
__host__ __device__ inline MultiSmem multi_layout(uint32_t ncol, uint32_t incols, uint32_t maxCols) {
  const uint32_t ngrp = ncol / 8u, nactw = (((ngrp + 31u) / 32u) + 3u) & ~3u;
  MultiSmem s{};
  uint32_t o = 0;
  s.spk0 = o; o += ncol;
  s.spk1 = o; o += ncol;
  s.act0 = o; o += nactw;
  s.act1 = o; o += nactw;
  s.d = o; o += ncol;
  s.b = o; o += ncol;
  s.stim = o; o += (incols + 3u) & ~3u;
  s.hist = o; o += 256;
  s.red = o; o += 192;
  s.flag = o; o += 4;
  s.vk = o; o += maxCols;
  s.vk1 = o; o += maxCols;
  s.lcol = o; o += maxCols;
  s.task = o; o += kChunk * 32;
  s.bbl = o; o += kChunk * 32;
  s.ltp = o; o += kChunk * 32;
  s.ltd = o; o += kChunk * 32;
  s.colc = o; o += kChunk;
  s.total = o;
  return s;
}
}  // namespace

// NT threads per CTA (one CTA per SM), U W3 tiles in flight per warp.
template <int NT, int U>
__global__ void __launch_bounds__(NT, 1) k_multi(MultiDev m, MultiCfg c) {
  extern __shared__ __align__(16) uint32_t sm[];
  __shared__ MultiNet sNet;
  __shared__ MultiPresent sPr;
  const uint32_t ncol = c.ncol, incols = c.incols, ngrp = ncol / 8u;
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, wpb = blockDim.x >> 5;
  const MultiSmem L = multi_layout(ncol, incols, wpb * c.maxCpw);
  uint32_t* sD = sm + L.d;
  uint32_t* sB = sm + L.b;
  uint32_t* sStim = sm + L.stim;
  uint32_t* sHist = sm + L.hist;
  uint32_t* sRed = sm + L.red;
  uint32_t* sFlag = sm + L.flag;  // [0] barrier flag, [1] learning-column count, [2] task count
  uint32_t* sVk = sm + L.vk;
  uint32_t* sVk1 = sm + L.vk1;
  uint32_t* sLcol = sm + L.lcol;
  uint32_t* sTask = sm + L.task;
  uint32_t* sBBL = sm + L.bbl;
  uint32_t* sLTP = sm + L.ltp;
  uint32_t* sLTD = sm + L.ltd;
  uint32_t* sColC = sm + L.colc;

  // the slot of this CTA
  uint32_t slot = 0;
  while (slot + 1u < m.nslots && blockIdx.x >= m.slots[slot + 1u].cta0) ++slot;
  const MultiSlot S = m.slots[slot];
  if (blockIdx.x < S.cta0 || blockIdx.x >= S.cta0 + S.ncta) return;  // not covered (the host never does this)
  const uint32_t rank = blockIdx.x - S.cta0, nb = S.ncta;
  const uint32_t gw = rank * wpb + warp, nwS = nb * wpb;
  const uint32_t cpw = (ncol + nwS - 1u) / nwS;  // <= c.maxCpw by construction
  uint32_t* bar = m.bars + slot * 32u;
  if (tid == 0) { sFlag[1] = 0u; sFlag[2] = 0u; }
  uint32_t gstep = 0;   // slot-wide step counter: barrier epoch and exchange parity
  uint32_t nTiles = 0;  // W3 tiles this warp read (summed into m.work at the end)
  uint32_t thPrev = 0;  // last threshold: a starting guess for the next selection

  for (uint32_t qi = S.q0; qi < S.q1; ++qi) {
    __syncthreads();
    if (tid == 0) sNet = m.nets[m.queue[qi]];
    __syncthreads();
    const uint32_t nprog = sNet.nprog;
    for (uint32_t pi = 0; pi < nprog; ++pi) {
      if (tid == 0) sPr = sNet.prog[pi];
      __syncthreads();
      const uint32_t T = sPr.T, clampSteps = sPr.clampSteps, learn = sPr.learn, useBias = sPr.useBias;
      const uint32_t kk = sPr.k, facil = sPr.facil;
      uint32_t* sSpk0 = sm + L.spk0;
      uint32_t* sSpk1 = sm + L.spk1;
      uint32_t* sAct0 = sm + L.act0;
      uint32_t* sAct1 = sm + L.act1;
      for (uint32_t i = tid; i < ncol; i += blockDim.x) sSpk0[i] = 0u;
      for (uint32_t i = tid; i < L.act1 - L.act0; i += blockDim.x) sAct0[i] = 0u;
      for (uint32_t i = tid; i < incols; i += blockDim.x) sStim[i] = sPr.stim[i];
      __syncthreads();

      for (uint32_t t = 0; t < T; ++t, ++gstep) {
        const uint32_t* sIn = (t & 1u) ? sSpk1 : sSpk0;
        uint32_t* sOut = (t & 1u) ? sSpk0 : sSpk1;
        const uint32_t* sActIn = (t & 1u) ? sAct1 : sAct0;
        uint32_t* sActOut = (t & 1u) ? sAct0 : sAct1;
        const uint4* sIn4 = reinterpret_cast<const uint4*>(sIn);
        const uint32_t par = gstep & 1u;
        const bool clamp = t < clampSteps;
        const uint32_t phase = (!learn || !c.contrast) ? 0u
                               : (clamp ? 1u : (((t - clampSteps) % c.ltdEvery == 0u) ? 2u : 3u));

        // ---------------- phase A: drive (k_drive, src/axon.mm:150-190) + ungated k-WTA
        {
          const uint4* W3 = sNet.d.W3;
          const uint32_t* conn = sNet.d.conn;
          uint32_t* biasG = sNet.d.bias;
          uint32_t* accG = sNet.d.acc;
          uint32_t* bbG = sNet.d.bbits;
          uint32_t* xdrive = sNet.d.xdrive + par * ncol;
          uint32_t* xball = sNet.d.xball + par * ncol;
          uint32_t* driveG = sNet.d.drive;
          uint32_t* margG = sNet.d.marg;
          uint32_t cnNext = gw < ncol ? __ldg(conn + gw * kNslot + lane) : 0u;
          for (uint32_t i = 0; i < cpw; ++i) {
            const uint32_t cc = gw + i * nwS;
            if (cc >= ncol) break;  // warp-uniform
            const uint32_t cn = cnNext;
            if (cc + nwS < ncol) cnNext = __ldg(conn + (cc + nwS) * kNslot + lane);
            // k_bias of the previous step (src/axon.mm:240-253) runs here, on the bias value
            // this step's drive reads anyway: fired(t-1) is the bit of spk(t-1)
            const bool biasStep = learn && t > 0u && cc >= incols;
            uint32_t bsrc = (useBias || biasStep) ? __ldcg(biasG + cc * 32u + lane) : 0u;
            if (biasStep) {
              const int dec = (((t - 1u) % max(c.biasDownEvery, 1u)) == 0u) ? (int)c.biasDown : 0;
              const int nbv = (int)bsrc + (((sIn[cc] >> lane) & 1u) ? (int)c.biasUp : -dec);
              bsrc = (uint32_t)max(0, nbv);
              __stcg(biasG + cc * 32u + lane, bsrc);
            }
            uint32_t active = __ballot_sync(kFull, (sActIn[cn >> 5] >> (cn & 31u)) & 1u);
            nTiles += __popc(active);
            uint32_t a = 0, b2 = 0;
            const uint4* Wt = W3 + (size_t)cc * kNslot * kTileU4 + lane;
            while (active) {
              uint32_t s[U];
              bool v[U];
              uint4 w0[U], w1[U];
#pragma unroll
              for (int u = 0; u < U; ++u) {
                v[u] = active != 0u;
                s[u] = v[u] ? (uint32_t)(__ffs(active) - 1) : 0u;
                active &= active - 1u;
              }
#pragma unroll
              for (int u = 0; u < U; ++u)
                if (v[u]) {
                  w0[u] = __ldcg(Wt + s[u] * kTileU4);
                  w1[u] = __ldcg(Wt + s[u] * kTileU4 + 32);
                }
#pragma unroll
              for (int u = 0; u < U; ++u)
                if (v[u]) {
                  const uint32_t g = __shfl_sync(kFull, cn, s[u]);
                  const uint32_t cnt = popc4(w0[u], sIn4[2 * g]) + popc4(w1[u], sIn4[2 * g + 1]);
                  const bool nmda = cnt >= c.dthr;
                  if (nmda) b2 |= 1u << s[u];
                  a += c.mode == 0u ? cnt : (c.mode == 1u ? (nmda ? cnt + c.boost : cnt) : (nmda ? 1u : 0u));
                }
            }
            if (facil != 0u && ((sIn[cc] >> lane) & 1u)) a += facil;
            const uint32_t bi = useBias ? (bsrc >> c.biasShift) : 0u;
            a = a > bi ? a - bi : 0u;
            __stcg(accG + cc * 32u + lane, a);
            __stcg(bbG + cc * 32u + lane, b2);
            const uint32_t drv = __reduce_add_sync(kFull, a);
            uint32_t vk, vk1;
            const uint32_t ball = warp_kwta(a, lane, kk, vk, vk1);
            if (lane == 0) {
              __stcg(xdrive + cc, drv);
              __stcg(xball + cc, ball);
              driveG[cc] = drv;
              margG[cc] = vk > vk1 ? 1u : 0u;
              sVk[warp * cpw + i] = vk;
              sVk1[warp * cpw + i] = vk1;
            }
          }
        }

        if (!grid_barrier(bar, m.err, nb + c.missing, gstep, c.waitNs, sFlag)) return;

        // ---------------- phase B: column threshold (k_topk) and the full spike vector
        {
          const uint4* xd = reinterpret_cast<const uint4*>(sNet.d.xdrive + par * ncol);
          const uint4* xb = reinterpret_cast<const uint4*>(sNet.d.xball + par * ncol);
          for (uint32_t i = tid; i < ncol / 4u; i += blockDim.x) cp_async16(reinterpret_cast<uint4*>(sD) + i, xd + i);
          cp_async_commit();
          for (uint32_t i = tid; i < ncol / 4u; i += blockDim.x) cp_async16(reinterpret_cast<uint4*>(sB) + i, xb + i);
          cp_async_commit();
          cp_async_wait<1>();
          __syncthreads();
          const uint32_t theta = block_theta(sD, incols, ncol, c.targetCols, c.topkPar, sHist, sRed, thPrev);
          thPrev = theta;
          cp_async_wait<0>();
          __syncthreads();
          emit_groups(sD, sB, sStim, sOut, sActOut, max(theta, 1u), clamp, incols, ngrp);
          __syncthreads();
          if (rank == 0 && tid == 0) { sNet.d.theta[0] = theta; sNet.d.theta[1] = 0u; }
        }

        // ---------------- phase C: own-column records, bias and learning
        {
          uint32_t* stats = sPr.stats;
          uint32_t* dlog = sPr.driveLog;
          uint32_t* hist = sPr.hist;
          const uint32_t* refBall = sPr.refBall;
          for (uint32_t i = 0; i < cpw; ++i) {
            const uint32_t cc = gw + i * nwS;
            if (cc >= ncol) break;
            const uint32_t b = sOut[cc];
            const bool recur = cc >= incols;
            const bool fired = (b >> lane) & 1u;
            const uint32_t vk = sVk[warp * cpw + i], vk1 = sVk1[warp * cpw + i];
            if (recur) {
              // stats[2] and driveLog, src/axon.mm:213-220
              const uint32_t refb = refBall ? __ldcg(refBall + cc) : 0u;
              if (stats && b != 0u) {
                const uint32_t bb = fired ? __ldcg(sNet.d.bbits + cc * 32u + lane) : 0u;
                const uint32_t coinc = __reduce_add_sync(kFull, (uint32_t)__popc(bb));
                if (lane == 0 && coinc) atomicAdd(stats + 2, coinc);
              }
              if (dlog && refb != 0u) {
                const bool member = (refb >> lane) & 1u;
                const uint32_t a = member ? __ldcg(sNet.d.acc + cc * 32u + lane) : 0u;
                const bool shared = member && __ldg(sNet.d.mult + cc * 32u + lane) > 1u;
                const uint32_t mS = __ballot_sync(kFull, member && shared), mE = __ballot_sync(kFull, member && !shared);
                const uint32_t sumS = __reduce_add_sync(kFull, (member && shared) ? a : 0u);
                const uint32_t sumE = __reduce_add_sync(kFull, (member && !shared) ? a : 0u);
                if (lane == 0) {
                  if (mS) { atomicAdd(dlog + t * 4u + 0u, sumS); atomicAdd(dlog + t * 4u + 1u, (uint32_t)__popc(mS)); }
                  if (mE) { atomicAdd(dlog + t * 4u + 2u, sumE); atomicAdd(dlog + t * 4u + 3u, (uint32_t)__popc(mE)); }
                }
              }
            }
            if (lane == 0) {
              if (hist) hist[(size_t)t * ncol + cc] = b;
              if (stats && b != 0u && recur) {  // src/axon.mm:225-234
                const uint32_t sb = 64u + t * 8u;
                atomicAdd(stats + 0, 1u);
                atomicAdd(stats + 1, (uint32_t)__popc(b));
                atomicAdd(stats + sb + 0u, vk - vk1);
                atomicAdd(stats + sb + 1u, vk);
                atomicAdd(stats + sb + 2u, 1u);
                if (vk == vk1) atomicAdd(stats + sb + 3u, 1u);
                if (vk == 0u) atomicAdd(stats + sb + 4u, 1u);
              }
            }
            if (!learn) continue;
            // (k_bias of this step runs in the next step's phase A, or after the last step)
            // k_learn, src/axon.mm:436-495: the column learns this step
            if (phase == 3u || b == 0u) continue;
            if (c.marginGate != 0u && !(vk > vk1)) continue;
            if (lane == 0) sLcol[atomicAdd(sFlag + 1, 1u)] = cc;
          }
          if (learn) {
            __syncthreads();
            const uint32_t nL = sFlag[1];
            for (uint32_t base = 0; base < nL; base += kChunk) {
              const uint32_t ncx = min(kChunk, nL - base);
              // each voted branch of a chunk column becomes one task for any warp
              for (uint32_t j = warp; j < ncx; j += wpb) {
                const uint32_t cc = sLcol[base + j];
                const uint32_t bb = __ldcg(sNet.d.bbits + cc * 32u + lane);
                const bool fired = (sOut[cc] >> lane) & 1u;
                const uint32_t vmask = __reduce_or_sync(kFull, fired ? bb : 0u);
                sBBL[j * 32u + lane] = bb;
                sLTP[j * 32u + lane] = 0u;
                sLTD[j * 32u + lane] = 0u;
                if (lane == 0) sColC[j] = cc;
                if ((vmask >> lane) & 1u) sTask[atomicAdd(sFlag + 2, 1u)] = (j << 5) | lane;
              }
              __syncthreads();
              const uint32_t ntask = sFlag[2];
              if (tid == 0) atomicAdd(m.work + 1, (unsigned long long)ntask);
              for (uint32_t k = warp; k < ntask; k += wpb) {
                const uint32_t tk = sTask[k], j = tk >> 5, s = tk & 31u;
                const uint32_t cc = sColC[j];
                const bool want = ((sOut[cc] >> lane) & 1u) && ((sBBL[j * 32u + lane] >> s) & 1u);
                const uint32_t g = __ldg(sNet.d.conn + cc * kNslot + s);
                const size_t base4 = ((size_t)cc * kNslot + s) * kTileU4 + lane;
                uint4* P0 = sNet.d.W0;
                uint4* P1 = sNet.d.W1;
                uint4* P2 = sNet.d.W2;
                uint4* P3 = sNet.d.W3;
                uint4 p0[2], p1[2], p2[2], p3[2];
#pragma unroll
                for (int jj = 0; jj < 2; ++jj) {
                  p0[jj] = __ldcg(P0 + base4 + 32 * jj);
                  p1[jj] = __ldcg(P1 + base4 + 32 * jj);
                  p2[jj] = __ldcg(P2 + base4 + 32 * jj);
                  p3[jj] = __ldcg(P3 + base4 + 32 * jj);
                }
                uint32_t nLTP = 0, nLTD = 0;
#pragma unroll
                for (int jj = 0; jj < 2; ++jj) {
                  const uint4 sp4 = sIn4[2 * g + jj];
                  learn_word(p0[jj].x, p1[jj].x, p2[jj].x, p3[jj].x, sp4.x, want, phase, t, c, nLTP, nLTD);
                  learn_word(p0[jj].y, p1[jj].y, p2[jj].y, p3[jj].y, sp4.y, want, phase, t, c, nLTP, nLTD);
                  learn_word(p0[jj].z, p1[jj].z, p2[jj].z, p3[jj].z, sp4.z, want, phase, t, c, nLTP, nLTD);
                  learn_word(p0[jj].w, p1[jj].w, p2[jj].w, p3[jj].w, sp4.w, want, phase, t, c, nLTP, nLTD);
                }
#pragma unroll
                for (int jj = 0; jj < 2; ++jj) {
                  __stcg(P0 + base4 + 32 * jj, p0[jj]);
                  __stcg(P1 + base4 + 32 * jj, p1[jj]);
                  __stcg(P2 + base4 + 32 * jj, p2[jj]);
                  __stcg(P3 + base4 + 32 * jj, p3[jj]);
                }
                if (nLTP) atomicAdd(sLTP + j * 32u + lane, nLTP);
                if (nLTD) atomicAdd(sLTD + j * 32u + lane, nLTD);
              }
              __syncthreads();
              // plasticity counters per neuron and step, src/axon.mm:491-494
              if (stats) {
                for (uint32_t j = warp; j < ncx; j += wpb) {
                  const uint32_t nLTP = sLTP[j * 32u + lane], nLTD = sLTD[j * 32u + lane];
                  const uint32_t sumP = __reduce_add_sync(kFull, nLTP), sumD = __reduce_add_sync(kFull, nLTD);
                  const uint32_t kP = __popc(__ballot_sync(kFull, nLTP != 0u));
                  const uint32_t kD = __popc(__ballot_sync(kFull, nLTD != 0u));
                  if (lane == 0) {
                    if (sumP) atomicAdd(stats + 8, sumP);
                    if (sumD) atomicAdd(stats + 9, sumD);
                    if (kP) atomicAdd(stats + 10, kP);
                    if (kD) atomicAdd(stats + 11, kD);
                  }
                }
              }
              if (tid == 0) sFlag[2] = 0u;
              __syncthreads();
            }
            if (tid == 0) sFlag[1] = 0u;
          }
        }
        __syncthreads();  // sOut / sActOut complete before the next step reads them
      }

      // ---------------- end of the presentation: k_bias of the last step, then the buffers
      // present() leaves behind
      if (learn) {
        const uint32_t* sLast = (T & 1u) ? sSpk1 : sSpk0;  // spk(T-1)
        const int dec = (((T - 1u) % max(c.biasDownEvery, 1u)) == 0u) ? (int)c.biasDown : 0;
        uint32_t* biasG = sNet.d.bias;
        const uint32_t first = gw + ((incols > gw) ? ((incols - gw + nwS - 1u) / nwS) * nwS : 0u);  // first owned recurrent column
        for (uint32_t c0 = first; c0 < ncol; c0 += 4u * nwS) {  // four columns' loads in flight
          uint32_t v[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const uint32_t cc = c0 + (uint32_t)k * nwS;
            v[k] = cc < ncol ? __ldcg(biasG + cc * 32u + lane) : 0u;
          }
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const uint32_t cc = c0 + (uint32_t)k * nwS;
            if (cc >= ncol) break;
            const int nbv = (int)v[k] + (((sLast[cc] >> lane) & 1u) ? (int)c.biasUp : -dec);
            __stcg(biasG + cc * 32u + lane, (uint32_t)max(0, nbv));
          }
        }
      }
      {
        const uint32_t* sLast = (T & 1u) ? sSpk1 : sSpk0;  // spk(T-1)
        const uint32_t* sPrev = (T & 1u) ? sSpk0 : sSpk1;  // spk(T-2), zero when T == 1
        uint32_t* gLast = ((T - 1u) & 1u) ? sNet.d.spkA : sNet.d.spkB;
        uint32_t* gPrev = ((T - 1u) & 1u) ? sNet.d.spkB : sNet.d.spkA;
        uint32_t* fin = sPr.finalOut;
        for (uint32_t cc = gw; cc < ncol; cc += nwS)
          if (lane == 0) {
            gLast[cc] = sLast[cc];
            gPrev[cc] = T >= 2u ? sPrev[cc] : 0u;
            if (fin) fin[cc] = sLast[cc];
          }
      }
      __syncthreads();
    }
  }
  if (lane == 0 && nTiles) atomicAdd(m.work, (unsigned long long)nTiles);
}

// ---------------------------------------------------------------- launch helpers
size_t multi_smem_bytes(uint32_t ncol, uint32_t incols, uint32_t maxCpw, int threads) {
  return (size_t)multi_layout(ncol, incols, (uint32_t)(threads / 32) * maxCpw).total * 4;
}

static const void* multi_fn(int threads, int tiles) {
  if (threads == 1024 && tiles == 4) return (const void*)k_multi<1024, 4>;
  if (threads == 896 && tiles == 4) return (const void*)k_multi<896, 4>;
  if (threads == 512 && tiles == 8) return (const void*)k_multi<512, 8>;
  return nullptr;
}

cudaError_t multi_max_blocks_per_sm(int threads, int tiles, size_t smem, int* out) {
  const void* fn = multi_fn(threads, tiles);
  if (!fn) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, fn, threads, smem);
}

cudaError_t launch_multi(const MultiDev& m, const MultiCfg& c, const MultiShape& s, cudaStream_t st) {
  const void* fn = multi_fn(s.threads, s.tiles);
  if (!fn) return cudaErrorInvalidValue;
  void* args[] = {(void*)&m, (void*)&c};
  return cudaLaunchCooperativeKernel(fn, dim3(s.grid), dim3(s.threads), args, s.smem, st);
}

}  // namespace axon
