// Plain AXON path on sm_100a: one persistent launch runs all T steps of a presentation.
//
// Reference: rakib-nyc/axon src/axon.mm. There, present() (src/axon.mm:815-888) encodes
// T x {k_drive, k_topk, k_emit, k_bias, k_learn} as five Metal dispatches per step. Here
// the whole step loop is one cooperative launch with ONE grid barrier per step:
//
//   phase A  each warp owns one column (lane = neuron): drive over the column's non-silent
//            branches, the exact k-of-32 ballot, and the column drive; drive + ungated
//            ballot are published, and the drive is counted into the step's histogram.
//            The W3 tiles of the non-silent branches of all the CTA's columns are in flight
//            at once: each branch's lane issues one 1 KiB TMA bulk copy into a CTA-wide
//            shared-memory pool (slots claimed per column), completed on a per-column
//            mbarrier; spikes come from shared memory.
//   barrier
//   phase B  every CTA reads all published drives/ballots (L2), selects the column
//            threshold (the target-th largest recurrent drive) and rebuilds the whole
//            spike vector spk(t) in its own shared memory; no second barrier is needed.
//   phase C  each warp finishes its own column: hist/stats/driveLog records, intrinsic
//            bias (in a register for the whole launch) and bit-serial learning on W0..W3.
//
// Per-neuron state that only its owner touches (bias, conn row, multiplicity) lives in
// registers for the whole presentation; HBM traffic per step is the W3 tiles of
// non-silent branches plus the learning read-modify-writes.
#include <cstdint>

#include "axon_device.cuh"
#include "batch_common.cuh"
#include "plain.cuh"
#include "emit.cuh"
#include "learn.cuh"
#include "theta.cuh"

namespace axon {

// LEARN is c.learn as a template argument: readout launches carry none of the learning
// code's register pressure.
template <int CPW, bool LEARN>
__global__ void __launch_bounds__(kPresentMaxWarps * 32, 1) k_present(NetDev d, PresentCfg c) {
  extern __shared__ __align__(16) uint32_t sm[];
  const uint32_t ncol = c.ncol, incols = c.incols;
  const uint32_t ngrp = ncol / 8u, nactw = (((ngrp + 31u) / 32u) + 3u) & ~3u;  // 16-byte multiple
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, wpb = blockDim.x >> 5;
  const uint32_t maxCols = wpb * CPW;      // columns owned by this CTA
  const PresentSmem L = present_smem_layout(ncol, incols, CPW);
  uint32_t* sSpk0 = sm;                    // spike vectors, ping-pong
  uint32_t* sSpk1 = sm + ncol;
  uint32_t* sAct0 = sm + 2 * ncol;         // group-activity bits, ping-pong
  uint32_t* sAct1 = sAct0 + nactw;
  uint32_t* sStim = sAct1 + nactw;         // input clamp pattern
  uint32_t* sHist = sStim + ((incols + 3u) & ~3u);  // the step's drive histogram (kHistWords)
  uint32_t* sFlag = sHist + kHistWords;    // [0] barrier flag, [1] learning-task count, [2] candidates,
                                           // [3] tile-pool slots claimed, [4..7] threshold select
  uint64_t* sMbar = reinterpret_cast<uint64_t*>(sFlag + 16);  // one per column slot (tile pool)
  uint32_t* sTask = sFlag + 16 + 2 * kMaxColSlots;  // learning tasks: (column slot << 5) | branch
  uint32_t* sBBL = sTask + maxCols * 32;   // branch-NMDA masks of the learning columns
  uint32_t* sLTP = sBBL + maxCols * 32;    // per-neuron potentiation counts of this step
  uint32_t* sLTD = sLTP + maxCols * 32;    // per-neuron depression counts
  uint32_t* sFiredL = sLTD + maxCols * 32; // spike ballot of each learning column
  uint32_t* sColL = sFiredL + maxCols;     // its column index
  uint32_t* sMark = sColL + maxCols;       // step+1 when the slot learns this step
  uint32_t* sBias = sMark + maxCols;       // intrinsic bias of each owned neuron (slot * 32 + lane)
  uint32_t* sMul = sBias + maxCols * 32;   // assembly multiplicity of each owned neuron
  uint32_t* sRef = sMul + maxCols * 32;    // reference ball of each owned column
  // phase A's tile pool; phase B reuses its start for the staged drives, the ungated
  // ballots and the threshold candidates
  uint4* sPool = reinterpret_cast<uint4*>(sm + L.poolWord);
  const uint32_t poolTiles = L.poolTiles;
  uint32_t* sD = sm + L.poolWord;          // staged drives of the current step
  uint32_t* sB = sD + ncol;                // staged ungated ballots
  uint32_t* sCand = sB + ncol;             // drives of the threshold's histogram bin (up to ncol)

  // columns are dealt to warps CTA-interleaved (column = warp * grid + CTA): the clamped
  // input columns, which all fire and learn during the clamp, spread over every CTA instead
  // of loading the first few
  const uint32_t gwarp = warp * gridDim.x + blockIdx.x, nwarps = gridDim.x * wpb;
  uint32_t* xhist = d.bar + 64;            // step t counts its recurrent drives into histogram t mod 3
  // branch term of k_drive (src/axon.mm:174-178): the count (modes 0, 1) plus, when the
  // branch reaches dthr, the boost (mode 1) or 1 (mode 2)
  const uint32_t linMask = c.mode != 2u ? kFull : 0u;
  const uint32_t addN = c.mode == 1u ? c.boost : (c.mode == 2u ? 1u : 0u);

  for (uint32_t i = tid; i < ncol; i += blockDim.x) sSpk0[i] = 0u;
  for (uint32_t i = tid; i < nactw; i += blockDim.x) sAct0[i] = 0u;
  for (uint32_t i = tid; i < maxCols; i += blockDim.x) sMark[i] = 0u;
  if (tid == 0) {
    sFlag[1] = 0u;
    sFlag[3] = 0u;
    for (uint32_t i = 0; i < maxCols; ++i) mbar_init(&sMbar[i], 1);
    fence_proxy_async_smem();
  }
  for (uint32_t i = tid; i < incols; i += blockDim.x) sStim[i] = d.stim[i];

  // the columns this warp owns and their conn rows (lane = branch) stay in registers; the
  // rest of their per-neuron state lives in shared memory by column slot (warp * CPW + i)
  uint32_t col[CPW], cn[CPW];
  uint32_t mph = 0;  // bit i: phase parity of column slot i's mbarrier
#pragma unroll
  for (int i = 0; i < CPW; ++i) {
    col[i] = gwarp + (uint32_t)i * nwarps;
    cn[i] = 0u;
    const uint32_t slot = warp * CPW + (uint32_t)i;
    if (col[i] < ncol) {
      cn[i] = d.conn[col[i] * kNslot + lane];
      sBias[slot * 32u + lane] = d.bias[col[i] * 32u + lane];
      sMul[slot * 32u + lane] = d.mult[col[i] * 32u + lane];
      if (lane == 0) sRef[slot] = d.refBall[col[i]];
    }
  }
  __syncthreads();

  // what phase A leaves for phase C; readout launches keep a step's values until its records
  // are written, during the next step's tile copies
  uint32_t acc[CPW], bb[CPW], vk[CPW], vk1[CPW];
#pragma unroll
  for (int i = 0; i < CPW; ++i) acc[i] = bb[i] = vk[i] = vk1[i] = 0u;
  // Records of column slot i for step tr, whose spike ballot is bw: the final state at the
  // last step, stats[2] and driveLog (src/axon.mm:213-220), hist and the k_emit counters
  // (src/axon.mm:224-234).
  auto records = [&](int i, uint32_t tr, uint32_t bw) {
    const uint32_t cc = col[i];
    const uint32_t slot = warp * CPW + (uint32_t)i;
    const bool recur = cc >= incols;
    const bool fired = (bw >> lane) & 1u;
    if (tr + 1u == c.T) {  // final state of the owned neurons, as present() leaves it
      d.acc[cc * 32u + lane] = acc[i];
      d.bbits[cc * 32u + lane] = bb[i];
      if (lane == 0) d.marg[cc] = vk[i] > vk1[i] ? 1u : 0u;
    }
    if (recur) {
      const uint32_t coinc = __reduce_add_sync(kFull, fired ? (uint32_t)__popc(bb[i]) : 0u);
      const bool member = (sRef[slot] >> lane) & 1u;
      const bool shared = sMul[slot * 32u + lane] > 1u;
      const uint32_t mS = __ballot_sync(kFull, member && shared), mE = __ballot_sync(kFull, member && !shared);
      const uint32_t sumS = __reduce_add_sync(kFull, (member && shared) ? acc[i] : 0u);
      const uint32_t sumE = __reduce_add_sync(kFull, (member && !shared) ? acc[i] : 0u);
      if (lane == 0) {
        if (coinc) atomicAdd(d.stats + 2, coinc);
        if (mS) { atomicAdd(d.driveLog + tr * 4u + 0u, sumS); atomicAdd(d.driveLog + tr * 4u + 1u, (uint32_t)__popc(mS)); }
        if (mE) { atomicAdd(d.driveLog + tr * 4u + 2u, sumE); atomicAdd(d.driveLog + tr * 4u + 3u, (uint32_t)__popc(mE)); }
      }
    }
    if (lane == 0) {
      d.hist[(size_t)tr * ncol + cc] = bw;
      if (bw != 0u && recur) {
        const uint32_t sb = 64u + tr * 8u;
        atomicAdd(d.stats + 0, 1u);
        atomicAdd(d.stats + 1, (uint32_t)__popc(bw));
        atomicAdd(d.stats + sb + 0u, vk[i] - vk1[i]);
        atomicAdd(d.stats + sb + 1u, vk[i]);
        atomicAdd(d.stats + sb + 2u, 1u);
        if (vk[i] == vk1[i]) atomicAdd(d.stats + sb + 3u, 1u);
        if (vk[i] == 0u) atomicAdd(d.stats + sb + 4u, 1u);
      }
    }
  };

  for (uint32_t t = 0; t < c.T; ++t) {
    const uint32_t* sIn = (t & 1u) ? sSpk1 : sSpk0;
    uint32_t* sOut = (t & 1u) ? sSpk0 : sSpk1;
    const uint32_t* sActIn = (t & 1u) ? sAct1 : sAct0;
    uint32_t* sActOut = (t & 1u) ? sAct0 : sAct1;
    const uint4* sIn4 = reinterpret_cast<const uint4*>(sIn);
    const uint32_t par = t & 1u;
    const bool clamp = t < c.clampSteps;
    const uint32_t phase = (!LEARN || !c.contrast) ? 0u
                           : (clamp ? 1u : (((t - c.clampSteps) % c.ltdEvery == 0u) ? 2u : 3u));
    if (LEARN) {
#pragma unroll
      for (int i = 0; i < CPW; ++i) acc[i] = bb[i] = vk[i] = vk1[i] = 0u;
    }

    // per-phase device timer stamps of the profile mode (thread 0 of every CTA)
    unsigned long long* stamp = d.prof ? d.prof + ((size_t)t * gridDim.x + blockIdx.x) * 5u : nullptr;
    if (stamp && tid == 0) stamp[0] = globaltimer_ns();
    // ---------------- phase A: drive (k_drive, src/axon.mm:150-190) + ungated k-WTA
    // The owner warp claims one pool slot per non-silent branch of its column; the lane of
    // each such branch issues the tile's bulk copy, so all of the CTA's tiles are in flight
    // together. A column whose claim does not fit the pool streams its tiles through
    // registers instead, four at a time. Spikes come from shared memory.
#pragma unroll
    for (int i = 0; i < CPW; ++i) {
      if (col[i] >= ncol) continue;  // warp-uniform
      const uint32_t cc = col[i];
      const bool on = (sActIn[cn[i] >> 5] >> (cn[i] & 31u)) & 1u;
      uint32_t active = __ballot_sync(kFull, on);
      const uint32_t n = (uint32_t)__popc(active);
      uint32_t a = 0, b2 = 0;
      uint32_t slot0 = 0;
      if (lane == 0 && n != 0u) slot0 = atomicAdd(sFlag + 3, n);
      slot0 = __shfl_sync(kFull, slot0, 0);
      const bool pooled = n != 0u && slot0 + n <= poolTiles;
      uint64_t* mb = &sMbar[warp * CPW + (uint32_t)i];
      if (pooled) {
        if (lane == 0) mbar_expect_tx(mb, n * 1024u);
        __syncwarp();
        if (on) {
          const uint32_t r = (uint32_t)__popc(active & ((1u << lane) - 1u));
          fence_proxy_async_smem();
          bulk_g2s(sPool + (size_t)(slot0 + r) * kTileU4, d.W3 + ((size_t)cc * kNslot + lane) * kTileU4, 1024u, mb);
        }
      }
      // a readout writes the previous step's records while this step's tiles are in flight
      if (!LEARN) {
        if (t > 0u) records(i, t - 1u, sIn[cc]);
        acc[i] = bb[i] = vk[i] = vk1[i] = 0u;
      }
      if (pooled) {
        const uint32_t ph = (mph >> i) & 1u;
        if (!mbar_wait(mb, ph, c.waitNs)) {
          // the copies did not land in time: record it, wait (bounded) for them, and let
          // the grid barrier end the launch
          if (lane == 0) atomicCAS(d.err, 0u, kErrTimeout);
          mbar_wait(mb, ph, c.waitNs > kDrainNs ? c.waitNs : kDrainNs);
        }
        mph ^= 1u << i;
        const uint4* T = sPool + (size_t)slot0 * kTileU4 + lane;
        for (uint32_t r = 0; active; ++r, T += kTileU4) {
          const uint32_t s = (uint32_t)(__ffs(active) - 1);
          active &= active - 1u;
          const uint32_t g = __shfl_sync(kFull, cn[i], s);
          const uint32_t cnt = popc4(T[0], sIn4[2 * g]) + popc4(T[32], sIn4[2 * g + 1]);
          const bool nmda = cnt >= c.dthr;
          if (nmda) b2 |= 1u << s;
          a += (cnt & linMask) + (nmda ? addN : 0u);
        }
      } else {
        const uint4* Wt = d.W3 + (size_t)cc * kNslot * kTileU4 + lane;
        while (active) {
          uint32_t s[4];
          bool v[4];
          uint4 w0[4], w1[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            v[u] = active != 0u;
            s[u] = v[u] ? (uint32_t)(__ffs(active) - 1) : 0u;
            active &= active - 1u;
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (v[u]) {
              w0[u] = __ldcg(Wt + s[u] * kTileU4);
              w1[u] = __ldcg(Wt + s[u] * kTileU4 + 32);
            }
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (v[u]) {
              const uint32_t g = __shfl_sync(kFull, cn[i], s[u]);
              const uint32_t cnt = popc4(w0[u], sIn4[2 * g]) + popc4(w1[u], sIn4[2 * g + 1]);
              const bool nmda = cnt >= c.dthr;
              if (nmda) b2 |= 1u << s[u];
              a += (cnt & linMask) + (nmda ? addN : 0u);
            }
        }
      }
      if (c.facil != 0u && ((sIn[cc] >> lane) & 1u)) a += c.facil;
      const uint32_t bi = c.useBias ? (sBias[(warp * CPW + (uint32_t)i) * 32u + lane] >> c.biasShift) : 0u;
      a = a > bi ? a - bi : 0u;
      acc[i] = a;
      bb[i] = b2;
      const uint32_t drv = __reduce_add_sync(kFull, a);
      const uint32_t ball = warp_kwta(a, lane, c.k, vk[i], vk1[i]);
      if (lane == 0) {
        __stcg(d.xdrive + par * ncol + cc, drv);
        __stcg(d.xball + par * ncol + cc, ball);
        if (cc >= incols && drv < (1u << 24)) {
          uint32_t* h = xhist + (t % 3u) * kHistWords + theta_key(drv);
          atomicAdd(h, 1u);
          atomicMax(h + kThetaBins, drv);
          atomicMax(h + 2u * kThetaBins, ~drv);
        }
        if (t + 1u == c.T) d.drive[cc] = drv;  // final state: the last step's column drive
      }
    }

    if (stamp) {
      __syncthreads();
      if (tid == 0) stamp[1] = globaltimer_ns();
    }
    if (!grid_barrier(d.bar, d.err, gridDim.x + c.missing, t, c.waitNs, sFlag)) return;
    if (stamp && tid == 0) stamp[2] = globaltimer_ns();

    // ---------------- phase B: column threshold (k_topk) and the full spike vector
    // this step's drive histogram, the drives and the ballots come from L2 by asynchronous
    // copies, in that order (three groups): warp 0 scans the histogram while the drives and
    // ballots keep arriving
    for (uint32_t i = tid; i < kHistWords / 4u; i += blockDim.x)
      cp_async16(reinterpret_cast<uint4*>(sHist) + i, reinterpret_cast<const uint4*>(xhist + (t % 3u) * kHistWords) + i);
    cp_async_commit();
    for (uint32_t i = tid; i < ncol / 4u; i += blockDim.x)
      cp_async16(reinterpret_cast<uint4*>(sD) + i, reinterpret_cast<const uint4*>(d.xdrive + par * ncol) + i);
    cp_async_commit();
    for (uint32_t i = tid; i < ncol / 4u; i += blockDim.x)
      cp_async16(reinterpret_cast<uint4*>(sB) + i, reinterpret_cast<const uint4*>(d.xball + par * ncol) + i);
    cp_async_commit();
    if (tid == 0) { sFlag[2] = 0u; sFlag[3] = 0u; }  // every warp has claimed its pool slots
    // histogram t+2 (last read in step t-1, before this barrier) is cleared for its next use
    if (blockIdx.x == 0 && t >= 1u)
      for (uint32_t i = tid; i < kHistWords; i += blockDim.x) __stcg(xhist + ((t + 2u) % 3u) * kHistWords + i, 0u);
    cp_async_wait<2>();  // the histogram
    __syncthreads();
    const uint32_t theta = hist_theta<1>(sD, sHist, sCand, sFlag + 2, incols, ncol, c.targetCols, c.topkPar);
    const uint32_t gate = max(theta, 1u);
    cp_async_wait<0>();
    __syncthreads();
    emit_groups(sD, sB, sStim, sOut, sActOut, gate, clamp, incols, ngrp);
    __syncthreads();
    if (blockIdx.x == 0 && tid == 0) { d.theta[0] = theta; d.theta[1] = 0u; }

    if (stamp && tid == 0) stamp[3] = globaltimer_ns();
    // ---------------- phase C: own-column records, bias and learning
#pragma unroll
    for (int i = 0; i < CPW; ++i) {
      if (col[i] >= ncol) continue;
      const uint32_t cc = col[i];
      const uint32_t slot = warp * CPW + (uint32_t)i;
      const uint32_t b = sOut[cc];
      const bool recur = cc >= incols;
      const bool fired = (b >> lane) & 1u;
      if (!LEARN) continue;  // a readout's records wait for the next step's tile copies
      records(i, t, b);
      // k_bias, src/axon.mm:240-253
      if (recur) {
        const int dec = ((t % max(c.biasDownEvery, 1u)) == 0u) ? (int)c.biasDown : 0;
        const int nb = (int)sBias[slot * 32u + lane] + (fired ? (int)c.biasUp : -dec);
        sBias[slot * 32u + lane] = (uint32_t)max(0, nb);
      }
      // k_learn, src/axon.mm:436-495: each voted branch of a learning column becomes a
      // task that any warp of the CTA runs, so a column's read-modify-writes overlap
      if (phase == 3u || b == 0u) continue;
      if (c.marginGate != 0u && !(vk[i] > vk1[i])) continue;
      const uint32_t vmask = __reduce_or_sync(kFull, fired ? bb[i] : 0u);
      sBBL[slot * 32u + lane] = bb[i];
      sLTP[slot * 32u + lane] = 0u;
      sLTD[slot * 32u + lane] = 0u;
      if (lane == 0) { sFiredL[slot] = b; sColL[slot] = cc; sMark[slot] = t + 1u; }
      if ((vmask >> lane) & 1u) sTask[atomicAdd(sFlag + 1, 1u)] = (slot << 5) | lane;
    }
    if (LEARN) {
      __syncthreads();
      const uint32_t ntask = sFlag[1];
      for (uint32_t k = warp; k < ntask; k += wpb) {
        const uint32_t tk = sTask[k], slot = tk >> 5, s = tk & 31u;
        const uint32_t cc = sColL[slot];
        const bool want = ((sFiredL[slot] >> lane) & 1u) && ((sBBL[slot * 32u + lane] >> s) & 1u);
        const uint32_t g = __ldg(d.conn + cc * kNslot + s);
        const size_t base = ((size_t)cc * kNslot + s) * kTileU4 + lane;
        uint4 p0[2], p1[2], p2[2], p3[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          p0[j] = __ldcg(d.W0 + base + 32 * j);
          p1[j] = __ldcg(d.W1 + base + 32 * j);
          p2[j] = __ldcg(d.W2 + base + 32 * j);
          p3[j] = __ldcg(d.W3 + base + 32 * j);
        }
        uint32_t nLTP = 0, nLTD = 0;
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const uint4 sp4 = sIn4[2 * g + j];
          learn_word(p0[j].x, p1[j].x, p2[j].x, p3[j].x, sp4.x, want, phase, t, c, nLTP, nLTD);
          learn_word(p0[j].y, p1[j].y, p2[j].y, p3[j].y, sp4.y, want, phase, t, c, nLTP, nLTD);
          learn_word(p0[j].z, p1[j].z, p2[j].z, p3[j].z, sp4.z, want, phase, t, c, nLTP, nLTD);
          learn_word(p0[j].w, p1[j].w, p2[j].w, p3[j].w, sp4.w, want, phase, t, c, nLTP, nLTD);
        }
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          __stcg(d.W0 + base + 32 * j, p0[j]);
          __stcg(d.W1 + base + 32 * j, p1[j]);
          __stcg(d.W2 + base + 32 * j, p2[j]);
          __stcg(d.W3 + base + 32 * j, p3[j]);
        }
        if (nLTP) atomicAdd(sLTP + slot * 32u + lane, nLTP);
        if (nLTD) atomicAdd(sLTD + slot * 32u + lane, nLTD);
      }
      __syncthreads();
      // plasticity counters per neuron and step, src/axon.mm:491-494
#pragma unroll
      for (int i = 0; i < CPW; ++i) {
        const uint32_t slot = warp * CPW + (uint32_t)i;
        if (col[i] >= ncol || sMark[slot] != t + 1u) continue;
        const uint32_t nLTP = sLTP[slot * 32u + lane], nLTD = sLTD[slot * 32u + lane];
        const uint32_t sumP = __reduce_add_sync(kFull, nLTP), sumD = __reduce_add_sync(kFull, nLTD);
        const uint32_t kP = __popc(__ballot_sync(kFull, nLTP != 0u)), kD = __popc(__ballot_sync(kFull, nLTD != 0u));
        if (lane == 0) {
          if (sumP) atomicAdd(d.stats + 8, sumP);
          if (sumD) atomicAdd(d.stats + 9, sumD);
          if (kP) atomicAdd(d.stats + 10, kP);
          if (kD) atomicAdd(d.stats + 11, kD);
        }
      }
      if (tid == 0) sFlag[1] = 0u;
    }
    __syncthreads();  // sOut / sActOut complete before the next step reads them
    if (stamp && tid == 0) stamp[4] = globaltimer_ns();
  }

  // ---------------- final state, as the reference's buffers hold it after present()
  const uint32_t T = c.T;
  const uint32_t* sLast = (T & 1u) ? sSpk1 : sSpk0;   // spk(T-1)
  if (!LEARN) {  // the last step's records
#pragma unroll
    for (int i = 0; i < CPW; ++i)
      if (col[i] < ncol) records(i, T - 1u, sLast[col[i]]);
  }
  const uint32_t* sPrev = (T & 1u) ? sSpk0 : sSpk1;   // spk(T-2), zero when T == 1
  uint32_t* gLast = ((T - 1u) & 1u) ? d.spkA : d.spkB;
  uint32_t* gPrev = ((T - 1u) & 1u) ? d.spkB : d.spkA;
#pragma unroll
  for (int i = 0; i < CPW; ++i) {
    if (col[i] >= ncol) continue;
    const uint32_t cc = col[i];
    if (LEARN) d.bias[cc * 32u + lane] = sBias[(warp * CPW + (uint32_t)i) * 32u + lane];
    if (lane == 0) {
      gLast[cc] = sLast[cc];
      gPrev[cc] = T >= 2u ? sPrev[cc] : 0u;
      if (d.finalOut) d.finalOut[cc] = sLast[cc];
    }
  }
}

// ---------------------------------------------------------------- launch helpers
size_t present_smem_bytes(uint32_t ncol, uint32_t incols, int cpw) {
  return present_smem_layout(ncol, incols, cpw).bytes;
}

static const void* present_fn(int cpw, bool learn) {
  switch (cpw) {
    case 1: return learn ? (const void*)k_present<1, true> : (const void*)k_present<1, false>;
    case 2: return learn ? (const void*)k_present<2, true> : (const void*)k_present<2, false>;
    default: return nullptr;
  }
}

cudaError_t launch_present(const NetDev& d, const PresentCfg& c, const LaunchShape& ls, cudaStream_t st) {
  void* args[] = {(void*)&d, (void*)&c};
  const void* fn = present_fn(ls.cpw, c.learn != 0u);
  if (!fn) return cudaErrorInvalidValue;
  // barrier counter and the three drive histograms start at zero
  const cudaError_t e = cudaMemsetAsync(d.bar, 0, kBarRegionWords * 4u, st);
  if (e != cudaSuccess) return e;
  return cudaLaunchCooperativeKernel(fn, dim3(ls.grid), dim3(ls.wpb * 32), args, ls.smem, st);
}

// Sets the shared-memory size of both forms (learning, readout) and returns the smaller
// number of co-resident blocks per SM.
cudaError_t present_max_blocks_per_sm(int cpw, int threads, size_t smem, int* out) {
  *out = 0;
  int best = 1 << 30;
  for (bool learn : {false, true}) {
    const void* fn = present_fn(cpw, learn);
    if (!fn) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int n = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, smem);
    if (e != cudaSuccess) return e;
    best = n < best ? n : best;
  }
  *out = best;
  return cudaSuccess;
}

// ---------------------------------------------------------------- init kernels
// k_init_w, src/axon.mm:86-104: one thread per uint4 of each plane.
__global__ void k_init_w(uint4* W0, uint4* W1, uint4* W2, uint4* W3, uint32_t nAnd, uint32_t seed, uint64_t nU4) {
  const uint64_t gg = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gg >= nU4) return;
  const uint32_t g = (uint32_t)gg ^ (seed * 0x9E3779B9u);
  uint32_t m0 = kFull, m1 = kFull, m2 = kFull, m3 = kFull;
  for (uint32_t i = 0; i < nAnd; ++i) {
    m0 &= hash32(g * 32u + i * 4u + 0u);
    m1 &= hash32(g * 32u + i * 4u + 1u);
    m2 &= hash32(g * 32u + i * 4u + 2u);
    m3 &= hash32(g * 32u + i * 4u + 3u);
  }
  const uint4 m = make_uint4(m0, m1, m2, m3);
  const uint4 cc = make_uint4(hash32(g * 8u + 11u), hash32(g * 8u + 13u), hash32(g * 8u + 17u), hash32(g * 8u + 19u));
  W3[gg] = m;
  W2[gg] = make_uint4(~m.x | cc.x, ~m.y | cc.y, ~m.z | cc.z, ~m.w | cc.w);
  W1[gg] = cc;
  W0[gg] = make_uint4(~cc.x, ~cc.y, ~cc.z, ~cc.w);
}
// k_init_conn, src/axon.mm:109-117
__global__ void k_init_conn(uint32_t* conn, uint32_t nGrp, uint32_t nInGrp, uint32_t inBr, uint32_t seed, uint32_t n) {
  const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const uint32_t s = g % kNslot;
  const uint32_t h = hash32(g * 2246822519u + 7u + seed * 2654435761u);
  conn[g] = (s < inBr) ? (h % nInGrp) : (nInGrp + h % (nGrp - nInGrp));
}

cudaError_t launch_init(const NetDev& d, uint32_t ncol, uint32_t incols, uint32_t inbr, uint32_t nand, uint32_t seed,
                        cudaStream_t st) {
  const uint64_t nU4 = (uint64_t)ncol * kNslot * kTileU4;
  k_init_w<<<(unsigned)((nU4 + 255) / 256), 256, 0, st>>>(d.W0, d.W1, d.W2, d.W3, nand, seed, nU4);
  const uint32_t n = ncol * kNslot;
  k_init_conn<<<(n + 255) / 256, 256, 0, st>>>(d.conn, ncol / 8u, incols / 8u, inbr, seed, n);
  return cudaGetLastError();
}

// ---------------------------------------------------------------- diagnostics
// k_wstat, src/axon.mm:641-646
__global__ void k_wstat(const uint4* W3, uint64_t nU4, uint32_t* out) {
  uint32_t s = 0;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nU4; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint4 w = __ldcs(W3 + i);
    s += __popc(w.x) + __popc(w.y) + __popc(w.z) + __popc(w.w);
  }
  s = __reduce_add_sync(kFull, s);
  if ((threadIdx.x & 31u) == 0u) atomicAdd(out, s);
}

// k_within, src/axon.mm:524-562: warp per column, lane per postsynaptic neuron.
__global__ void k_within(const uint4* W3, const uint32_t* conn, const uint32_t* ball, uint32_t inBr, uint32_t inCols,
                         uint32_t ncol, uint32_t useMask, const uint32_t* postMask, const uint32_t* mult, uint32_t* out) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t colw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (colw >= ncol || colw < inCols) return;
  const uint32_t gid = colw * 32u + lane;
  bool sel = useMask ? (postMask[gid] != 0u) : (((ball[colw] >> lane) & 1u) != 0u);
  uint32_t fIn = 0, pIn = 0, fOut = 0, pOut = 0;
  if (sel) {
    const uint4* ballV = reinterpret_cast<const uint4*>(ball);
    for (uint32_t s = inBr; s < kNslot; ++s) {
      const uint32_t g = conn[colw * kNslot + s];
      for (uint32_t j = 0; j < 2; ++j) {
        const uint4 ap = ballV[2 * g + j];
        const uint4 w = W3[((size_t)colw * kNslot + s) * kTileU4 + 32 * j + lane];
        fIn += popc4(w, ap);
        pIn += __popc(ap.x) + __popc(ap.y) + __popc(ap.z) + __popc(ap.w);
        const uint4 nap = make_uint4(~ap.x, ~ap.y, ~ap.z, ~ap.w);
        fOut += popc4(w, nap);
        pOut += __popc(nap.x) + __popc(nap.y) + __popc(nap.z) + __popc(nap.w);
      }
    }
    atomicAdd(out + 0, fIn); atomicAdd(out + 1, pIn); atomicAdd(out + 2, fOut); atomicAdd(out + 3, pOut);
    const uint32_t m = mult ? mult[gid] : 0u;
    const uint32_t b = m > 1u ? 4u : 6u;
    atomicAdd(out + b, fIn); atomicAdd(out + b + 1, pIn);
    atomicAdd(out + (m > 1u ? 8u : 9u), 1u);
  }
}

// k_indeg, src/axon.mm:566-581 and k_untouched, src/axon.mm:501-519 (which = 0 / 1)
__global__ void k_indeg_untouched(const uint4* W0, const uint4* W1, const uint4* W2, const uint4* W3, uint32_t inBr,
                                  uint32_t ncol, uint32_t which, uint32_t* out) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t colw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (colw >= ncol) return;
  uint32_t r = 0;
  for (uint32_t s = inBr; s < kNslot; ++s)
    for (uint32_t j = 0; j < 2; ++j) {
      const size_t idx = ((size_t)colw * kNslot + s) * kTileU4 + 32 * j + lane;
      const uint4 a3 = W3[idx];
      if (which == 0u) {
        r += __popc(a3.x) + __popc(a3.y) + __popc(a3.z) + __popc(a3.w);
      } else {
        const uint4 a0 = W0[idx], a1 = W1[idx], a2 = W2[idx];
        const uint32_t x[4] = {a0.x, a0.y, a0.z, a0.w}, y[4] = {a1.x, a1.y, a1.z, a1.w},
                       z[4] = {a2.x, a2.y, a2.z, a2.w}, w[4] = {a3.x, a3.y, a3.z, a3.w};
        for (int q = 0; q < 4; ++q) {
          const uint32_t v5 = ~w[q] & z[q] & ~y[q] & x[q], v6 = ~w[q] & z[q] & y[q] & ~x[q];
          r += __popc(v5 | v6);
        }
      }
    }
  out[colw * 32u + lane] = r;
}

// k_wdiag, src/axon.mm:591-638
__global__ void k_wdiag(const uint4* W0, const uint4* W1, const uint4* W2, const uint4* W3, const uint32_t* conn,
                        const uint32_t* memb, const uint32_t* asmSpk, uint32_t nstim, uint32_t inBr, uint32_t sel,
                        uint32_t ncol, uint32_t* hist) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t colw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (colw >= ncol) return;
  const uint32_t mypost = memb[colw * 32u + lane];
  if (mypost == 0u) return;
  uint32_t acc[48];
  for (int i = 0; i < 48; ++i) acc[i] = 0u;
  for (uint32_t s = 0; s < kNslot; ++s) {
    const bool isAff = s < inBr;
    if (sel == 0u && isAff) continue;
    if (sel == 1u && !isAff) continue;
    const uint32_t g = conn[colw * kNslot + s];
    for (uint32_t j = 0; j < 2; ++j) {
      const size_t idx = ((size_t)colw * kNslot + s) * kTileU4 + 32 * j + lane;
      const uint4 A0 = W0[idx], A1 = W1[idx], A2 = W2[idx], A3 = W3[idx];
      const uint32_t a0[4] = {A0.x, A0.y, A0.z, A0.w}, a1[4] = {A1.x, A1.y, A1.z, A1.w},
                     a2[4] = {A2.x, A2.y, A2.z, A2.w}, a3[4] = {A3.x, A3.y, A3.z, A3.w};
      for (int q = 0; q < 4; ++q) {
        uint32_t within = 0, anyp = 0;
        for (uint32_t qq = 0; qq < nstim; ++qq) {
          const uint32_t ap = asmSpk[(size_t)qq * ncol + 8u * g + 4u * j + q];
          anyp |= ap;
          if ((mypost >> qq) & 1u) within |= ap;
        }
        const uint32_t between = anyp & ~within;
        for (uint32_t v = 0; v < 16u; ++v) {
          const uint32_t eq = ((v & 1u) ? a0[q] : ~a0[q]) & ((v & 2u) ? a1[q] : ~a1[q]) & ((v & 4u) ? a2[q] : ~a2[q]) &
                              ((v & 8u) ? a3[q] : ~a3[q]);
          acc[v] += __popc(eq & within);
          acc[16 + v] += __popc(eq & between);
          acc[32 + v] += __popc(eq);
        }
      }
    }
  }
  for (int i = 0; i < 48; ++i)
    if (acc[i]) atomicAdd(hist + i, acc[i]);
}

// k_bstest, src/axon.mm:424-434: one thread per 32-synapse word
__global__ void k_bstest(uint32_t* A0, uint32_t* A1, uint32_t* A2, uint32_t* A3, const uint32_t* M, uint32_t op,
                         uint32_t lo, uint32_t hi, uint64_t n) {
  const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  uint32_t a0 = A0[g], a1 = A1[g], a2 = A2[g], a3 = A3[g];
  if (op == 0u) bs_inc(a0, a1, a2, a3, M[g]);
  else if (op == 1u) bs_dec(a0, a1, a2, a3, M[g]);
  else bs_clip(a0, a1, a2, a3, lo, hi);
  A0[g] = a0; A1[g] = a1; A2[g] = a2; A3[g] = a3;
}

// The kernels' k-of-32 (warp_kwta, src/axon.mm:134-144) on n columns of 32 values, one warp
// per column: out[3i..3i+2] = winners ballot, vk, vk1.
__global__ void k_kwtatest(const uint32_t* v, const uint32_t* k, uint32_t* out, uint32_t n) {
  const uint32_t lane = threadIdx.x & 31u, col = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (col >= n) return;  // whole warps
  uint32_t vk, vk1;
  const uint32_t ball = warp_kwta(v[(size_t)col * 32u + lane], lane, k[col], vk, vk1);
  if (lane == 0) {
    out[3u * col] = ball;
    out[3u * col + 1u] = vk;
    out[3u * col + 2u] = vk1;
  }
}

cudaError_t launch_wstat(const NetDev& d, uint32_t ncol, uint32_t* out, cudaStream_t st) {
  const uint64_t nU4 = (uint64_t)ncol * kNslot * kTileU4;
  k_wstat<<<148 * 8, 256, 0, st>>>(d.W3, nU4, out);
  return cudaGetLastError();
}
cudaError_t launch_within(const NetDev& d, uint32_t ncol, uint32_t inBr, uint32_t inCols, const uint32_t* ball,
                          uint32_t useMask, const uint32_t* postMask, const uint32_t* mult, uint32_t* out,
                          cudaStream_t st) {
  k_within<<<(ncol * 32 + 255) / 256, 256, 0, st>>>(d.W3, d.conn, ball, inBr, inCols, ncol, useMask, postMask, mult, out);
  return cudaGetLastError();
}
cudaError_t launch_indeg_untouched(const NetDev& d, uint32_t ncol, uint32_t inBr, uint32_t which, uint32_t* out,
                                   cudaStream_t st) {
  k_indeg_untouched<<<(ncol * 32 + 255) / 256, 256, 0, st>>>(d.W0, d.W1, d.W2, d.W3, inBr, ncol, which, out);
  return cudaGetLastError();
}
cudaError_t launch_wdiag(const NetDev& d, uint32_t ncol, const uint32_t* memb, const uint32_t* asmSpk, uint32_t nstim,
                         uint32_t inBr, uint32_t sel, uint32_t* hist, cudaStream_t st) {
  k_wdiag<<<(ncol * 32 + 127) / 128, 128, 0, st>>>(d.W0, d.W1, d.W2, d.W3, d.conn, memb, asmSpk, nstim, inBr, sel, ncol,
                                                  hist);
  return cudaGetLastError();
}
cudaError_t launch_bstest(uint32_t* a0, uint32_t* a1, uint32_t* a2, uint32_t* a3, const uint32_t* m, uint32_t op,
                          uint32_t lo, uint32_t hi, uint64_t n, cudaStream_t st) {
  k_bstest<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a0, a1, a2, a3, m, op, lo, hi, n);
  return cudaGetLastError();
}
cudaError_t launch_kwtatest(const uint32_t* v, const uint32_t* k, uint32_t* out, uint32_t n, cudaStream_t st) {
  k_kwtatest<<<(n + 7u) / 8u, 256, 0, st>>>(v, k, out, n);
  return cudaGetLastError();
}

}  // namespace axon
