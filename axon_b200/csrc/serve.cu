// Recall-serving tick: one readout step for every admitted trajectory.
//
// The step is k_drive + k_topk + k_emit of src/axon.mm:150-236 with learn = 0 (no bias, no
// learning), exactly as the plain kernel runs a readout. Trajectories start and end at
// any tick, so each carries its own local step: it reads spk(t-1) from its slot (all zero
// at t = 0) and writes spk(t) into the other half of its ping-pong pair.
//
// k_serve_drive: a warp takes one (group of up to kServeGroup trajectories of one network, column)
// item. It loads each W3 tile that any member needs once and applies it to every member
// whose presynaptic group is active, so the weights are read once per column per group
// instead of once per trajectory; it writes each member's per-neuron drives and column drive.
// k_serve_emit: a CTA per trajectory selects the column threshold over its drive vector,
// runs the exact k-of-32 only for the columns that pass the gate (the others cannot spike),
// and writes the spike vector and group-activity bits; a trajectory on its last step also
// copies its final spikes to the done buffer.
#include <cstdint>

#include "axon_device.cuh"
#include "serve.cuh"
#include "theta.cuh"

namespace axon {

constexpr int kServeThreads = 256;
constexpr int kEmitThreads = 1024;     // one trajectory per CTA at a time: a full SM's warps
constexpr uint32_t kEmitChunk = 256;   // gated columns whose per-neuron drives are staged at once

// Spike vectors and activity bits were written by the previous tick's emit kernel and are
// read-only here, so they are read through the non-coherent L1 path.
__global__ void __launch_bounds__(kServeThreads, 4) k_serve_drive(ServeDev d, ServeCfg c) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t ncol = c.ncol, ngroups = d.counts[1];
  const uint64_t items = (uint64_t)ngroups * ncol;
  for (uint64_t it = gwarp; it < items; it += nwarps) {
    const uint32_t gi = (uint32_t)(it / ncol), cc = (uint32_t)(it % ncol);
    const ServeGroup& G = d.grp[gi];
    const ServeNet net = d.nets[G.net];
    const uint32_t cn = __ldg(net.conn + cc * kNslot + lane);
    const uint32_t n = G.n;
    uint32_t actm[kServeGroup], acc[kServeGroup];
    const uint32_t* spkIn[kServeGroup];
    uint32_t uni = 0;
#pragma unroll
    for (int j = 0; j < (int)kServeGroup; ++j) {
      actm[j] = 0u;
      acc[j] = 0u;
      spkIn[j] = nullptr;
      if ((uint32_t)j < n) {
        const ServeEntry e = d.ent[G.e[j]];
        if (e.tloc > 0u) {  // spk(t-1) and its group-activity bits
          const uint32_t* base = d.slots + (size_t)e.slot * d.slotWords;
          const uint32_t par = (e.tloc - 1u) & 1u;
          spkIn[j] = base + par * ncol;
          const uint32_t* act = base + 2u * ncol + par * d.nactw;
          actm[j] = __ballot_sync(kFull, (__ldg(act + (cn >> 5)) >> (cn & 31u)) & 1u);
        }
      }
      uni |= actm[j];
    }
    const uint4* Wt = net.W3 + (size_t)cc * kNslot * kTileU4 + lane;
    while (uni) {
      uint32_t s[4];
      bool v[4];
      uint4 w0[4], w1[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        v[u] = uni != 0u;
        s[u] = v[u] ? (uint32_t)(__ffs(uni) - 1) : 0u;
        uni &= uni - 1u;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (v[u]) {
          w0[u] = __ldg(Wt + s[u] * kTileU4);
          w1[u] = __ldg(Wt + s[u] * kTileU4 + 32);
        }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        if (!v[u]) continue;
        const uint32_t g = __shfl_sync(kFull, cn, s[u]);
#pragma unroll
        for (int j = 0; j < (int)kServeGroup; ++j) {
          if (!((actm[j] >> s[u]) & 1u)) continue;  // warp-uniform
          const uint4* sp = reinterpret_cast<const uint4*>(spkIn[j]);
          const uint32_t cnt = popc4(w0[u], __ldg(sp + 2 * g)) + popc4(w1[u], __ldg(sp + 2 * g + 1));
          const bool nmda = cnt >= c.dthr;
          acc[j] += c.mode == 0u ? cnt : (c.mode == 1u ? (nmda ? cnt + c.boost : cnt) : (nmda ? 1u : 0u));
        }
      }
    }
#pragma unroll
    for (int j = 0; j < (int)kServeGroup; ++j) {
      if ((uint32_t)j >= n) break;
      uint32_t a = acc[j];
      if (c.facil != 0u && spkIn[j] && ((__ldg(spkIn[j] + cc) >> lane) & 1u)) a += c.facil;
      const uint32_t drv = __reduce_add_sync(kFull, a);
      uint32_t* base = d.slots + (size_t)d.ent[G.e[j]].slot * d.slotWords;
      if (c.acc32) __stcg(base + serve_acc_off(ncol) + cc * 32u + lane, a);
      else __stcg(reinterpret_cast<unsigned short*>(base + serve_acc_off(ncol)) + cc * 32u + lane, (unsigned short)a);
      if (lane == 0) __stcg(base + 2u * ncol + 2u * d.nactw + cc, drv);  // xdrive
    }
  }
}

__global__ void __launch_bounds__(kEmitThreads) k_serve_emit(ServeDev d, ServeCfg c) {
  extern __shared__ __align__(16) uint32_t sm[];
  const uint32_t ncol = c.ncol, incols = c.incols, ngrp = ncol / 8u;
  uint32_t* sD = sm;
  uint32_t* sSpk = sD + ncol;
  uint32_t* sList = sSpk + ncol;  // threshold candidates, then the gated columns
  uint32_t* sStim = sList + ncol;
  uint32_t* sHist = sStim + ((incols + 3u) & ~3u);
  uint32_t* sRed = sHist + 256;
  uint32_t* sAccS = sRed + 192;                    // per-neuron drives of up to kEmitChunk gated columns
  uint32_t* sCnt = sAccS + kEmitChunk * 32u;       // [0] gated columns
  const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nw = blockDim.x >> 5;
  const uint32_t nent = d.counts[0];
  // work units: (trajectory, part). Every part selects the threshold over all drives; then
  // it handles the columns of its own range, a multiple of 256 columns (whole groups and
  // whole activity words), so the parts of a trajectory write disjoint data.
  const uint32_t P = max(d.emitParts, 1u);
  const uint32_t span = ((ncol + P * 256u - 1u) / (P * 256u)) * 256u;
  for (uint32_t u = blockIdx.x; u < nent * P; u += gridDim.x) {
    const uint32_t ei = u / P, part = u - ei * P;
    const uint32_t c0 = min(part * span, ncol), c1 = min(c0 + span, ncol);
    const ServeEntry e = d.ent[ei];
    uint32_t* base = d.slots + (size_t)e.slot * d.slotWords;
    const uint32_t* xdrive = base + 2u * ncol + 2u * d.nactw;
    for (uint32_t i = tid; i < ncol / 4u; i += blockDim.x)
      cp_async16(reinterpret_cast<uint4*>(sD) + i, reinterpret_cast<const uint4*>(xdrive) + i);
    cp_async_commit();
    const bool clamp = e.tloc < e.clamp;
    if (tid == 0) sCnt[0] = 0u;
    if (clamp) {  // clamp words of the cue (src/axon.mm:800-804: 0xFFFFFFFF on the cue's columns)
      for (uint32_t i = tid; i < incols; i += blockDim.x) sStim[i] = 0u;
      __syncthreads();
      for (uint32_t i = tid; i < e.ncue; i += blockDim.x) {
        const uint32_t col = d.cues[e.cueOff + i];
        if (col < incols) sStim[col] = 0xFFFFFFFFu;
      }
    }
    cp_async_wait<0>();
    __syncthreads();
    const uint32_t theta = block_theta(sD, incols, ncol, c.targetCols, c.topkPar, sHist, sRed, 0u);
    const uint32_t gate = max(theta, 1u);
    // k_emit's gate and clamp (src/axon.mm:211-212): clamped input columns take the cue,
    // other columns spike only when their drive reaches the gate
    for (uint32_t cc = c0 + tid; cc < c1; cc += blockDim.x) {
      uint32_t v = 0u;
      if (clamp && cc < incols) v = sStim[cc];
      else if (sD[cc] >= gate) sList[atomicAdd(sCnt, 1u)] = cc;
      sSpk[cc] = v;
    }
    __syncthreads();
    const uint32_t npend = sCnt[0];
    // exact k-of-32 of the gated columns: their per-neuron drives are staged in shared
    // memory, all copies of a chunk in flight at once, then each warp takes columns
    const uint32_t rowB = c.acc32 ? 128u : 64u, pieces = rowB / 16u;
    const char* accB = reinterpret_cast<const char*>(base + serve_acc_off(ncol));
    for (uint32_t p0 = 0; p0 < npend; p0 += kEmitChunk) {
      const uint32_t np = min(kEmitChunk, npend - p0);
      for (uint32_t i = tid; i < np * pieces; i += blockDim.x) {
        const uint32_t p = i / pieces, q = i - p * pieces;
        cp_async16(reinterpret_cast<char*>(sAccS) + p * rowB + q * 16u, accB + (size_t)sList[p0 + p] * rowB + q * 16u);
      }
      cp_async_commit();
      cp_async_wait<0>();
      __syncthreads();
      for (uint32_t p = warp; p < np; p += nw) {
        const uint32_t cc = sList[p0 + p];
        const uint32_t a = c.acc32 ? sAccS[p * 32u + lane] : (uint32_t)reinterpret_cast<const unsigned short*>(sAccS)[p * 32u + lane];
        uint32_t vk, vk1;
        const uint32_t ball = warp_kwta(a, lane, c.k, vk, vk1);
        if (lane == 0) sSpk[cc] = ball;
      }
      __syncthreads();
    }
    uint32_t* spkOut = base + (e.tloc & 1u) * ncol;
    uint32_t* actOut = base + 2u * ncol + (e.tloc & 1u) * d.nactw;
    uint4* dst = e.done != 0xFFFFFFFFu ? reinterpret_cast<uint4*>(d.doneBuf + (size_t)e.done * ncol) : nullptr;
    for (uint32_t i = c0 / 4u + tid; i < c1 / 4u; i += blockDim.x) {
      const uint4 v = reinterpret_cast<const uint4*>(sSpk)[i];
      __stcg(reinterpret_cast<uint4*>(spkOut) + i, v);
      if (dst) dst[i] = v;
    }
    if (e.nextIdx != 0xFFFFFFFFu) {  // entry lists of the next tick: groups with spikes, their nonzero words
      const ServeNet net = d.nets[e.net];
      const uint32_t q = d.par ^ 1u;
      uint2* e1Out = net.ent1 + (size_t)q * ngrp * kServeMaxB;
      uint4* eMOut = net.entM + (size_t)q * ngrp * kServeMaxB;
      uint32_t* c1Out = net.ecnt + (size_t)q * 2 * ngrp;
      uint32_t* cMOut = c1Out + ngrp;
      for (uint32_t g = c0 / 8u + tid; g < c1 / 8u; g += blockDim.x) {
        const uint4 p = reinterpret_cast<const uint4*>(sSpk)[2 * g], q4 = reinterpret_cast<const uint4*>(sSpk)[2 * g + 1];
        const uint32_t w[8] = {p.x, p.y, p.z, p.w, q4.x, q4.y, q4.z, q4.w};
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
          const uint32_t at = atomicAdd(c1Out + g, 1u);
          __stcg(e1Out + (size_t)g * kServeMaxB + at, make_uint2(e.nextIdx | (w0 << 16), S0));
        } else if (k > 1) {
          const uint32_t at = atomicAdd(cMOut + g, 1u);
          __stcg(eMOut + (size_t)g * kServeMaxB + at, make_uint4(e.nextIdx | (nz << 16), S0, S1, S2));
        }
      }
    }
    for (uint32_t gb = c0 / 8u + warp * 32u; gb < c1 / 8u; gb += nw * 32u) {  // group-activity bits
      const uint32_t g = gb + lane;
      bool any = false;
      if (g < c1 / 8u) {
        const uint4 p = reinterpret_cast<const uint4*>(sSpk)[2 * g], q = reinterpret_cast<const uint4*>(sSpk)[2 * g + 1];
        any = (p.x | p.y | p.z | p.w | q.x | q.y | q.z | q.w) != 0u;
      }
      const uint32_t wv = __ballot_sync(kFull, any);
      if (lane == 0) __stcg(actOut + (gb >> 5), wv);
    }
    __syncthreads();
  }
}

size_t serve_emit_smem_bytes(uint32_t ncol, uint32_t incols) {
  return (3ull * ncol + ((incols + 3u) & ~3u) + 256 + 192 + kEmitChunk * 32ull + 4) * 4;
}

cudaError_t serve_prepare(size_t emitSmem) {
  return cudaFuncSetAttribute(k_serve_emit, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)emitSmem);
}

// list lengths of the next tick start at zero (every network, parity par ^ 1)
__global__ void k_serve_zero_counts(ServeDev d, uint32_t nnets, uint32_t ngrp) {
  const uint32_t q = d.par ^ 1u;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nnets * 2u * ngrp; i += gridDim.x * blockDim.x) {
    const uint32_t n = i / (2u * ngrp), j = i - n * 2u * ngrp;
    d.nets[n].ecnt[(size_t)q * 2 * ngrp + j] = 0u;
  }
}

cudaError_t launch_serve_batched(const ServeDev& d, const ServeCfg& c, int sms, cudaStream_t st);

cudaError_t launch_serve_drive(const ServeDev& d, const ServeCfg& c, int sms, bool gather, bool batched,
                               cudaStream_t st) {
  if (gather) {
    k_serve_drive<<<sms * 8, kServeThreads, 0, st>>>(d, c);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (batched) return launch_serve_batched(d, c, sms, st);
  return cudaSuccess;
}

cudaError_t launch_serve_emit(const ServeDev& d, const ServeCfg& c, int sms, size_t emitSmem, cudaStream_t st,
                              uint32_t nnets) {
  k_serve_zero_counts<<<16, 256, 0, st>>>(d, nnets, c.ncol / 8u);
  k_serve_emit<<<sms * 2, kEmitThreads, emitSmem, st>>>(d, c);
  return cudaGetLastError();
}

}  // namespace axon
