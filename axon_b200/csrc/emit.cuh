// Column gate and spike-vector rebuild shared by the plain and multi-network kernels.
#pragma once
#include <cstdint>

#include "axon_device.cuh"

namespace axon {

// k_emit's gate and clamp (src/axon.mm:211-212) for a whole network, run redundantly by
// every CTA of the network: column c spikes with its ungated ballot sB[c] when its drive
// sD[c] reaches the gate; input columns take the clamp pattern during clamped steps. One
// presynaptic group of 8 columns per lane; the group-activity bits (is any column of the
// group spiking) go to sActOut for the next step's drive. Every thread of the CTA calls it.
__device__ __forceinline__ void emit_groups(const uint32_t* sD, const uint32_t* sB, const uint32_t* sStim,
                                            uint32_t* sOut, uint32_t* sActOut, uint32_t gate, bool clamp,
                                            uint32_t incols, uint32_t ngrp) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, wpb = blockDim.x >> 5;
  for (uint32_t gb = warp * 32u; gb < ngrp; gb += wpb * 32u) {
    const uint32_t g = gb + lane;
    bool any = false;
    if (g < ngrp) {
      const uint4* d4 = reinterpret_cast<const uint4*>(sD) + 2 * g;
      const uint4* b4 = reinterpret_cast<const uint4*>(sB) + 2 * g;
      uint32_t w[8];
      const uint4 d0 = d4[0], d1 = d4[1], b0 = b4[0], b1 = b4[1];
      w[0] = d0.x < gate ? 0u : b0.x; w[1] = d0.y < gate ? 0u : b0.y;
      w[2] = d0.z < gate ? 0u : b0.z; w[3] = d0.w < gate ? 0u : b0.w;
      w[4] = d1.x < gate ? 0u : b1.x; w[5] = d1.y < gate ? 0u : b1.y;
      w[6] = d1.z < gate ? 0u : b1.z; w[7] = d1.w < gate ? 0u : b1.w;
      if (clamp && 8u * g < incols) {
#pragma unroll
        for (uint32_t k = 0; k < 8u; ++k)
          if (8u * g + k < incols) w[k] = sStim[8u * g + k];
      }
      reinterpret_cast<uint4*>(sOut)[2 * g] = make_uint4(w[0], w[1], w[2], w[3]);
      reinterpret_cast<uint4*>(sOut)[2 * g + 1] = make_uint4(w[4], w[5], w[6], w[7]);
      any = (w[0] | w[1] | w[2] | w[3] | w[4] | w[5] | w[6] | w[7]) != 0u;
    }
    const uint32_t wv = __ballot_sync(kFull, any);
    if (lane == 0) sActOut[gb >> 5] = wv;
  }
}

}  // namespace axon
