// Bit-serial learning rule shared by the plain and multi-network kernels.
#pragma once
#include <cstdint>

#include "axon_device.cuh"

namespace axon {

// One 32-synapse word of k_learn's update, src/axon.mm:466-488: co-active pairs are
// potentiated (phase 1), depressed ltdRep times (phase 2) or take the legacy rule
// (phase 0); optional heterosynaptic LTD; then the clip band on every lane. `C` is any
// configuration with the fields ltdRep, hetero, bandLo and bandHi.
template <class C>
__device__ __forceinline__ void learn_word(uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t& a3, uint32_t sp,
                                           bool want, uint32_t phase, uint32_t t, const C& c, uint32_t& nLTP,
                                           uint32_t& nLTD) {
  const uint32_t co = want ? sp : 0u;
  if (phase == 1u) {
    bs_inc(a0, a1, a2, a3, co);
    nLTP += __popc(co);
  } else if (phase == 2u) {
    for (uint32_t r = 0; r < c.ltdRep; ++r) bs_dec(a0, a1, a2, a3, co);
    nLTD += __popc(co) * c.ltdRep;
  } else {
    bs_inc(a0, a1, a2, a3, co);
    bs_dec(a0, a1, a2, a3, (want && (t % 2u == 1u)) ? ~sp : 0u);
  }
  if (c.hetero != 0u && phase == 1u) bs_dec(a0, a1, a2, a3, want ? ~sp : 0u);
  if (c.bandHi != 0u) bs_clip(a0, a1, a2, a3, c.bandLo, c.bandHi);
}

}  // namespace axon
