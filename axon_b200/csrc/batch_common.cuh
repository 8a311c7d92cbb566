// Device pieces shared by the batched readout kernels (batch.cu, serve_batched.cu): the W3
// tile layout they read, bounded TMA bulk copies into shared memory, the dendritic term
// and the packed per-(trajectory, neuron) drive counters.
#pragma once
#include <cstdint>

#include "axon_device.cuh"
#include "batch.cuh"

namespace axon {

// Tile layout for the batched kernel: word w of row r of a (column, branch) tile is stored
// at w*32 + (r XOR 4w). Rows r..r+3 (r a multiple of 4) of one word are then 16 contiguous
// bytes, lanes reading different words hit different groups of 4 banks, and the offset
// never wraps, so each read's address is one XOR and one add from the word's base.
__host__ __device__ __forceinline__ uint32_t w3r_pos(uint32_t r, uint32_t w) { return w * 32u + (r ^ (4u * w)); }

// ---------------------------------------------------------------- TMA bulk copy + mbarrier
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// bounded wait for one phase of an mbarrier
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
  if (mbar_test(bar, parity)) return true;
  const uint64_t t0 = globaltimer_ns();
  for (uint32_t it = 1;; ++it) {
    if (mbar_test(bar, parity)) return true;
    if ((it & 255u) == 0u && globaltimer_ns() - t0 > limit_ns) return false;
  }
}

// dendritic nonlinearity of k_drive, src/axon.mm:174-178, applied to a non-silent branch.
// LIN (modes 0, 1): count plus bst when the count reaches dthr; otherwise (mode 2) 0 or 1.
template <bool LIN>
__device__ __forceinline__ uint32_t branch_term(uint32_t cnt, uint32_t dthr, uint32_t bst) {
  if (LIN) return cnt + (cnt >= dthr ? bst : 0u);
  return cnt >= dthr ? 1u : 0u;
}

constexpr uint32_t kColWords = kNslot * 256;             // one column's 32 tiles
constexpr uint64_t kDrainNs = 1000000000ull;             // bound on waiting for own copies after a timeout
constexpr uint32_t kItemWords = kRecallCpi * kColWords;  // one work item

// The dendritic terms of four counts (rows r..r+3) added into the counters. Packed counters
// compute two terms at once in one word: with the counts c0, c1 (each below 2^15) in the
// low and high halves, adding 0x8000 - dthr to each half sets bit 15 of a half exactly when
// its count reaches dthr (no half carries into the next), so the terms are
// P + bst * N (modes 0, 1) or N (mode 2), N the two threshold bits moved to bit 0 of their
// halves. The host keeps packing for drives below 2^16, so no half overflows.
template <bool PACK, bool LIN>
__device__ __forceinline__ void acc_add4c(uint32_t* accb, uint32_t r, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                          uint32_t dthr, uint32_t bst) {
  if (PACK) {
    const uint32_t k = (0x8000u - min(dthr, 0x8000u)) * 0x00010001u;
    const uint32_t p0 = c0 + (c1 << 16), p1 = c2 + (c3 << 16);
    const uint32_t n0 = ((p0 + k) >> 15) & 0x00010001u, n1 = ((p1 + k) >> 15) & 0x00010001u;
    atomicAdd(accb + (r >> 1), LIN ? p0 + bst * n0 : n0);
    atomicAdd(accb + (r >> 1) + 1, LIN ? p1 + bst * n1 : n1);
  } else {
    atomicAdd(accb + r, branch_term<LIN>(c0, dthr, bst));
    atomicAdd(accb + r + 1, branch_term<LIN>(c1, dthr, bst));
    atomicAdd(accb + r + 2, branch_term<LIN>(c2, dthr, bst));
    atomicAdd(accb + r + 3, branch_term<LIN>(c3, dthr, bst));
  }
}

}  // namespace axon
