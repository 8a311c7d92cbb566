// Device-side building blocks shared by the AXON kernels (sm_100a).
//
// The integer rules follow rakib-nyc/axon src/axon.mm (cited per function); the code is
// organised for CUDA: one warp per column, lane = neuron, warp reductions in place of
// simd_* collectives, and a bounded grid barrier for the persistent step loop.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace axon {

constexpr uint32_t kFull = 0xFFFFFFFFu;
constexpr uint32_t kNslot = 32;   // branches per neuron
constexpr uint32_t kTileU4 = 64;  // uint4 per (column, branch) tile: 2 halves x 32 lanes

// error codes written to the device error word
constexpr uint32_t kErrTimeout = 1;

// hash32, src/axon.mm:54
__host__ __device__ __forceinline__ uint32_t hash32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}

__device__ __forceinline__ uint32_t popc4(uint4 a, uint4 b) {
  return __popc(a.x & b.x) + __popc(a.y & b.y) + __popc(a.z & b.z) + __popc(a.w & b.w);
}

// ---------------------------------------------------------------- bit-serial counters
// 4-bit counters held as 4 bitplanes; one 32-bit word per plane = 32 synapses.
// Saturating +1 / -1 and the symmetric clip of src/axon.mm:371-420.
__device__ __forceinline__ void bs_inc(uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t& a3, uint32_t m) {
  uint32_t c = m, t;
  t = a0 ^ c; c &= a0; a0 = t;
  t = a1 ^ c; c &= a1; a1 = t;
  t = a2 ^ c; c &= a2; a2 = t;
  t = a3 ^ c; c &= a3; a3 = t;
  a0 |= c; a1 |= c; a2 |= c; a3 |= c;
}
__device__ __forceinline__ void bs_dec(uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t& a3, uint32_t m) {
  uint32_t b = m, t;
  t = a0 ^ b; b &= ~a0; a0 = t;
  t = a1 ^ b; b &= ~a1; a1 = t;
  t = a2 ^ b; b &= ~a2; a2 = t;
  t = a3 ^ b; b &= ~a3; a3 = t;
  a0 &= ~b; a1 &= ~b; a2 &= ~b; a3 &= ~b;
}
// synapses whose value is < K (lt) and > K (gt); K in 0..15
__device__ __forceinline__ uint32_t bs_lt(uint32_t a3, uint32_t a2, uint32_t a1, uint32_t a0, uint32_t K) {
  uint32_t lt = 0, eq = kFull;
  if ((K >> 3) & 1u) lt |= eq & ~a3;
  eq &= ((K >> 3) & 1u) ? a3 : ~a3;
  if ((K >> 2) & 1u) lt |= eq & ~a2;
  eq &= ((K >> 2) & 1u) ? a2 : ~a2;
  if ((K >> 1) & 1u) lt |= eq & ~a1;
  eq &= ((K >> 1) & 1u) ? a1 : ~a1;
  if (K & 1u) lt |= eq & ~a0;
  return lt;
}
__device__ __forceinline__ uint32_t bs_gt(uint32_t a3, uint32_t a2, uint32_t a1, uint32_t a0, uint32_t K) {
  uint32_t gt = 0, eq = kFull;
  if (!((K >> 3) & 1u)) gt |= eq & a3;
  eq &= ((K >> 3) & 1u) ? a3 : ~a3;
  if (!((K >> 2) & 1u)) gt |= eq & a2;
  eq &= ((K >> 2) & 1u) ? a2 : ~a2;
  if (!((K >> 1) & 1u)) gt |= eq & a1;
  eq &= ((K >> 1) & 1u) ? a1 : ~a1;
  if (!(K & 1u)) gt |= eq & a0;
  return gt;
}
__device__ __forceinline__ void bs_set(uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t& a3, uint32_t m, uint32_t C) {
  const uint32_t keep = ~m;
  a0 = (a0 & keep) | ((C & 1u) ? m : 0u);
  a1 = (a1 & keep) | ((C & 2u) ? m : 0u);
  a2 = (a2 & keep) | ((C & 4u) ? m : 0u);
  a3 = (a3 & keep) | ((C & 8u) ? m : 0u);
}
__device__ __forceinline__ void bs_clip(uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t& a3, uint32_t lo, uint32_t hi) {
  const uint32_t l = bs_lt(a3, a2, a1, a0, lo);
  const uint32_t g = bs_gt(a3, a2, a1, a0, hi);
  bs_set(a0, a1, a2, a3, l, lo);
  bs_set(a0, a1, a2, a3, g, hi);
}

// ---------------------------------------------------------------- exact k-of-32
// rank = #{j : v_j > v_i or (v_j == v_i and j < i)}; winners rank < k; vk / vk1 are the
// values ranked k-1 and k (0 if no lane has that rank). src/axon.mm:134-144.
// Method: a bit-sliced comparison. Over the significant bits of the largest value, most
// significant first, one ballot per bit; each lane keeps the lanes whose values are larger
// than its own (gt) and those equal so far (eq): a lane holding 0 at a bit moves the equal
// lanes holding 1 there into gt and drops them from eq, a lane holding 1 drops the equal
// lanes holding 0. Then rank = popc(gt) + the equal lanes below it. The ballots do not
// depend on one another; each lane's update chain is a few integer operations per bit.
__device__ __forceinline__ uint32_t warp_kwta(uint32_t v, uint32_t lane, uint32_t k, uint32_t& vk, uint32_t& vk1) {
  if (k == 0u) { vk = 0u; vk1 = __reduce_max_sync(kFull, v); return 0u; }
  if (k > 32u) { vk = 0u; vk1 = 0u; return kFull; }
  const uint32_t M = __reduce_max_sync(kFull, v);
  uint32_t gt = 0u, eq = kFull;
  for (int bit = (int)(32u - __clz(M)) - 1; bit >= 0; --bit) {
    const uint32_t ones = __ballot_sync(kFull, (v >> bit) & 1u);
    if ((v >> bit) & 1u) {
      eq &= ones;
    } else {
      gt |= eq & ones;
      eq &= ~ones;
    }
  }
  const uint32_t rank = (uint32_t)__popc(gt) + (uint32_t)__popc(eq & ((1u << lane) - 1u));
  vk = __shfl_sync(kFull, v, __ffs(__ballot_sync(kFull, rank == k - 1u)) - 1);
  vk1 = k == 32u ? 0u : __shfl_sync(kFull, v, __ffs(__ballot_sync(kFull, rank == k)) - 1);
  return __ballot_sync(kFull, rank < k);
}

// ---------------------------------------------------------------- asynchronous copies
// 16-byte global->shared copies that bypass L1 (the source was written by other SMs)
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// ---------------------------------------------------------------- bounded grid barrier
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
  return *reinterpret_cast<const volatile uint32_t*>(p);
}
// arrival at a grid barrier: a release at GPU scope (cumulative over the writes the CTA's
// threads made before the preceding __syncthreads) that does not wait for a reply
__device__ __forceinline__ void red_release_add_gpu(uint32_t* p, uint32_t v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier over `nblocks` co-resident CTAs. `bar` is zeroed before the launch;
// barrier number `epoch` (0, 1, 2, ...) waits until all CTAs have arrived `epoch+1`
// times. The wait gives up after `limit_ns` nanoseconds, or as soon as another CTA has
// given up, and then records kErrTimeout in `err`. Returns false if the CTA must exit.
// Every thread of the CTA must call it.
__device__ __forceinline__ bool grid_barrier(uint32_t* bar, uint32_t* err, uint32_t nblocks, uint32_t epoch,
                                             uint64_t limit_ns, uint32_t* s_flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t ok = 1;
    red_release_add_gpu(bar, 1u);
    const uint32_t target = (epoch + 1u) * nblocks;
    const uint64_t t0 = globaltimer_ns();
    uint32_t it = 0;
    while (ld_acquire_gpu(bar) < target) {
      if ((++it & 63u) == 0u) {
        if (ld_volatile(err) != 0u || globaltimer_ns() - t0 > limit_ns) {
          atomicCAS(err, 0u, kErrTimeout);
          ok = 0;
          break;
        }
      }
    }
    *s_flag = ok;  // the acquire load that saw the count orders the CTA's later reads
  }
  __syncthreads();
  return *s_flag != 0u;
}

}  // namespace axon
