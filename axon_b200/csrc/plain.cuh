// Host/device interface of the plain AXON kernels (plain.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace axon {

// Device pointers of one network (all owned by the host-side axon_net).
struct NetDev {
  uint4 *W0, *W1, *W2, *W3;  // bitplanes, tile-major: ((col*32 + s)*2 + j)*32 + lane
  uint32_t *conn, *spkA, *spkB, *drive, *bbits, *acc, *bias, *marg, *refBall, *driveLog, *mult, *stim, *stats,
      *hist, *theta;
  uint32_t *xdrive, *xball;  // 2 x ncol exchange slots (step parity) for drives / ungated ballots
  uint32_t *bar, *err;       // grid barrier counter (a kBarRegionWords region, below), device error word
  uint32_t* finalOut;        // optional copy of the last step's spikes (recall), or null
  unsigned long long* prof;  // optional phase timestamps [T][grid][5] (device timer, ns), or null
};

// The barrier word heads a region of kBarRegionWords words that launch_present clears
// before every launch: words [0, 64) for the barrier (and the caller's own flags), then
// three histograms of the recurrent column drives, one per step mod 3. A histogram holds
// per theta_key bin the count, the largest drive and the complement of the smallest.
constexpr uint32_t kThetaBins = 640;
constexpr uint32_t kHistWords = 3u * kThetaBins;
constexpr uint32_t kBarRegionWords = 64u + 3u * kHistWords;

// Dynamic shared memory of k_present: the fixed part (spike vectors, activity bits, clamp
// pattern, histogram, flags, mbarriers, learning lists), then on a 1 KiB boundary the tile
// pool of phase A, as large as the 227 KiB limit allows (at least the 3 x ncol words that
// phase B stages into the same space).
constexpr uint32_t kMaxColSlots = 64;      // column slots per CTA (32 warps x 2 columns)
constexpr uint32_t kPresentMaxWarps = 28;  // k_present is compiled for 896 threads (72 registers)
constexpr uint32_t kSmemLimitBytes = 227u * 1024u;
struct PresentSmem {
  uint32_t poolWord;   // first word of the pool
  uint32_t poolTiles;  // 1 KiB W3 tiles the pool holds
  uint32_t bytes;      // dynamic shared memory of the launch
};
__host__ __device__ inline PresentSmem present_smem_layout(uint32_t ncol, uint32_t incols, int cpw) {
  const uint32_t ngrp = ncol / 8u, nactw = (((ngrp + 31u) / 32u) + 3u) & ~3u;
  const uint32_t maxCols = 32u * (uint32_t)cpw;
  uint32_t w = 2u * ncol + 2u * nactw + ((incols + 3u) & ~3u) + kHistWords + 16u + 2u * kMaxColSlots +
               maxCols * (6u * 32u + 4u);
  w = (w + 255u) & ~255u;
  const uint32_t limitW = kSmemLimitBytes / 4u;
  uint32_t poolW = limitW > w ? (limitW - w) & ~255u : 0u;
  const uint32_t minW = (3u * ncol + 255u) & ~255u;
  if (poolW < minW) poolW = minW;  // beyond the limit: the occupancy check rejects the shape
  return {w, poolW / 256u, (w + poolW) * 4u};
}

// Everything one presentation needs (the reference's Params block, resolved for a
// present() call: src/axon.mm:810-845).
struct PresentCfg {
  uint32_t ncol, incols, T, clampSteps, learn, k, dthr, boost, mode, targetCols, useBias, facil, biasUp, biasDown,
      biasShift, biasDownEvery, bandLo, bandHi, marginGate, hetero, ltdRep, contrast, ltdEvery, topkPar;
  uint32_t missing;  // CTAs every grid barrier waits for beyond the launch: 0, or more to test failure detection
  uint64_t waitNs;
};

struct LaunchShape {
  int cpw;       // columns per warp (1, 2)
  int wpb;       // warps per block
  int grid;      // blocks (all co-resident)
  size_t smem;   // dynamic shared memory bytes
};

size_t present_smem_bytes(uint32_t ncol, uint32_t incols, int cpw);
cudaError_t present_max_blocks_per_sm(int cpw, int threads, size_t smem, int* out);
cudaError_t launch_present(const NetDev& d, const PresentCfg& c, const LaunchShape& ls, cudaStream_t st);
cudaError_t launch_init(const NetDev& d, uint32_t ncol, uint32_t incols, uint32_t inbr, uint32_t nand, uint32_t seed,
                        cudaStream_t st);
cudaError_t launch_wstat(const NetDev& d, uint32_t ncol, uint32_t* out, cudaStream_t st);
cudaError_t launch_within(const NetDev& d, uint32_t ncol, uint32_t inBr, uint32_t inCols, const uint32_t* ball,
                          uint32_t useMask, const uint32_t* postMask, const uint32_t* mult, uint32_t* out,
                          cudaStream_t st);
cudaError_t launch_indeg_untouched(const NetDev& d, uint32_t ncol, uint32_t inBr, uint32_t which, uint32_t* out,
                                   cudaStream_t st);
cudaError_t launch_wdiag(const NetDev& d, uint32_t ncol, const uint32_t* memb, const uint32_t* asmSpk, uint32_t nstim,
                         uint32_t inBr, uint32_t sel, uint32_t* hist, cudaStream_t st);
cudaError_t launch_bstest(uint32_t* a0, uint32_t* a1, uint32_t* a2, uint32_t* a3, const uint32_t* m, uint32_t op,
                          uint32_t lo, uint32_t hi, uint64_t n, cudaStream_t st);
cudaError_t launch_kwtatest(const uint32_t* v, const uint32_t* k, uint32_t* out, uint32_t n, cudaStream_t st);

}  // namespace axon
