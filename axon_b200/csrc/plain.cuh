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
  uint32_t *bar, *err;       // grid barrier counter, device error word
  uint32_t* finalOut;        // optional copy of the last step's spikes (recall), or null
  unsigned long long* prof;  // optional phase timestamps [T][grid][5] (device timer, ns), or null
};

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

}  // namespace axon
