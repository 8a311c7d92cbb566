// Host/device interface of the multi-network kernel (multi.cu): many independent AXON
// networks, each with its own program of presentations, advanced by one persistent launch.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "plain.cuh"

namespace axon {

// One presentation of a network's program (the arguments of one present() call of
// src/axon.mm:815-888, with the outputs it should leave behind).
struct MultiPresent {
  const uint32_t* stim;     // [ncol] clamp pattern
  const uint32_t* refBall;  // [ncol] reference assembly for the drive log, or null (all zero)
  uint32_t* hist;           // [T][ncol] spikes of every step, or null
  uint32_t* finalOut;       // [ncol] spikes of the last step, or null
  uint32_t* stats;          // [1024] counters (accumulated; zeroed by the host), or null
  uint32_t* driveLog;       // [256] member-drive log (accumulated), or null
  uint32_t T, clampSteps, learn, useBias, k, facil;
  uint32_t pad[2];
};

// One network of the launch: its buffers and its program.
struct MultiNet {
  NetDev d;
  const MultiPresent* prog;
  uint32_t nprog, pad;
};

// CTAs [cta0, cta0 + ncta) form one slot: they run the networks queue[q0 .. q1) one after
// the other, with a grid barrier of their own.
struct MultiSlot {
  uint32_t cta0, ncta, q0, q1;
};

struct MultiDev {
  const MultiNet* nets;
  const MultiSlot* slots;   // sorted by cta0, covering the whole grid
  const uint32_t* queue;    // network indices, grouped by slot
  uint32_t* bars;           // [nslots * 32] barrier counters (one 128-byte line each), zeroed
  uint32_t* err;            // device error word
  unsigned long long* work; // [0] W3 tiles read by the drive, [1] learning tasks (branch read-modify-writes)
  uint32_t nslots, pad;
};

// Network parameters shared by every network of the launch (src/axon.mm:56-83).
struct MultiCfg {
  uint32_t ncol, incols, dthr, boost, mode, targetCols, biasUp, biasDown, biasShift, biasDownEvery, bandLo, bandHi,
      marginGate, hetero, ltdRep, contrast, ltdEvery, topkPar;
  uint32_t maxCpw;   // largest columns-per-warp of any slot (sizes the shared memory)
  uint32_t missing;  // CTAs every slot barrier waits for beyond the slot: 0, or more to test failure detection
  uint64_t waitNs;
};

// Launch shape: (threads, tiles) is (1024, 4), (896, 4) or (512, 8), one CTA per SM;
// grid = CTAs of all slots.
struct MultiShape {
  int threads, tiles, grid;
  size_t smem;
};

size_t multi_smem_bytes(uint32_t ncol, uint32_t incols, uint32_t maxCpw, int threads);
cudaError_t multi_max_blocks_per_sm(int threads, int tiles, size_t smem, int* out);
cudaError_t launch_multi(const MultiDev& m, const MultiCfg& c, const MultiShape& s, cudaStream_t st);

}  // namespace axon
