// Host/device interface of the batched recall kernel (batch.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace axon {

constexpr uint32_t kRecallMaxB = 512;   // trajectories per launch (the host splits larger batches)
constexpr uint32_t kRecallCpi = 2;      // columns per phase-1 work item
constexpr uint32_t kRecallMaxT = 1024;  // steps of a batched readout without per-step records
constexpr uint32_t kUnitTab = 128;      // phase-1 units per work item with a precomputed start branch

// Device buffers of one batched recall launch over B trajectories of one network.
struct RecallDev {
  const uint32_t* W3R;      // W3 re-laid out [col][branch][row][word] (read-only during recall)
  const uint32_t* conn;     // [ncol*32]
  const uint32_t* bias;     // [N]
  const uint32_t* mult;     // [N]
  const uint32_t* stims;    // [B][ncol] clamp patterns
  const uint32_t* refBall;  // [B][ncol] logged reference assemblies, or null
  uint32_t* spk;            // [2][B][ncol] spike vectors by step parity (slot 0 zeroed before launch)
  uint2* ent1;              // [2][ngrp][B] per-group lists of trajectories with ONE nonzero spike word
  uint4* entM;              // [2][ngrp][B] per-group lists of trajectories with several nonzero words
  uint32_t* ecnt;           // [2 parity][2 lists][ngrp] list lengths (parity 0 zeroed before launch)
  uint32_t* drv;            // [B][ncol] column drives of the current step
  void* acc;                // per-neuron drives (u16 or u32) of the current step, [B][ncol][32]; on the packed
                            // path without bias, facilitation or drive log laid out [ncol][4][B] x 8 u16, and
                            // only the entries whose column drive reaches the trajectory's histogram floor
                            // are written
  uint32_t* finalOut;       // [B][ncol] spikes of the last step, or null
  uint32_t* hist;           // [B][T][ncol] spikes of every step, or null
  uint32_t* stats;          // [B][1024] counters (zeroed before launch), or null
  uint32_t* driveLog;       // [B][256] member-drive log (accumulated), or null
  uint32_t* theta;          // [B] threshold of the last step, or null
  uint32_t* thHist;         // [3][B][3 x 640] drive histograms by step mod 3 (zeroed before launch)
  uint32_t* thPrev;         // [B] each trajectory's latest threshold (zeroed before launch)
  uint32_t* aff;            // [ncol][4][B] x 4 words: afferent counters of the clamped steps (packed fast path), or null
  uint32_t* work;           // [max(T, 64)] phase-1 work counters (zeroed before launch)
  uint32_t* bar;            // grid barrier counter (zeroed before launch)
  uint32_t* err;            // device error word
};

struct RecallCfg {
  uint32_t ncol, incols, B, T, clampSteps, useBias, k, dthr, boost, mode, targetCols, facil, biasShift, topkPar;
  uint32_t acc32;  // 1: per-neuron drive kept as u32 (packing two 16-bit sums would overflow)
  uint32_t bst;    // dendritic bonus per branch at or above dthr: boost (mode 1), 0 (mode 0)
  uint32_t dacc;   // 1: two counter buffers (alternating items), when they fit in shared memory
  uint32_t mma;    // 1: phase-1 AND-popcounts on the tensor cores (binary MMA), 0: __popc on the CUDA cores
  uint32_t slabFull;     // 1: the write-back stores every per-neuron drive (packed path)
  uint32_t slabAllStep;  // the step at which it stores every one anyway (0xFFFFFFFF: none)
  uint64_t waitNs;
};

struct RecallShape {
  int grid, threads;
  size_t smem;
};

size_t recall_smem_bytes(uint32_t ncol, uint32_t B, uint32_t acc32, uint32_t dacc);
cudaError_t recall_max_blocks_per_sm(int acc32, int threads, size_t smem, int* out);
cudaError_t launch_recall(const RecallDev& d, const RecallCfg& c, const RecallShape& s, cudaStream_t st);
// W3 [col][s][j][lane][comp] -> W3R [col][s][row = lane][word = 4j + comp]
cudaError_t launch_make_w3r(const uint4* W3, uint32_t* W3R, uint32_t ncol, cudaStream_t st);

}  // namespace axon
