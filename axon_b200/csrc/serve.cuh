// Host/device interface of the recall-serving kernels (serve.cu, serve_batched.cu).
//
// A server holds trajectory slots in device memory; every tick advances each admitted
// trajectory by one readout step (present() with learn = 0, src/axon.mm:815-888):
//   drive     per network, either k_serve_batched (column tiles staged once in shared
//             memory for all of the network's trajectories, lanes over (branch,
//             trajectory) entries of nonzero spike words) or, for a network with few
//             trajectories this tick, k_serve_drive (warps over columns, tiles shared by
//             groups of kServeGroup trajectories); both leave per-neuron and column drives in the slot;
//   emit      k_serve_emit: threshold select, exact k-of-32 for the gated columns, the
//             spike vector, group-activity bits, and the entry lists of the next tick.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace axon {

constexpr uint32_t kServeGroup = 2;      // trajectories of one network sharing a tile load (gather kernel)
constexpr uint32_t kServeMaxB = 512;     // trajectories of one network per tick (list capacity)
constexpr uint32_t kServeMaxB32 = 300;   // the same when drives are kept as u32 (shared-memory bound)
constexpr uint32_t kServeBatchMin = 24;  // fewer trajectories of a network in a tick: gather kernel

struct ServeNet {
  const uint4* W3;
  const uint32_t* conn;
  const uint32_t* W3R;  // W3 in the batched tile layout
  uint2* ent1;          // [2 parity][ngrp][kServeMaxB] single-word entries: (index | word << 16, spikes)
  uint4* entM;          // [2 parity][ngrp][kServeMaxB] multi-word entries: (index | nz << 16, S0, S1, S2)
  uint32_t* ecnt;       // [2 parity][2 lists][ngrp] list lengths
};

// One admitted trajectory in the current tick.
struct ServeEntry {
  uint32_t slot;     // slot index (its buffers)
  uint32_t net;      // network index
  uint32_t tloc;     // local step this tick runs (0 = first)
  uint32_t clamp;    // clamped steps
  uint32_t ncue;     // cue columns (valid while tloc < clamp)
  uint32_t cueOff;   // word offset of the cue columns in the tick's cue area
  uint32_t done;     // index in the done buffer when this is the last step, else 0xFFFFFFFF
  uint32_t nextIdx;  // index in its network's next-tick batch (entry lists), 0xFFFFFFFF when done
};

// Up to kServeGroup entries of one network (gather kernel).
struct ServeGroup {
  uint32_t net, n;
  uint32_t e[kServeGroup];
};

// A network the batched kernel advances this tick: B trajectories whose (slot, tloc) are
// tab[tabOff .. tabOff + B) in batch-index order.
struct ServeBNet {
  uint32_t net, B, tabOff, pad;
};

struct ServeDev {
  const ServeNet* nets;
  uint32_t* slots;           // slot s at slots + s * slotWords: spk[2][ncol], act[2][nactw], xdrive[ncol], acc[ncol*32]
  const ServeEntry* ent;
  const ServeGroup* grp;
  const ServeBNet* bnets;
  const uint2* btab;         // (slot, tloc) per batch index of the batched networks
  const uint32_t* counts;    // [0] entries, [1] gather groups, [2] batched networks, [3] batched work items
  uint32_t* work;            // work-item counter of the batched kernel (zeroed by the tick's upload)
  const uint32_t* cues;      // cue columns of the tick
  uint32_t* doneBuf;         // [done][ncol] final spikes of trajectories that end this tick
  uint32_t slotWords, nactw;
  uint32_t par;              // tick parity: entry lists are read at par and written at par ^ 1
  uint32_t emitParts;        // CTAs sharing one trajectory's emit, each on its own column range
  uint32_t dacc;             // batched drive with two counter buffers: every batched network of the
                             // tick has at most serve_batched_dacc_maxb() trajectories
  uint64_t waitNs;           // bound on the batched kernel's copy waits
  uint32_t* err;             // device error word
};

struct ServeCfg {
  uint32_t ncol, incols, dthr, boost, mode, targetCols, k, facil, topkPar;
  uint32_t acc32;  // per-neuron drive kept as u32 (u16 would overflow), else u16
  uint32_t bst;    // dendritic bonus per branch reaching dthr: boost in mode 1, else 0
  uint32_t pad;
};

__host__ __device__ inline uint32_t serve_nactw(uint32_t ncol) { return ((((ncol / 8u) + 31u) / 32u) + 3u) & ~3u; }
// offset (words) of the per-neuron drives in a slot, and the slot's size (256-byte multiple)
__host__ __device__ inline uint32_t serve_acc_off(uint32_t ncol) { return (3u * ncol + 2u * serve_nactw(ncol) + 63u) & ~63u; }
__host__ __device__ inline uint32_t serve_slot_words(uint32_t ncol, uint32_t acc32) {
  return (serve_acc_off(ncol) + (acc32 ? 32u : 16u) * ncol + 63u) & ~63u;
}

size_t serve_emit_smem_bytes(uint32_t ncol, uint32_t incols);
size_t serve_batched_smem_bytes(uint32_t packed);
// most trajectories per network for which the batched drive keeps two counter buffers
uint32_t serve_batched_dacc_maxb(uint32_t packed);
cudaError_t serve_prepare(size_t emitSmem);
cudaError_t serve_batched_prepare(uint32_t packed);
// drive kernels of one tick (gather for the groups, batched for the batched networks)
cudaError_t launch_serve_drive(const ServeDev& d, const ServeCfg& c, int sms, bool gather, bool batched,
                               cudaStream_t st);
// clears the next tick's list lengths of nnets networks, then the emit kernel
cudaError_t launch_serve_emit(const ServeDev& d, const ServeCfg& c, int sms, size_t emitSmem, cudaStream_t st,
                              uint32_t nnets);

}  // namespace axon
