// Host/device interface of the recall-serving kernels (serve.cu).
//
// A server holds trajectory slots in device memory; every tick advances each admitted
// trajectory by one readout step (present() with learn = 0, src/axon.mm:815-888) with two
// launches: k_serve_drive (drive + ungated k-WTA, trajectories of one network sharing
// each W3 tile load) and k_serve_emit (threshold select + spike rebuild per trajectory).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace axon {

constexpr uint32_t kServeGroup = 8;  // trajectories of one network sharing a tile load

struct ServeNet {
  const uint4* W3;
  const uint32_t* conn;
};

// One admitted trajectory in the current tick.
struct ServeEntry {
  uint32_t slot;   // slot index (its buffers)
  uint32_t net;    // network index
  uint32_t tloc;   // local step this tick runs (0 = first)
  uint32_t clamp;  // clamped steps
  uint32_t ncue;   // cue columns (valid while tloc < clamp)
  uint32_t cueOff; // word offset of the cue columns in the tick's cue area
  uint32_t done;   // index in the done buffer when this is the last step, else 0xFFFFFFFF
  uint32_t pad;
};

// Up to kServeGroup entries of one network.
struct ServeGroup {
  uint32_t net, n;
  uint32_t e[kServeGroup];
};

struct ServeDev {
  const ServeNet* nets;
  uint32_t* slots;           // slot s at slots + s * slotWords: spk[2][ncol], act[2][nactw], xdrive[ncol], acc[ncol*32]
  const ServeEntry* ent;
  const ServeGroup* grp;
  const uint32_t* counts;    // [0] entries, [1] groups
  const uint32_t* cues;      // cue columns of the tick
  uint32_t* doneBuf;         // [done][ncol] final spikes of trajectories that end this tick
  uint32_t slotWords, nactw;
};

struct ServeCfg {
  uint32_t ncol, incols, dthr, boost, mode, targetCols, k, facil, topkPar;
  uint32_t acc32;  // per-neuron drive kept as u32 (u16 would overflow), else u16
};

__host__ __device__ inline uint32_t serve_nactw(uint32_t ncol) { return ((((ncol / 8u) + 31u) / 32u) + 3u) & ~3u; }
// offset (words) of the per-neuron drives in a slot, and the slot's size (256-byte multiple)
__host__ __device__ inline uint32_t serve_acc_off(uint32_t ncol) { return (3u * ncol + 2u * serve_nactw(ncol) + 63u) & ~63u; }
__host__ __device__ inline uint32_t serve_slot_words(uint32_t ncol, uint32_t acc32) {
  return (serve_acc_off(ncol) + (acc32 ? 32u : 16u) * ncol + 63u) & ~63u;
}

size_t serve_emit_smem_bytes(uint32_t ncol, uint32_t incols);
cudaError_t serve_prepare(size_t emitSmem);
// the two kernels of one tick; `between` (may be null) is recorded after the first
cudaError_t launch_serve_tick(const ServeDev& d, const ServeCfg& c, int sms, size_t emitSmem, cudaStream_t st,
                              cudaEvent_t between);

}  // namespace axon
