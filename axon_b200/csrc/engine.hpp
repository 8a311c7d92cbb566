// Host-side network object behind the C ABI: owns the device state of one AXON network
// and launches the plain kernels. The reference keeps the same state in MTLBuffers
// allocated at src/axon.mm:749-768.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/axon_capi.h"
#include "batch.cuh"
#include "plain.cuh"

namespace axon {

axon_status cuda_fail(cudaError_t e, const char* what);
axon_status set_error(axon_status s, const std::string& msg);
std::string validate_cfg(const axon_cfg& c);
// Params of one presentation, as present() resolves them (src/axon.mm:812, 818-845).
PresentCfg make_present_cfg(const axon_cfg& c, uint32_t T, uint32_t clampSteps, bool learn, uint32_t useBias,
                            uint64_t waitNs);
// Co-resident launch shape of k_present for a network of ncol columns on a GPU with `sms`
// SMs: one column per warp when the grid fits in one wave, else two.
axon_status pick_present_shape(uint32_t ncol, uint32_t incols, int sms, LaunchShape* out);

}  // namespace axon

// Grow-only device allocation reused across calls.
struct DevArena {
  void* p = nullptr;
  size_t cap = 0;
  axon_status ensure(size_t bytes);
  void release();
};

struct axon_net {
  axon_cfg cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t ncol = 0, n = 0;
  uint64_t plane_words = 0;
  axon::NetDev d{};
  void* base = nullptr;        // one device allocation for all buffers
  size_t base_bytes = 0;
  uint32_t* hstim = nullptr;   // pinned staging for the clamp pattern
  uint32_t* hscratch = nullptr;  // pinned staging for small reads (error word)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  axon::LaunchShape shape{};
  bool initialized = false;
  uint64_t wait_ns = 2000000000ull;
  uint32_t inject_missing = 0;  // one-shot: the next persistent launch waits for this many absent CTAs

  axon_status create(const axon_cfg& c, int dev);
  void release();
  axon_status init(uint32_t seed);
  axon_status present(const uint32_t* stim, uint32_t T, uint32_t clampSteps, bool learn, bool freeze,
                      uint32_t useBias, double* msPerStep);
  // one presentation with device-timer stamps at every phase boundary: out = us per step of
  // drive + k-of-32, grid barrier, threshold + emit, records + bias + learning, the whole
  // step, then the launch in ms
  axon_status profile_present(const uint32_t* stim, uint32_t T, uint32_t clampSteps, bool learn, uint32_t useBias,
                              double out[6]);
  axon_status clone_from(const axon_net& src);  // same configuration: copies every device buffer
  uint64_t buf_words(axon_buf which) const;
  uint32_t* buf_ptr(axon_buf which) const;
  axon_status read(axon_buf which, uint32_t* host, uint64_t words);
  axon_status write(axon_buf which, const uint32_t* host, uint64_t words);
  axon_status wstat(uint32_t* count);
  axon_status within(const uint32_t* ball, uint32_t useMask, const uint32_t* postMask, const uint32_t* mult,
                     uint32_t out[10]);
  axon_status indeg_untouched(uint32_t which, uint32_t* out);
  axon_status wdiag(const uint32_t* memb, const uint32_t* asmSpk, uint32_t nstim, uint32_t sel, uint32_t hist48[48]);
  axon::PresentCfg present_cfg(uint32_t T, uint32_t clampSteps, bool learn, uint32_t useBias) const;
  axon_status check_device_error();

  // batched readout
  uint32_t* w3b = nullptr;      // W3 as [col][branch][word][lane], rebuilt when weights change
  bool w3b_valid = false;
  DevArena scratch, io;
  int sm_count = 0;
  axon_status recall(const uint32_t* cues, uint32_t B, const axon_recall_args& a, const uint32_t* refBall,
                     uint32_t* finalOut, uint32_t* hist, uint32_t* stats, uint32_t* driveLog, bool dev, double* ms);
  axon_status ensure_w3b();
  // the batched readout as a captured CUDA graph, with the arguments it was captured for
  cudaGraphExec_t recallGraph = nullptr;
  std::vector<uint64_t> recallKey;
};
