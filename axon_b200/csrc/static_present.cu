// axon_present_static: one presentation on caller-owned device buffers, with no
// allocation of any kind during the call.
//
// Who needs it: hosts that own every byte of device memory themselves and are not allowed
// to call cudaMalloc - a framework whose caching allocator must see all device memory, a
// real-time service that forbids allocation after start-up, or a process where the
// allocator lock is held by someone else at call time. axon_present goes through an
// axon_net, whose creation allocates the network's buffers and the launch scratch; this
// entry point instead takes the caller's buffers directly and keeps the only scratch the
// persistent kernel needs (drive/ballot exchange slots, barrier counter, error word) in a
// fixed file-scope device array.
//
// The array is sized for networks of up to kStaticMaxNcol columns; every GPU that loads
// this library holds it until process exit. The first call on a device looks up the
// array's device address with cudaGetSymbolAddress (the host-side symbol is only a
// stand-in and must never be passed to a kernel) and keeps it for the life of the
// process: the library must not outlive a cudaDeviceReset of that device. Every call
// runs on the legacy default stream and synchronizes with it before returning, so it must
// not be made while any stream of the device is being captured. Every pointer must be
// 16-byte aligned (AXON_EINVAL otherwise).
//
// All calls on a device share the one array, and the kernel leaves the previous call's
// values in it: the barrier counter and error word are cleared at the start of every
// call, the exchange slots are fully rewritten before they are read. Calls that overlap
// on the GPU (other threads, other streams) race on the array and must not be issued.
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>

#include "engine.hpp"

using namespace axon;

namespace {

constexpr uint32_t kStaticMaxNcol = 4096;
// 2 x ncol drive slots + 2 x ncol ballot slots + the barrier region (barrier, error word at
// +16, drive histograms at +64)
constexpr uint32_t kStaticScratchWords = 4 * kStaticMaxNcol + kBarRegionWords;

static __device__ __align__(256) uint32_t g_present_scratch[kStaticScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
uint32_t* g_scratch_addr[kMaxDevices] = {nullptr};

axon_status scratch_address(int dev, uint32_t** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (dev < 0 || dev >= kMaxDevices) return set_error(AXON_EINVAL, "device index out of range");
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_present_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_present_scratch)");
    g_scratch_addr[dev] = (uint32_t*)p;
  }
  *out = g_scratch_addr[dev];
  return AXON_OK;
}

}  // namespace

#define CK(call)                                        \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

extern "C" axon_status axon_present_static(const axon_cfg* cfg, const axon_state_dev* s, uint32_t T,
                                           uint32_t clamp_steps, int learn, uint32_t use_bias) {
  if (!cfg || !s) return set_error(AXON_EINVAL, "null argument");
  std::string why = validate_cfg(*cfg);
  if (!why.empty()) return set_error(AXON_EINVAL, why);
  if (cfg->ncol > kStaticMaxNcol)
    return set_error(AXON_EINVAL, "axon_present_static supports ncol <= " + std::to_string(kStaticMaxNcol) +
                                      " (fixed device scratch); use axon_present for larger networks");
  if (T == 0 || T > 64) return set_error(AXON_EINVAL, "T must be in 1..64 (hist holds 64 steps)");
  if (use_bias > 2) return set_error(AXON_EINVAL, "use_bias must be 0, 1 or 2");
  const void* need[] = {s->w0, s->w1, s->w2, s->w3, s->conn, s->bias, s->mult, s->refball, s->stim, s->spk_a,
                        s->spk_b, s->drive, s->bbits, s->acc, s->marg, s->drive_log, s->stats, s->hist, s->theta};
  for (const void* p : need) {
    if (!p) return set_error(AXON_EINVAL, "every device pointer of axon_state_dev is required");
    // the kernel reads the planes and spike vectors as 16-byte vectors and copies W3 tiles
    // with cp.async.bulk, whose source must be 16-byte aligned
    if (((uintptr_t)p & 15u) != 0u)
      return set_error(AXON_EINVAL, "every device pointer of axon_state_dev must be 16-byte aligned");
  }

  int dev = 0;
  CK(cudaGetDevice(&dev));
  uint32_t* scratch = nullptr;
  axon_status st = scratch_address(dev, &scratch);
  if (st != AXON_OK) return st;

  const uint32_t ncol = cfg->ncol;
  NetDev d{};
  d.W0 = (uint4*)s->w0; d.W1 = (uint4*)s->w1; d.W2 = (uint4*)s->w2; d.W3 = (uint4*)s->w3;
  d.conn = s->conn; d.spkA = s->spk_a; d.spkB = s->spk_b; d.drive = s->drive; d.bbits = s->bbits;
  d.acc = s->acc; d.bias = s->bias; d.marg = s->marg; d.refBall = s->refball; d.driveLog = s->drive_log;
  d.mult = s->mult; d.stim = s->stim; d.stats = s->stats; d.hist = s->hist; d.theta = s->theta;
  d.xdrive = scratch;
  d.xball = scratch + 2 * ncol;
  d.bar = scratch + 4 * kStaticMaxNcol;
  d.err = d.bar + 16;
  d.finalOut = nullptr;

  // Params of present() and the co-resident launch shape: the same helpers axon_net uses
  const PresentCfg p = make_present_cfg(*cfg, T, clamp_steps, learn != 0, use_bias, 2000000000ull);
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  LaunchShape ls{};
  st = pick_present_shape(ncol, cfg->incols, sms, &ls);
  if (st != AXON_OK) return st;

  // clear what the kernel expects at zero: stats (launch_present clears the barrier
  // region, error word included)
  CK(cudaMemsetAsync(d.stats, 0, 1024 * 4, 0));
  CK(launch_present(d, p, ls, 0));
  CK(cudaStreamSynchronize(0));
  uint32_t errw = 0;
  CK(cudaMemcpy(&errw, d.err, 4, cudaMemcpyDeviceToHost));
  if (errw != 0u) return set_error(AXON_ETIMEOUT, "grid wait timed out in the persistent kernel");
  return AXON_OK;
}
