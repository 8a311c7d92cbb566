// Host-side network object: allocation, init, present() and diagnostics.
#include <algorithm>
#include <cstring>
#include <vector>

#include "engine.hpp"

using namespace axon;

#define CK(call)                                        \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

namespace axon {

// Configurations the kernels are built for. The reference accepts some of these and then
// indexes past its fixed buffers or divides by zero; here they are refused.
std::string validate_cfg(const axon_cfg& c) {
  // the fused step keeps two spike vectors, the drives and the ballots of the whole
  // network in each CTA's shared memory: 8,192 columns is the widest that fits every kernel
  if (c.ncol == 0 || c.ncol % 32 != 0 || c.ncol > 8192) return "ncol must be a multiple of 32 in [32, 8192]";
  if (c.incols >= c.ncol) return "incols must be below ncol";
  if (c.inbr > 32) return "inbr must be <= 32";
  const uint32_t nInGrp = c.incols / 8, nGrp = c.ncol / 8;
  if (c.inbr > 0 && nInGrp == 0) return "incols must be >= 8 when inbr > 0";
  if (c.inbr < 32 && nGrp <= nInGrp) return "recurrent groups required when inbr < 32";
  if (c.contrast && c.ltdevery == 0) return "ltdevery must be >= 1 when contrast != 0";
  if (c.mode > 2) return "mode must be 0, 1 or 2";
  return "";
}

PresentCfg make_present_cfg(const axon_cfg& cfg, uint32_t T, uint32_t clampSteps, bool learn, uint32_t useBias,
                            uint64_t waitNs) {
  PresentCfg p{};
  p.ncol = cfg.ncol;
  p.incols = cfg.incols;
  p.T = T;
  p.clampSteps = clampSteps;
  p.learn = learn ? 1u : 0u;
  // src/axon.mm:818-822: readout-only k override and facilitation; bias auto = learning
  p.k = learn ? cfg.k : (cfg.ktest ? cfg.ktest : cfg.k);
  p.facil = learn ? 0u : cfg.facil;
  p.useBias = (useBias == 2u) ? (learn ? 1u : 0u) : (useBias ? 1u : 0u);
  p.dthr = cfg.dthr;
  p.boost = cfg.boost;
  p.mode = cfg.mode;
  p.targetCols = cfg.target;
  p.biasUp = cfg.biasup;
  p.biasDown = cfg.biasdown;
  p.biasShift = cfg.biasshift;
  p.biasDownEvery = cfg.biasdownevery;
  p.bandLo = cfg.bandlo;
  p.bandHi = cfg.contrast ? cfg.bandhi : 0u;  // src/axon.mm:812
  p.marginGate = cfg.margingate;
  p.hetero = cfg.hetero;
  p.ltdRep = cfg.ltdrep;
  p.contrast = cfg.contrast;
  p.ltdEvery = cfg.ltdevery ? cfg.ltdevery : 1u;
  p.topkPar = cfg.topkpar;
  p.waitNs = waitNs;
  return p;
}

axon_status pick_present_shape(uint32_t ncol, uint32_t incols, int sms, LaunchShape* out) {
  for (int cpw : {1, 2}) {
    const uint32_t warps = (ncol + cpw - 1) / cpw;
    int wpb = (int)std::min<uint32_t>(kPresentMaxWarps, (warps + sms - 1) / sms);
    wpb = std::max(wpb, 1);
    const int grid = (int)((warps + wpb - 1) / wpb);
    const size_t smem = present_smem_bytes(ncol, incols, cpw);
    int per_sm = 0;
    CK(present_max_blocks_per_sm(cpw, wpb * 32, smem, &per_sm));
    if (per_sm >= 1 && grid <= per_sm * sms) {
      out->cpw = cpw;
      out->wpb = wpb;
      out->grid = grid;
      out->smem = smem;
      return AXON_OK;
    }
  }
  return set_error(AXON_EINVAL, "no co-resident launch shape for this ncol");
}

}  // namespace axon

axon_status axon_net::create(const axon_cfg& c, int dev) {
  cfg = c;
  device = dev;
  ncol = c.ncol;
  n = c.ncol * 32u;
  plane_words = (uint64_t)ncol * 32 * 64 * 4;
  CK(cudaSetDevice(device));
  CK(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  CK(cudaEventCreate(&ev0));
  CK(cudaEventCreate(&ev1));
  // one allocation: 4 planes, then the small buffers, each 256-byte aligned
  const uint64_t small[] = {(uint64_t)ncol * 32, ncol, ncol, ncol, n, n, n, ncol, ncol, 256, n, ncol, 1024,
                            64ull * ncol, 16, 2ull * ncol, 2ull * ncol, kBarRegionWords, 64};
  uint64_t total = 4 * plane_words * 4;
  for (uint64_t w : small) total += (w * 4 + 255) & ~255ull;
  base_bytes = total;
  if (cudaMalloc(&base, total) != cudaSuccess) {
    cudaGetLastError();
    base = nullptr;
    return set_error(AXON_ENOMEM, "device allocation failed");
  }
  CK(cudaMemsetAsync(base, 0, total, stream));
  char* p = (char*)base;
  auto take = [&](uint64_t words) {
    uint32_t* r = (uint32_t*)p;
    p += (words * 4 + 255) & ~255ull;
    return r;
  };
  d.W0 = (uint4*)take(plane_words);
  d.W1 = (uint4*)take(plane_words);
  d.W2 = (uint4*)take(plane_words);
  d.W3 = (uint4*)take(plane_words);
  d.conn = take(small[0]);
  d.spkA = take(small[1]);
  d.spkB = take(small[2]);
  d.drive = take(small[3]);
  d.bbits = take(small[4]);
  d.acc = take(small[5]);
  d.bias = take(small[6]);
  d.marg = take(small[7]);
  d.refBall = take(small[8]);
  d.driveLog = take(small[9]);
  d.mult = take(small[10]);
  d.stim = take(small[11]);
  d.stats = take(small[12]);
  d.hist = take(small[13]);
  d.theta = take(small[14]);
  d.xdrive = take(small[15]);
  d.xball = take(small[16]);
  d.bar = take(small[17]);
  d.err = take(small[18]);
  CK(cudaMallocHost(&hstim, (size_t)ncol * 4));
  CK(cudaMallocHost(&hscratch, 64 * 4));

  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, device));
  sm_count = prop.multiProcessorCount;
  axon_status sst = pick_present_shape(ncol, c.incols, sm_count, &shape);
  if (sst != AXON_OK) return sst;
  CK(cudaStreamSynchronize(stream));
  return AXON_OK;
}

void axon_net::release() {
  if (recallGraph) cudaGraphExecDestroy(recallGraph);
  recallGraph = nullptr;
  scratch.release();
  io.release();
  if (w3b) cudaFree(w3b);
  w3b = nullptr;
  if (base) cudaFree(base);
  if (hstim) cudaFreeHost(hstim);
  if (hscratch) cudaFreeHost(hscratch);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (stream) cudaStreamDestroy(stream);
  base = nullptr;
  hstim = hscratch = nullptr;
}

axon_status axon_net::init(uint32_t seed) {
  CK(cudaSetDevice(device));
  CK(launch_init(d, ncol, cfg.incols, cfg.inbr, cfg.nand, seed, stream));
  CK(cudaMemsetAsync(d.bias, 0, (size_t)n * 4, stream));
  CK(cudaMemsetAsync(d.theta, 0, 16 * 4, stream));
  CK(cudaMemsetAsync(d.stats, 0, 1024 * 4, stream));
  CK(cudaStreamSynchronize(stream));
  initialized = true;
  w3b_valid = false;
  return AXON_OK;
}

PresentCfg axon_net::present_cfg(uint32_t T, uint32_t clampSteps, bool learn, uint32_t useBias) const {
  return make_present_cfg(cfg, T, clampSteps, learn, useBias, wait_ns);
}

axon_status axon_net::check_device_error() {
  CK(cudaMemcpyAsync(hscratch, d.err, 4, cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  if (hscratch[0] != 0u) {
    const uint32_t code = hscratch[0];
    CK(cudaMemsetAsync(d.err, 0, 4, stream));
    CK(cudaStreamSynchronize(stream));
    return set_error(AXON_ETIMEOUT, "grid wait timed out in the persistent kernel (code " + std::to_string(code) + ")");
  }
  return AXON_OK;
}

axon_status axon_net::present(const uint32_t* stim, uint32_t T, uint32_t clampSteps, bool learn, bool freeze,
                              uint32_t useBias, double* msPerStep) {
  (void)freeze;  // the reference sets P.freeze but no kernel reads it
  if (!initialized) return set_error(AXON_ESTATE, "present before init");
  if (T == 0 || T > 64) return set_error(AXON_EINVAL, "T must be in 1..64 (hist holds 64 steps)");
  if (useBias > 2) return set_error(AXON_EINVAL, "use_bias must be 0, 1 or 2");
  CK(cudaSetDevice(device));
  std::memcpy(hstim, stim, (size_t)ncol * 4);
  CK(cudaMemcpyAsync(d.stim, hstim, (size_t)ncol * 4, cudaMemcpyHostToDevice, stream));
  CK(cudaMemsetAsync(d.stats, 0, 1024 * 4, stream));
  PresentCfg pc = present_cfg(T, clampSteps, learn, useBias);
  pc.missing = inject_missing;
  inject_missing = 0;
  if (learn) w3b_valid = false;
  CK(cudaEventRecord(ev0, stream));
  CK(launch_present(d, pc, shape, stream));
  CK(cudaEventRecord(ev1, stream));
  axon_status st = check_device_error();
  if (st != AXON_OK) return st;
  if (msPerStep) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ev0, ev1));
    *msPerStep = (double)ms / T;
  }
  return AXON_OK;
}

uint64_t axon_net::buf_words(axon_buf which) const {
  switch (which) {
    case AXON_BUF_W0: case AXON_BUF_W1: case AXON_BUF_W2: case AXON_BUF_W3: return plane_words;
    case AXON_BUF_CONN: return (uint64_t)ncol * 32;
    case AXON_BUF_SPK_A: case AXON_BUF_SPK_B: case AXON_BUF_DRIVE: case AXON_BUF_MARG: case AXON_BUF_REFBALL:
    case AXON_BUF_STIM: return ncol;
    case AXON_BUF_BBITS: case AXON_BUF_ACC: case AXON_BUF_BIAS: case AXON_BUF_MULT: return n;
    case AXON_BUF_DRIVELOG: return 256;
    case AXON_BUF_STATS: return 1024;
    case AXON_BUF_HIST: return 64ull * ncol;
    case AXON_BUF_THETA: return 16;
  }
  return 0;
}

uint32_t* axon_net::buf_ptr(axon_buf which) const {
  switch (which) {
    case AXON_BUF_W0: return (uint32_t*)d.W0;
    case AXON_BUF_W1: return (uint32_t*)d.W1;
    case AXON_BUF_W2: return (uint32_t*)d.W2;
    case AXON_BUF_W3: return (uint32_t*)d.W3;
    case AXON_BUF_CONN: return d.conn;
    case AXON_BUF_SPK_A: return d.spkA;
    case AXON_BUF_SPK_B: return d.spkB;
    case AXON_BUF_DRIVE: return d.drive;
    case AXON_BUF_BBITS: return d.bbits;
    case AXON_BUF_ACC: return d.acc;
    case AXON_BUF_BIAS: return d.bias;
    case AXON_BUF_MARG: return d.marg;
    case AXON_BUF_REFBALL: return d.refBall;
    case AXON_BUF_DRIVELOG: return d.driveLog;
    case AXON_BUF_MULT: return d.mult;
    case AXON_BUF_STIM: return d.stim;
    case AXON_BUF_STATS: return d.stats;
    case AXON_BUF_HIST: return d.hist;
    case AXON_BUF_THETA: return d.theta;
  }
  return nullptr;
}

axon_status axon_net::read(axon_buf which, uint32_t* host, uint64_t words) {
  uint32_t* p = buf_ptr(which);
  if (!p || words != buf_words(which)) return set_error(AXON_EINVAL, "buffer id or size mismatch");
  CK(cudaSetDevice(device));
  CK(cudaMemcpyAsync(host, p, words * 4, cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  return AXON_OK;
}

axon_status axon_net::write(axon_buf which, const uint32_t* host, uint64_t words) {
  uint32_t* p = buf_ptr(which);
  if (!p || words != buf_words(which)) return set_error(AXON_EINVAL, "buffer id or size mismatch");
  CK(cudaSetDevice(device));
  CK(cudaMemcpyAsync(p, host, words * 4, cudaMemcpyHostToDevice, stream));
  CK(cudaStreamSynchronize(stream));
  if (which == AXON_BUF_W0 || which == AXON_BUF_CONN) initialized = true;
  if (which == AXON_BUF_W3) w3b_valid = false;
  return AXON_OK;
}

axon_status axon_net::wstat(uint32_t* count) {
  CK(cudaSetDevice(device));
  uint32_t* tmp = d.err + 16;  // scratch words after the error word
  CK(cudaMemsetAsync(tmp, 0, 4, stream));
  CK(launch_wstat(d, ncol, tmp, stream));
  CK(cudaMemcpyAsync(hscratch, tmp, 4, cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  *count = hscratch[0];
  return AXON_OK;
}

namespace {
// temporary device buffers for diagnostic calls
struct DevTmp {
  void* p = nullptr;
  ~DevTmp() { if (p) cudaFree(p); }
};
}  // namespace

axon_status axon_net::within(const uint32_t* ball, uint32_t useMask, const uint32_t* postMask, const uint32_t* mult,
                             uint32_t out[10]) {
  CK(cudaSetDevice(device));
  DevTmp t;
  const size_t words = ncol + 2ull * n + 16;
  CK(cudaMalloc(&t.p, words * 4));
  uint32_t* dball = (uint32_t*)t.p;
  uint32_t* dpost = dball + ncol;
  uint32_t* dmult = dpost + n;
  uint32_t* dout = dmult + n;
  CK(cudaMemcpyAsync(dball, ball, (size_t)ncol * 4, cudaMemcpyHostToDevice, stream));
  if (useMask) CK(cudaMemcpyAsync(dpost, postMask, (size_t)n * 4, cudaMemcpyHostToDevice, stream));
  if (mult) CK(cudaMemcpyAsync(dmult, mult, (size_t)n * 4, cudaMemcpyHostToDevice, stream));
  else CK(cudaMemsetAsync(dmult, 0, (size_t)n * 4, stream));
  CK(cudaMemcpyAsync(dout, out, 10 * 4, cudaMemcpyHostToDevice, stream));
  CK(launch_within(d, ncol, cfg.inbr, cfg.incols, dball, useMask, dpost, dmult, dout, stream));
  CK(cudaMemcpyAsync(out, dout, 10 * 4, cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  return AXON_OK;
}

axon_status axon_net::indeg_untouched(uint32_t which, uint32_t* out) {
  CK(cudaSetDevice(device));
  DevTmp t;
  CK(cudaMalloc(&t.p, (size_t)n * 4));
  CK(launch_indeg_untouched(d, ncol, cfg.inbr, which, (uint32_t*)t.p, stream));
  CK(cudaMemcpyAsync(out, t.p, (size_t)n * 4, cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  return AXON_OK;
}

axon_status axon_net::wdiag(const uint32_t* memb, const uint32_t* asmSpk, uint32_t nstim, uint32_t sel,
                            uint32_t hist48[48]) {
  CK(cudaSetDevice(device));
  DevTmp t;
  const size_t words = (size_t)n + (size_t)nstim * ncol + 48;
  CK(cudaMalloc(&t.p, words * 4));
  uint32_t* dm = (uint32_t*)t.p;
  uint32_t* da = dm + n;
  uint32_t* dh = da + (size_t)nstim * ncol;
  CK(cudaMemcpyAsync(dm, memb, (size_t)n * 4, cudaMemcpyHostToDevice, stream));
  if (nstim) CK(cudaMemcpyAsync(da, asmSpk, (size_t)nstim * ncol * 4, cudaMemcpyHostToDevice, stream));
  CK(cudaMemcpyAsync(dh, hist48, 48 * 4, cudaMemcpyHostToDevice, stream));
  CK(launch_wdiag(d, ncol, dm, da, nstim, cfg.inbr, sel, dh, stream));
  CK(cudaMemcpyAsync(hist48, dh, 48 * 4, cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  return AXON_OK;
}

axon_status axon_net::profile_present(const uint32_t* stim, uint32_t T, uint32_t clampSteps, bool learn,
                                      uint32_t useBias, double out[6]) {
  if (!initialized) return set_error(AXON_ESTATE, "present before init");
  if (T == 0 || T > 64) return set_error(AXON_EINVAL, "T must be in 1..64 (hist holds 64 steps)");
  CK(cudaSetDevice(device));
  DevTmp tmp;
  const size_t nst = (size_t)T * shape.grid * 5;
  CK(cudaMalloc(&tmp.p, nst * 8));
  std::memcpy(hstim, stim, (size_t)ncol * 4);
  CK(cudaMemcpyAsync(d.stim, hstim, (size_t)ncol * 4, cudaMemcpyHostToDevice, stream));
  CK(cudaMemsetAsync(d.stats, 0, 1024 * 4, stream));
  CK(cudaMemsetAsync(tmp.p, 0, nst * 8, stream));
  NetDev dd = d;
  dd.prof = (unsigned long long*)tmp.p;
  const PresentCfg pc = present_cfg(T, clampSteps, learn, useBias);
  if (learn) w3b_valid = false;
  CK(cudaEventRecord(ev0, stream));
  CK(launch_present(dd, pc, shape, stream));
  CK(cudaEventRecord(ev1, stream));
  axon_status st = check_device_error();
  if (st != AXON_OK) return st;
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ev0, ev1));
  std::vector<unsigned long long> h(nst);
  CK(cudaMemcpy(h.data(), tmp.p, nst * 8, cudaMemcpyDeviceToHost));
  // per phase: mean over CTAs of each CTA's time in it, summed over the steps
  double ph[4] = {0, 0, 0, 0}, stepT = 0;
  for (uint32_t t = 0; t < T; ++t) {
    for (int b = 0; b < shape.grid; ++b) {
      const unsigned long long* s = h.data() + ((size_t)t * shape.grid + b) * 5;
      for (int k = 0; k < 4; ++k) ph[k] += (double)(s[k + 1] - s[k]);
      stepT += (double)(s[4] - s[0]);
    }
  }
  for (int k = 0; k < 4; ++k) out[k] = ph[k] / shape.grid / T / 1e3;  // us per step
  out[4] = stepT / shape.grid / T / 1e3;
  out[5] = ms;
  return AXON_OK;
}

axon_status axon_net::clone_from(const axon_net& src) {
  if (!src.initialized) return set_error(AXON_ESTATE, "clone before init");
  CK(cudaSetDevice(device));
  CK(cudaMemcpyAsync(base, src.base, base_bytes, cudaMemcpyDeviceToDevice, stream));
  CK(cudaStreamSynchronize(stream));
  initialized = true;
  w3b_valid = false;
  return AXON_OK;
}
