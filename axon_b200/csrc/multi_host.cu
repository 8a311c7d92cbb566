// Host side of axon_multi_train: many networks trained and read out by one persistent
// launch (multi.cu), with the launch shape picked by timing candidates.
//
// Each network runs the reference's experiment from its seed (src/axon.mm:669-1909,
// restricted to what the five published measurements need): patterns from the seed
// (src/axon.mm:793-799), epochs x nstim learning presentations plus the extra one of
// pattern 0 (src/axon.mm:1008-1033), the clamped references (src/axon.mm:1080-1105), the
// 75% cue completion row (src/axon.mm:1495-1508), the drive trace (src/axon.mm:1712-1728)
// and the wave (src/axon.mm:1804-1858). The ten settle presentations of src/axon.mm:1001
// are left out: they change no weight and no bias, so no measurement depends on them.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "engine.hpp"
#include "multi.cuh"
#include "setops.hpp"
#include "stimulus.hpp"

using namespace axon;

#define CK(call)                                        \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

namespace {

size_t al(size_t bytes) { return (bytes + 255) & ~(size_t)255; }
constexpr uint32_t kCalPresents = 3;  // learning presentations per slot when timing a shape
constexpr uint32_t kMaxSlots = 1024;

// Device arena of one call, released on every exit path.
struct Arena {
  void* p = nullptr;
  ~Arena() {
    if (p) cudaFree(p);
  }
};

// Plan of one network: its cues, its program and where its outputs go.
struct NetPlan {
  uint32_t seed = 0, nstim = 0, nq = 0, TT = 0, TW = 0;
  std::vector<std::vector<uint32_t>> pats;
  std::vector<uint32_t> cues;  // [ncue][ncol] host copy
  size_t cuesOff = 0, refsOff = 0, recOff = 0, dlogOff = 0, waveOff = 0, progOff = 0;
  std::vector<MultiPresent> prog;
  uint32_t nTrain = 0;  // learning presentations at the head of prog
  uint64_t steps = 0, trainSteps = 0;
};

// cue indices within NetPlan::cues
struct CueIx {
  uint32_t nstim, nq;
  uint32_t train(uint32_t p) const { return p; }
  uint32_t extra() const { return nstim; }
  uint32_t ref(uint32_t p) const { return nstim + 1 + p; }
  uint32_t rec(uint32_t q) const { return 2 * nstim + 1 + q; }
  uint32_t drv(uint32_t q) const { return 3 * nstim + 1 + q; }
  uint32_t wave(uint32_t q) const { return 3 * nstim + 1 + nq + q; }
  uint32_t count() const { return 3 * nstim + 1 + 2 * nq; }
};

struct Shape {
  uint32_t slots = 1;
  int threads = 1024, tiles = 4;
};

// LPT assignment of networks (cost = steps) to slots whose speed is proportional to their
// CTA count; returns the predicted makespan in steps of one average slot.
double assign(const std::vector<uint64_t>& cost, const std::vector<uint32_t>& ncta,
              std::vector<std::vector<uint32_t>>& queues) {
  const uint32_t S = (uint32_t)ncta.size();
  queues.assign(S, {});
  std::vector<uint32_t> order(cost.size());
  std::iota(order.begin(), order.end(), 0u);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
  const double avg = std::accumulate(ncta.begin(), ncta.end(), 0.0) / S;
  std::vector<double> fin(S, 0.0);
  for (uint32_t i : order) {
    uint32_t best = 0;
    double bestT = 1e300;
    for (uint32_t s = 0; s < S; ++s) {
      const double t = fin[s] + (double)cost[i] * avg / ncta[s];
      if (t < bestT) { bestT = t; best = s; }
    }
    fin[best] = bestT;
    queues[best].push_back(i);
  }
  return *std::max_element(fin.begin(), fin.end());
}

std::vector<uint32_t> split_ctas(uint32_t grid, uint32_t S) {
  std::vector<uint32_t> v(S, grid / S);
  for (uint32_t s = 0; s < grid % S; ++s) ++v[s];
  return v;
}

// The call itself: the device arena and the per-network plans share one scope.
class MultiRun {
 public:
  MultiRun(axon_net* const* nets, uint32_t n, const axon_multi_args& a) : nets_(nets), n_(n), a_(a) {}
  axon_status run(const uint32_t* seeds, const uint32_t* nstim, axon_multi_result* res, axon_multi_report* rep);

 private:
  axon_net* const* nets_;
  uint32_t n_;
  axon_multi_args a_;
  axon_net* net0_ = nullptr;
  uint32_t ncol_ = 0, incols_ = 0;
  std::vector<NetPlan> plans_;
  Arena arena_;
  char* base_ = nullptr;
  size_t ctlOff_ = 0;  // MultiNet / slots / queue / bars / err / plain-path scratch region
  MultiCfg cfg_{};
  unsigned long long lastWork_[2] = {0, 0};  // tiles read, learning tasks of the last launch

  uint32_t* dev(size_t off) const { return (uint32_t*)(base_ + off); }
  axon_status plan(const uint32_t* seeds, const uint32_t* nstim);
  axon_status init_all();
  axon_status launch(const Shape& sh, const std::vector<std::vector<uint32_t>>& queues,
                     const std::vector<uint32_t>& ncta, const std::vector<uint32_t>* nprogOverride, bool graph,
                     float* ms, bool* usedGraph);
  axon_status run_plain(float* ms);
  axon_status tune(Shape* best, std::vector<std::vector<uint32_t>>* bestQ, std::vector<uint32_t>* bestCta,
                   float* tuneMs, uint32_t* tried);
  axon_status measure(uint32_t i, axon_multi_result* r);
  uint32_t max_cpw(const std::vector<uint32_t>& ncta, int threads) const {
    uint32_t m = 1;
    for (uint32_t c : ncta) m = std::max(m, (ncol_ + c * (threads / 32) - 1) / (c * (threads / 32)));
    return m;
  }
  // control region layout (byte offsets from ctlOff_)
  size_t offSlots() const { return al(n_ * sizeof(MultiNet)); }
  size_t offQueue() const { return offSlots() + al(kMaxSlots * sizeof(MultiSlot)); }
  size_t offBars() const { return offQueue() + al(n_ * 4); }
  size_t offErr() const { return offBars() + al(kMaxSlots * 32 * 4); }
  size_t offHist() const { return offErr() + al(64); }
  size_t offStats() const { return offHist() + al((size_t)64 * ncol_ * 4); }
  size_t offDlog() const { return offStats() + al(1024 * 4); }
  size_t offZeros() const { return offDlog() + al(256 * 4); }
  size_t ctlBytes() const { return offZeros() + al(ncol_ * 4); }
};

axon_status MultiRun::plan(const uint32_t* seeds, const uint32_t* nstim) {
  const axon_cfg& cfg = net0_->cfg;
  const uint32_t T = a_.T, CL = a_.clamp_steps, TC = a_.train_clamp;
  plans_.resize(n_);
  size_t off = 0;
  for (uint32_t i = 0; i < n_; ++i) {
    NetPlan& P = plans_[i];
    P.seed = seeds[i];
    P.nstim = nstim[i];
    P.nq = std::min(P.nstim, 12u);
    P.TT = std::min(T + 20u, 40u);
    P.TW = std::min(a_.wave_t, 60u);
    P.pats = make_patterns(P.seed, P.nstim, incols_, a_.stimcols);
    const CueIx X{P.nstim, P.nq};
    P.cues.assign((size_t)X.count() * ncol_, 0u);
    auto cue = [&](uint32_t ix, uint32_t p, double keep, uint32_t seed) {
      make_clamp(P.pats[p], keep, seed, ncol_, P.cues.data() + (size_t)ix * ncol_);
    };
    for (uint32_t p = 0; p < P.nstim; ++p) cue(X.train(p), p, 1.0, 1000 + p);
    cue(X.extra(), 0, 1.0, 31337);
    for (uint32_t p = 0; p < P.nstim; ++p) cue(X.ref(p), p, 1.0, 2000 + p);
    for (uint32_t q = 0; q < P.nstim; ++q) cue(X.rec(q), q, 0.75, 4400 + q);
    for (uint32_t q = 0; q < P.nq; ++q) cue(X.drv(q), q, 1.0, 8600 + q);
    for (uint32_t q = 0; q < P.nq; ++q) cue(X.wave(q), q, 1.0, 7000 + q);
    P.cuesOff = off; off += al(P.cues.size() * 4);
    P.refsOff = off; off += al((size_t)P.nstim * ncol_ * 4);
    P.recOff = off; off += al((size_t)P.nstim * ncol_ * 4);
    P.dlogOff = off; off += al((size_t)P.nq * 256 * 4);
    P.waveOff = off; off += al((size_t)P.nq * P.TW * ncol_ * 4);
    const size_t nprog = (size_t)a_.epochs * P.nstim + 1 + (a_.readout ? 2 * P.nstim + 2 * P.nq : 0);
    P.progOff = off; off += al(nprog * sizeof(MultiPresent));
  }
  ctlOff_ = off;
  if (cudaMalloc(&arena_.p, off + ctlBytes()) != cudaSuccess) {
    cudaGetLastError();
    arena_.p = nullptr;
    return set_error(AXON_ENOMEM, "multi-network arena allocation failed");
  }
  base_ = (char*)arena_.p;
  CK(cudaMemsetAsync(base_, 0, off + ctlBytes(), net0_->stream));

  // programs (device pointers into the arena)
  const uint32_t kRead = cfg.ktest ? cfg.ktest : cfg.k;
  for (uint32_t i = 0; i < n_; ++i) {
    NetPlan& P = plans_[i];
    const CueIx X{P.nstim, P.nq};
    auto pres = [&](uint32_t ix, uint32_t T_, uint32_t clamp_, bool learn) {
      MultiPresent m{};
      m.stim = dev(P.cuesOff) + (size_t)ix * ncol_;
      m.T = T_;
      m.clampSteps = clamp_;
      m.learn = learn ? 1u : 0u;
      m.useBias = learn ? 1u : 0u;  // the bias follows learning unless asked (src/axon.mm:818-822)
      m.k = learn ? cfg.k : kRead;
      m.facil = learn ? 0u : cfg.facil;
      P.steps += T_;
      if (learn) P.trainSteps += T_;
      return m;
    };
    P.prog.clear();
    for (uint32_t ep = 0; ep < a_.epochs; ++ep)
      for (uint32_t p = 0; p < P.nstim; ++p) P.prog.push_back(pres(X.train(p), T, TC, true));
    P.prog.push_back(pres(X.extra(), T, TC, true));
    P.nTrain = (uint32_t)P.prog.size();
    if (a_.readout) {
      for (uint32_t p = 0; p < P.nstim; ++p) {
        MultiPresent m = pres(X.ref(p), T, T, false);
        m.finalOut = dev(P.refsOff) + (size_t)p * ncol_;
        P.prog.push_back(m);
      }
      for (uint32_t q = 0; q < P.nstim; ++q) {
        MultiPresent m = pres(X.rec(q), T, CL, false);
        m.finalOut = dev(P.recOff) + (size_t)q * ncol_;
        P.prog.push_back(m);
      }
      for (uint32_t q = 0; q < P.nq; ++q) {
        MultiPresent m = pres(X.drv(q), P.TT, CL, false);
        m.refBall = dev(P.refsOff) + (size_t)q * ncol_;
        m.driveLog = dev(P.dlogOff) + (size_t)q * 256;
        P.prog.push_back(m);
      }
      for (uint32_t q = 0; q < P.nq; ++q) {
        MultiPresent m = pres(X.wave(q), P.TW, CL, false);
        m.hist = dev(P.waveOff) + (size_t)q * P.TW * ncol_;
        P.prog.push_back(m);
      }
    }
    CK(cudaMemcpyAsync(dev(P.cuesOff), P.cues.data(), P.cues.size() * 4, cudaMemcpyHostToDevice, net0_->stream));
    CK(cudaMemcpyAsync(dev(P.progOff), P.prog.data(), P.prog.size() * sizeof(MultiPresent), cudaMemcpyHostToDevice,
                       net0_->stream));
  }
  CK(cudaStreamSynchronize(net0_->stream));
  return AXON_OK;
}

axon_status MultiRun::init_all() {
  for (uint32_t i = 0; i < n_; ++i) {
    axon_status st = nets_[i]->init(plans_[i].seed);
    if (st != AXON_OK) return st;
  }
  return AXON_OK;
}

// One persistent launch over `queues` (network indices per slot), optionally captured as
// a CUDA graph. nprogOverride, when given, limits each network's program length.
axon_status MultiRun::launch(const Shape& sh, const std::vector<std::vector<uint32_t>>& queues,
                             const std::vector<uint32_t>& ncta, const std::vector<uint32_t>* nprogOverride,
                             bool graph, float* ms, bool* usedGraph) {
  cudaStream_t st = net0_->stream;
  const uint32_t S = (uint32_t)queues.size();
  if (S == 0 || S > kMaxSlots) return set_error(AXON_EINVAL, "bad slot count");
  char* ctl = base_ + ctlOff_;
  MultiNet* dNets = (MultiNet*)ctl;
  MultiSlot* dSlots = (MultiSlot*)(ctl + offSlots());
  uint32_t* dQueue = (uint32_t*)(ctl + offQueue());
  uint32_t* dBars = (uint32_t*)(ctl + offBars());
  uint32_t* dErr = (uint32_t*)(ctl + offErr());

  std::vector<MultiNet> hn(n_);
  for (uint32_t i = 0; i < n_; ++i) {
    hn[i].d = nets_[i]->d;
    hn[i].prog = (const MultiPresent*)dev(plans_[i].progOff);
    hn[i].nprog = nprogOverride ? (*nprogOverride)[i] : (uint32_t)plans_[i].prog.size();
  }
  std::vector<MultiSlot> hs(S);
  std::vector<uint32_t> hq;
  uint32_t cta = 0;
  for (uint32_t s = 0; s < S; ++s) {
    hs[s].cta0 = cta;
    hs[s].ncta = ncta[s];
    cta += ncta[s];
    hs[s].q0 = (uint32_t)hq.size();
    hq.insert(hq.end(), queues[s].begin(), queues[s].end());
    hs[s].q1 = (uint32_t)hq.size();
  }
  CK(cudaMemcpyAsync(dNets, hn.data(), n_ * sizeof(MultiNet), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dSlots, hs.data(), S * sizeof(MultiSlot), cudaMemcpyHostToDevice, st));
  if (!hq.empty()) CK(cudaMemcpyAsync(dQueue, hq.data(), hq.size() * 4, cudaMemcpyHostToDevice, st));

  MultiDev m{};
  m.nets = dNets;
  m.slots = dSlots;
  m.queue = dQueue;
  m.bars = dBars;
  m.err = dErr;
  m.work = reinterpret_cast<unsigned long long*>(dErr + 4);  // 16 bytes into the error word's 64-byte line
  m.nslots = S;
  MultiCfg c = cfg_;
  c.maxCpw = max_cpw(ncta, sh.threads);
  MultiShape shp{};
  shp.threads = sh.threads;
  shp.tiles = sh.tiles;
  shp.grid = (int)cta;
  shp.smem = multi_smem_bytes(ncol_, incols_, c.maxCpw, sh.threads);
  int per = 0;
  CK(multi_max_blocks_per_sm(sh.threads, sh.tiles, shp.smem, &per));
  if (per < 1 || (int)cta > per * net0_->sm_count) return set_error(AXON_EINVAL, "multi-network shape does not fit the GPU");

  auto body = [&]() -> cudaError_t {
    cudaError_t e = cudaMemsetAsync(dBars, 0, (size_t)S * 32 * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(dErr, 0, 32, st);  // error word and work counters
    if (e == cudaSuccess) e = launch_multi(m, c, shp, st);
    return e;
  };
  *usedGraph = false;
  cudaGraphExec_t exec = nullptr;
  if (graph) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const cudaError_t eb = body();
    const cudaError_t ee = cudaStreamEndCapture(st, &g);
    if (eb == cudaSuccess && ee == cudaSuccess && g) {
      const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
      if (ei != cudaSuccess) exec = nullptr;
    }
    if (g) cudaGraphDestroy(g);
    if (!exec) {
      cudaGetLastError();
      return set_error(AXON_ECUDA, "capturing the multi-network launch as a CUDA graph failed");
    }
  }
  CK(cudaEventRecord(net0_->ev0, st));
  if (exec) {
    const cudaError_t e = cudaGraphLaunch(exec, st);
    if (e != cudaSuccess) {
      cudaGraphExecDestroy(exec);
      return cuda_fail(e, "cudaGraphLaunch");
    }
    *usedGraph = true;
  } else {
    CK(body());
  }
  CK(cudaEventRecord(net0_->ev1, st));
  const cudaError_t es = cudaStreamSynchronize(st);
  if (exec) cudaGraphExecDestroy(exec);
  if (es != cudaSuccess) return cuda_fail(es, "multi-network launch");
  CK(cudaEventElapsedTime(ms, net0_->ev0, net0_->ev1));
  uint32_t words[8] = {0};
  CK(cudaMemcpy(words, dErr, 32, cudaMemcpyDeviceToHost));
  const uint32_t err = words[0];
  std::memcpy(lastWork_, words + 4, 16);
  if (err)
    return set_error(AXON_ETIMEOUT, "grid wait timed out in the multi-network kernel (code " + std::to_string(err) + ")");
  return AXON_OK;
}

// The same programs through the plain path: one k_present launch per presentation.
axon_status MultiRun::run_plain(float* ms) {
  cudaStream_t st = net0_->stream;
  char* ctl = base_ + ctlOff_;
  uint32_t* sHist = (uint32_t*)(ctl + offHist());
  uint32_t* sStats = (uint32_t*)(ctl + offStats());
  uint32_t* sDlog = (uint32_t*)(ctl + offDlog());
  uint32_t* zeros = (uint32_t*)(ctl + offZeros());
  CK(cudaMemsetAsync(zeros, 0, ncol_ * 4, st));
  CK(cudaEventRecord(net0_->ev0, st));
  for (uint32_t i = 0; i < n_; ++i) {
    axon_net* net = nets_[i];
    for (const MultiPresent& p : plans_[i].prog) {
      NetDev dd = net->d;
      dd.stim = const_cast<uint32_t*>(p.stim);
      dd.refBall = p.refBall ? const_cast<uint32_t*>(p.refBall) : zeros;
      dd.hist = p.hist ? p.hist : sHist;
      dd.stats = p.stats ? p.stats : sStats;
      dd.driveLog = p.driveLog ? p.driveLog : sDlog;
      dd.finalOut = p.finalOut;
      const PresentCfg pc = net->present_cfg(p.T, p.clampSteps, p.learn != 0u, p.useBias);
      CK(launch_present(dd, pc, net->shape, st));
    }
  }
  CK(cudaEventRecord(net0_->ev1, st));
  CK(cudaStreamSynchronize(st));
  CK(cudaEventElapsedTime(ms, net0_->ev0, net0_->ev1));
  for (uint32_t i = 0; i < n_; ++i) {
    axon_status s = nets_[i]->check_device_error();
    if (s != AXON_OK) return s;
  }
  return AXON_OK;
}

// Times every candidate shape on the networks themselves (kCalPresents learning
// presentations per slot), predicts each candidate's makespan from the measured time per
// step and the LPT assignment of the full programs, and keeps the best. The networks are
// re-initialised by the caller afterwards.
axon_status MultiRun::tune(Shape* best, std::vector<std::vector<uint32_t>>* bestQ, std::vector<uint32_t>* bestCta,
                           float* tuneMs, uint32_t* tried) {
  const uint32_t grid = (uint32_t)net0_->sm_count;
  std::vector<uint64_t> cost(n_);
  for (uint32_t i = 0; i < n_; ++i) cost[i] = plans_[i].steps;
  const uint32_t slotCands[] = {1, 2, 3, 4, 5, 6, 8, 10, 12, 16, 20, 25, 32, 40, 50, 64, 74};
  const int shapeCands[][2] = {{1024, 4}, {896, 4}, {512, 8}};
  double bestT = 1e300;
  *tuneMs = 0.f;
  *tried = 0;
  for (const auto& sc : shapeCands) {
    for (uint32_t S : slotCands) {
      if (S > n_ || S > grid) continue;
      const std::vector<uint32_t> ncta = split_ctas(grid, S);
      if (multi_smem_bytes(ncol_, incols_, max_cpw(ncta, sc[0]), sc[0]) > 227 * 1024) continue;
      // calibration: slot s runs network s for a few learning presentations
      std::vector<std::vector<uint32_t>> q(S);
      std::vector<uint32_t> np(n_, 0u);
      uint64_t stepsPerSlot = 0;  // the longest calibration program of a slot
      for (uint32_t s = 0; s < S; ++s) {
        q[s].push_back(s);
        np[s] = std::min<uint32_t>(kCalPresents, plans_[s].nTrain);
        uint64_t k = 0;
        for (uint32_t j = 0; j < np[s]; ++j) k += plans_[s].prog[j].T;
        stepsPerSlot = std::max(stepsPerSlot, k);
      }
      float ms = 0.f;
      bool g = false;
      const Shape sh{S, sc[0], sc[1]};
      axon_status st = launch(sh, q, ncta, &np, false, &ms, &g);
      if (st != AXON_OK) return st;
      *tuneMs += ms;
      ++*tried;
      const double perStep = stepsPerSlot ? ms / (double)stepsPerSlot : 1e9;  // ms per step of one slot
      std::vector<std::vector<uint32_t>> queues;
      const double span = assign(cost, ncta, queues) * perStep;
      if (span < bestT) {
        bestT = span;
        *best = sh;
        *bestQ = queues;
        *bestCta = ncta;
      }
    }
  }
  if (bestT >= 1e300) return set_error(AXON_EINVAL, "no multi-network shape fits the GPU");
  return AXON_OK;
}

// The measurements of one network from its readout outputs, computed as the reference's
// printing blocks compute them (src/axon.mm:1495-1508, 1695-1730, 1804-1858).
axon_status MultiRun::measure(uint32_t i, axon_multi_result* r) {
  const NetPlan& P = plans_[i];
  axon_net* net = nets_[i];
  cudaStream_t st = net0_->stream;
  const uint32_t ncol = ncol_, incols = incols_, CL = a_.clamp_steps;
  std::vector<uint32_t> refs((size_t)P.nstim * ncol), rec((size_t)P.nstim * ncol), dlog((size_t)P.nq * 256),
      wave((size_t)P.nq * P.TW * ncol);
  CK(cudaMemcpyAsync(refs.data(), dev(P.refsOff), refs.size() * 4, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(rec.data(), dev(P.recOff), rec.size() * 4, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(dlog.data(), dev(P.dlogOff), dlog.size() * 4, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(wave.data(), dev(P.waveOff), wave.size() * 4, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  std::vector<Ids> refCols(P.nstim), refN(P.nstim);
  for (uint32_t q = 0; q < P.nstim; ++q) {
    refCols[q] = active_columns(&refs[(size_t)q * ncol], incols, ncol);
    refN[q] = active_neurons(&refs[(size_t)q * ncol], incols, ncol);
  }
  // the 75% cue row of the completion table
  double s1 = 0, o1 = 0;
  for (uint32_t q = 0; q < P.nstim; ++q) {
    const Ids a = active_columns(&rec[(size_t)q * ncol], incols, ncol);
    s1 += cos_overlap(a, refCols[q]);
    double b1 = 0;
    for (uint32_t o = 0; o < P.nstim; ++o)
      if (o != q) b1 = std::max(b1, cos_overlap(a, refCols[o]));
    o1 += b1;
  }
  r->recall = s1 / P.nstim;
  r->best_other = o1 / P.nstim;
  // within-assembly density over the first 12 references
  double fIn = 0, pIn = 0;
  for (uint32_t q = 0; q < P.nq; ++q) {
    uint32_t out[10] = {0};
    axon_status s = net->within(&refs[(size_t)q * ncol], 0, nullptr, nullptr, out);
    if (s != AXON_OK) return s;
    fIn += out[0];
    pIn += out[1];
  }
  r->within_pct = pIn > 0 ? 100.0 * fIn / pIn : 0.0;
  // free-phase drive to the members at step 6
  double sum6 = 0, cnt6 = 0;
  if (6 < P.TT)
    for (uint32_t q = 0; q < P.nq; ++q) {
      const uint32_t* dl = &dlog[(size_t)q * 256 + 6 * 4];
      sum6 += dl[0] + dl[2];
      cnt6 += dl[1] + dl[3];
    }
  r->drive_t6 = cnt6 ? sum6 / cnt6 : 0.0;
  // wave: neuron-level overlap with the clamped reference at the first free and last step
  auto ov_at = [&](uint32_t t) {
    double s = 0;
    for (uint32_t q = 0; q < P.nq; ++q) {
      const Ids cur = active_neurons(&wave[((size_t)q * P.TW + t) * ncol], incols, ncol);
      const Ids& ref = refN[q];
      s += (cur.empty() || ref.empty()) ? 0.0 : (double)n_common(cur, ref) / std::sqrt((double)cur.size() * ref.size());
    }
    return s / P.nq;
  };
  r->wave_first = CL < P.TW ? ov_at(CL) : 0.0;
  r->wave_last = ov_at(P.TW - 1);
  uint32_t c = 0;
  axon_status s = net->wstat(&c);
  if (s != AXON_OK) return s;
  r->wdens_pct = 100.0 * c / ((double)net->n * 8192.0);
  r->steps = P.steps;
  return AXON_OK;
}

axon_status MultiRun::run(const uint32_t* seeds, const uint32_t* nstim, axon_multi_result* res,
                          axon_multi_report* rep) {
  for (uint32_t i = 0; i < n_; ++i)
    if (!nets_[i]) return set_error(AXON_EINVAL, "null network");
  net0_ = nets_[0];
  const axon_cfg& c0 = net0_->cfg;
  for (uint32_t i = 0; i < n_; ++i) {
    if (nets_[i]->device != net0_->device) return set_error(AXON_EINVAL, "networks must share one device");
    if (std::memcmp(&nets_[i]->cfg, &c0, sizeof(axon_cfg)) != 0)
      return set_error(AXON_EINVAL, "networks must share one configuration");
    for (uint32_t j = 0; j < i; ++j)
      if (nets_[j] == nets_[i]) return set_error(AXON_EINVAL, "a network appears twice");
    if (nstim[i] == 0) return set_error(AXON_EINVAL, "nstim must be >= 1");
  }
  if (a_.T == 0 || a_.T > 64 || a_.train_clamp > 64 || a_.stimcols == 0 || a_.stimcols > c0.incols)
    return set_error(AXON_EINVAL, "bad T, train_clamp or stimcols");
  if (a_.readout && (a_.wave_t == 0 || a_.clamp_steps > a_.T))
    return set_error(AXON_EINVAL, "bad wave_t or clamp_steps");
  if (a_.method > 1) return set_error(AXON_EINVAL, "method must be 0 (one launch) or 1 (plain path)");
  ncol_ = net0_->ncol;
  incols_ = c0.incols;
  CK(cudaSetDevice(net0_->device));
  for (uint32_t i = 0; i < n_; ++i) CK(cudaStreamSynchronize(nets_[i]->stream));

  const PresentCfg pc = net0_->present_cfg(1, 0, true, 1);
  cfg_.ncol = ncol_; cfg_.incols = incols_; cfg_.dthr = pc.dthr; cfg_.boost = pc.boost; cfg_.mode = pc.mode;
  cfg_.targetCols = pc.targetCols; cfg_.biasUp = pc.biasUp; cfg_.biasDown = pc.biasDown; cfg_.biasShift = pc.biasShift;
  cfg_.biasDownEvery = pc.biasDownEvery; cfg_.bandLo = pc.bandLo; cfg_.bandHi = pc.bandHi;
  cfg_.marginGate = pc.marginGate; cfg_.hetero = pc.hetero; cfg_.ltdRep = pc.ltdRep; cfg_.contrast = pc.contrast;
  cfg_.ltdEvery = pc.ltdEvery; cfg_.topkPar = pc.topkPar; cfg_.waitNs = net0_->wait_ns;
  cfg_.missing = net0_->inject_missing;
  net0_->inject_missing = 0;

  axon_status st = plan(seeds, nstim);
  if (st != AXON_OK) return st;
  axon_multi_report R{};
  float ms = 0.f;
  if (a_.method == 1) {
    if ((st = init_all()) != AXON_OK) return st;
    if ((st = run_plain(&ms)) != AXON_OK) return st;
  } else {
    Shape sh;
    std::vector<std::vector<uint32_t>> queues;
    std::vector<uint32_t> ncta;
    if (a_.autotune) {
      if ((st = init_all()) != AXON_OK) return st;
      float tms = 0.f;
      uint32_t tried = 0;
      if ((st = tune(&sh, &queues, &ncta, &tms, &tried)) != AXON_OK) return st;
      R.tune_ms = tms;
      R.tried = tried;
    } else {
      sh.slots = a_.slots ? std::min(a_.slots, n_) : std::min(n_, (uint32_t)net0_->sm_count);
      sh.threads = (a_.threads == 512 || a_.threads == 896) ? (int)a_.threads : 1024;
      sh.tiles = sh.threads == 512 ? 8 : 4;
      if (sh.slots > (uint32_t)net0_->sm_count) return set_error(AXON_EINVAL, "more slots than SMs");
      ncta = split_ctas((uint32_t)net0_->sm_count, sh.slots);
      std::vector<uint64_t> cost(n_);
      for (uint32_t i = 0; i < n_; ++i) cost[i] = plans_[i].steps;
      assign(cost, ncta, queues);
    }
    if ((st = init_all()) != AXON_OK) return st;
    bool g = false;
    if ((st = launch(sh, queues, ncta, nullptr, a_.graph != 0, &ms, &g)) != AXON_OK) return st;
    R.slots = sh.slots;
    R.threads = (uint32_t)sh.threads;
    R.tiles = (uint32_t)sh.tiles;
    R.grid = std::accumulate(ncta.begin(), ncta.end(), 0u);
    R.graph = g ? 1u : 0u;
    R.w3_tiles = lastWork_[0];
    R.learn_tasks = lastWork_[1];
  }
  R.gpu_ms = ms;
  for (uint32_t i = 0; i < n_; ++i) {
    nets_[i]->w3b_valid = false;
    R.steps += plans_[i].steps;
    R.train_steps += plans_[i].trainSteps;
  }
  if (res) {
    for (uint32_t i = 0; i < n_; ++i) {
      std::memset(&res[i], 0, sizeof(res[i]));
      res[i].steps = plans_[i].steps;
      if (a_.readout && (st = measure(i, &res[i])) != AXON_OK) return st;
    }
  }
  if (rep) *rep = R;
  return AXON_OK;
}

}  // namespace

extern "C" axon_status axon_multi_train(axon_net* const* nets, uint32_t n, const uint32_t* seeds, const uint32_t* nstim,
                                        const axon_multi_args* args, axon_multi_result* results,
                                        axon_multi_report* report) {
  if (!nets || !seeds || !nstim || !args || n == 0) return set_error(AXON_EINVAL, "null argument or n == 0");
  if (n > 1024) return set_error(AXON_EINVAL, "at most 1024 networks per call");
  MultiRun r(nets, n, *args);
  return r.run(seeds, nstim, results, report);
}
