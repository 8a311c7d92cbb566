// Recall server: continuous batching of readout trajectories over device-resident networks.
//
// The reference answers one readout at a time (present() with learn = 0,
// src/axon.mm:815-888). The server accepts recall requests (network, cue columns, clamped
// and free steps) at any time and runs them on an internal thread, tick by tick: at every
// tick it admits requests that have arrived into free trajectory slots (the slot count is
// set by the device-memory budget given at creation), advances every admitted trajectory
// by one step in one batched pass (serve.cu), and retires the trajectories whose last step
// ran, with their final spikes. A request's result does not depend on what else is in
// flight: every trajectory reads only its own slot and the network's read-only weights.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "engine.hpp"
#include "serve.cuh"

using namespace axon;

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
size_t al(size_t bytes) { return (bytes + 255) & ~(size_t)255; }

struct Request {
  uint64_t tag = 0;
  uint32_t net = 0, clamp = 0, steps = 0;
  std::vector<uint32_t> cue;
  double arrive = 0, admit = 0;
};

struct Active {
  uint32_t slot;
  uint32_t tloc;
  Request req;
};

struct Done {
  axon_serve_result r;
  std::vector<uint32_t> spk;
};

// A trajectory whose last step ran in the previous tick: its result is read back and
// retired while the next tick runs.
struct Finished {
  axon_serve_result r;
  uint32_t done;  // its row in the done buffer
  uint32_t slot;
};

}  // namespace

struct axon_server {
  std::vector<axon_net*> nets;
  int device = 0, sms = 0;
  uint32_t ncol = 0, incols = 0, nslots = 0, capB = 0;
  uint64_t slotCost = 0, fixedCost = 0;  // device bytes per trajectory slot, and fixed
  ServeCfg cfg{};
  size_t emitSmem = 0;
  cudaStream_t stream = nullptr;
  void* dmem = nullptr;   // slots, entry lists, tables, done buffer, error word
  void* hmem = nullptr;   // pinned tick staging
  void* hdone = nullptr;  // pinned done buffer
  uint32_t* herr = nullptr;  // pinned copy of the error word
  ServeDev dev{};
  size_t stageBytes = 0;
  uint32_t par = 0;  // tick parity of the entry lists
  std::vector<ServeEntry> entH;  // the tick's tables, built on the server thread
  std::vector<ServeGroup> grpH;
  std::vector<ServeBNet> bnH;
  std::vector<uint2> tabH;
  std::vector<uint32_t> cueH;
  std::vector<uint32_t> freeSlots;

  std::mutex mu;
  std::condition_variable cv, cvIdle;
  std::deque<Request> queue;              // by arrival time
  std::vector<std::vector<Active>> act;   // per network, in batch-index order
  size_t nActive = 0;
  std::deque<Done> done;
  bool stop = false;
  axon_status err = AXON_OK;
  std::string errMsg;
  std::thread th;
  // statistics
  uint64_t ticks = 0, sumActive = 0, maxActive = 0, completed = 0;
  double busy = 0, driveS = 0, emitS = 0;
  cudaEvent_t ev[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};  // per tick parity
  // the previous tick, until its results are retired
  std::vector<Finished> pending;
  bool pendingTick = false;
  uint32_t pendingNe = 0, pendingEv = 0;
  size_t nRunning = 0;  // trajectories in the tables (nActive also counts those not yet retired)

  axon_status start(axon_net* const* ns, uint32_t n, uint64_t memBytes);
  void loop();
  axon_status tick();
  axon_status retire_pending();
  void fail(axon_status s, const std::string& m) {
    std::lock_guard<std::mutex> g(mu);
    if (err == AXON_OK) { err = s; errMsg = m; }
    cvIdle.notify_all();
  }
  ~axon_server();
};

#define CKS(call)                                                         \
  do {                                                                    \
    cudaError_t _e = (call);                                              \
    if (_e != cudaSuccess) return cuda_fail(_e, #call);                   \
  } while (0)

axon_status axon_server::start(axon_net* const* ns, uint32_t n, uint64_t memBytes) {
  nets.assign(ns, ns + n);
  axon_net* n0 = nets[0];
  for (uint32_t i = 0; i < n; ++i) {
    if (!nets[i] || !nets[i]->initialized) return set_error(AXON_ESTATE, "serving needs initialised networks");
    if (nets[i]->device != n0->device || nets[i]->ncol != n0->ncol || nets[i]->cfg.incols != n0->cfg.incols)
      return set_error(AXON_EINVAL, "served networks must share device, ncol and incols");
    if (std::memcmp(&nets[i]->cfg, &n0->cfg, sizeof(axon_cfg)) != 0)
      return set_error(AXON_EINVAL, "served networks must share one configuration");
  }
  device = n0->device;
  ncol = n0->ncol;
  incols = n0->cfg.incols;
  sms = n0->sm_count;
  if (ncol > 8192) return set_error(AXON_EINVAL, "serving supports ncol <= 8192");
  const PresentCfg pc = n0->present_cfg(1, 0, false, 0);  // readout parameters (learn = 0)
  cfg.ncol = ncol; cfg.incols = incols; cfg.dthr = pc.dthr; cfg.boost = pc.boost; cfg.mode = pc.mode;
  cfg.targetCols = pc.targetCols; cfg.k = pc.k; cfg.facil = pc.facil; cfg.topkPar = pc.topkPar;
  cfg.bst = cfg.mode == 1 ? cfg.boost : 0u;
  // per-neuron drive fits 16 bits unless one neuron's branches can add up past 65535
  const uint64_t maxAcc = (cfg.mode == 2 ? 32ull : 32ull * (256ull + cfg.boost)) + cfg.facil;
  cfg.acc32 = maxAcc > 65535ull ? 1u : 0u;
  const uint32_t packed = (!cfg.acc32 && cfg.facil == 0u) ? 1u : 0u;
  capB = packed ? kServeMaxB : kServeMaxB32;
  CKS(cudaSetDevice(device));
  for (axon_net* x : nets) {  // the batched tile layout of every served network
    axon_status st = x->ensure_w3b();
    if (st != AXON_OK) return st;
    CKS(cudaStreamSynchronize(x->stream));
  }
  const uint32_t ngrp = ncol / 8u;
  // fixed: network table, entry lists of every network, error word, tick tables' fixed part
  const size_t listBytes = al(2ull * ngrp * kServeMaxB * 8) + al(2ull * ngrp * kServeMaxB * 16) + al(4ull * ngrp * 4);
  const uint64_t fixed = al(n * sizeof(ServeNet)) + n * listBytes + 256 + 1024 + al(n * sizeof(ServeGroup)) +
                         al(n * sizeof(ServeBNet));
  // one slot: its buffers, its share of the done buffer and of the tick tables
  const size_t slotBytes = (size_t)serve_slot_words(ncol, cfg.acc32) * 4;
  const size_t perSlot = slotBytes + (size_t)ncol * 4 + sizeof(ServeEntry) + sizeof(ServeGroup) + sizeof(uint2) +
                         (size_t)incols * 4;
  if (memBytes <= fixed + perSlot) return set_error(AXON_EINVAL, "memory budget below one trajectory slot");
  nslots = (uint32_t)std::min<uint64_t>((memBytes - fixed) / (perSlot + 64), 1u << 16);
  slotCost = perSlot + 64;
  fixedCost = fixed;
  stageBytes = 1024 + al(nslots * sizeof(ServeEntry)) + al((nslots + n) * sizeof(ServeGroup)) +
               al(n * sizeof(ServeBNet)) + al(nslots * sizeof(uint2)) + al((size_t)nslots * incols * 4);
  const size_t netsOff = 0, listsOff = al(n * sizeof(ServeNet)), errOff = listsOff + n * listBytes,
               slotsOff = errOff + 256, stageOff = slotsOff + al((size_t)nslots * slotBytes),
               doneOff = stageOff + al(stageBytes), total = doneOff + al((size_t)nslots * ncol * 4);
  if (cudaMalloc(&dmem, total) != cudaSuccess) {
    cudaGetLastError();
    dmem = nullptr;
    return set_error(AXON_ENOMEM, "server device allocation failed");
  }
  CKS(cudaMallocHost(&hmem, stageBytes));
  CKS(cudaMallocHost(&hdone, (size_t)nslots * ncol * 4));
  CKS(cudaMallocHost((void**)&herr, 64));
  CKS(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  for (auto& evp : ev)
    for (auto& e : evp) CKS(cudaEventCreate(&e));
  char* b = (char*)dmem;
  CKS(cudaMemsetAsync(b + listsOff, 0, n * listBytes + 256, stream));  // list lengths and error word start at zero
  std::vector<ServeNet> hn(n);
  for (uint32_t i = 0; i < n; ++i) {
    char* L = b + listsOff + i * listBytes;
    hn[i].W3 = nets[i]->d.W3;
    hn[i].conn = nets[i]->d.conn;
    hn[i].W3R = nets[i]->w3b;
    hn[i].ent1 = (uint2*)L;
    hn[i].entM = (uint4*)(L + al(2ull * ngrp * kServeMaxB * 8));
    hn[i].ecnt = (uint32_t*)(L + al(2ull * ngrp * kServeMaxB * 8) + al(2ull * ngrp * kServeMaxB * 16));
  }
  CKS(cudaMemcpyAsync(b + netsOff, hn.data(), n * sizeof(ServeNet), cudaMemcpyHostToDevice, stream));
  dev.nets = (const ServeNet*)(b + netsOff);
  dev.slots = (uint32_t*)(b + slotsOff);
  dev.counts = (const uint32_t*)(b + stageOff);  // the tick's tables follow, packed per tick
  dev.doneBuf = (uint32_t*)(b + doneOff);
  dev.err = (uint32_t*)(b + errOff);
  dev.slotWords = serve_slot_words(ncol, cfg.acc32);
  dev.nactw = serve_nactw(ncol);
  dev.waitNs = n0->wait_ns;
  emitSmem = serve_emit_smem_bytes(ncol, incols);
  CKS(serve_prepare(emitSmem));
  CKS(serve_batched_prepare(packed));
  CKS(cudaStreamSynchronize(stream));
  for (uint32_t s = nslots; s-- > 0;) freeSlots.push_back(s);
  act.assign(n, {});
  th = std::thread([this] { loop(); });
  return AXON_OK;
}

axon_server::~axon_server() {
  {
    std::lock_guard<std::mutex> g(mu);
    stop = true;
  }
  cv.notify_all();
  if (th.joinable()) th.join();
  if (stream) cudaStreamSynchronize(stream);
  if (dmem) cudaFree(dmem);
  if (hmem) cudaFreeHost(hmem);
  if (hdone) cudaFreeHost(hdone);
  if (herr) cudaFreeHost(herr);
  for (auto& evp : ev)
    for (auto& e : evp)
      if (e) cudaEventDestroy(e);
  if (stream) cudaStreamDestroy(stream);
}

void axon_server::loop() {
  if (cudaSetDevice(device) != cudaSuccess) { fail(AXON_ECUDA, "cudaSetDevice in the server thread"); return; }
  for (;;) {
    {
      std::unique_lock<std::mutex> g(mu);
      for (;;) {
        if (stop || err != AXON_OK) return;
        if (nActive) break;
        if (!queue.empty()) {
          const double wait = queue.front().arrive - now_s();
          if (wait <= 0) break;
          cv.wait_for(g, std::chrono::duration<double>(std::min(wait, 0.05)));
        } else {
          cvIdle.notify_all();
          cv.wait_for(g, std::chrono::milliseconds(50));
        }
      }
    }
    const double t0 = now_s();
    const axon_status s = tick();
    if (s != AXON_OK) { fail(s, axon_last_error()); return; }
    std::lock_guard<std::mutex> g(mu);
    busy += now_s() - t0;
  }
}

axon_status axon_server::tick() {
  // admission: arrived requests, in arrival order, into free slots, while the request's
  // network has room in its batch
  {
    std::lock_guard<std::mutex> g(mu);
    const double t = now_s();
    while (!queue.empty() && !freeSlots.empty() && queue.front().arrive <= t && act[queue.front().net].size() < capB) {
      Active a{freeSlots.back(), 0u, std::move(queue.front())};
      freeSlots.pop_back();
      queue.pop_front();
      a.req.admit = t;
      act[a.req.net].push_back(std::move(a));
      ++nActive;
      ++nRunning;
    }
  }
  if (nRunning == 0) return retire_pending();
  // the tick's tables: every network's trajectories in batch-index order; a network with
  // many of them is advanced by the batched kernel, the others by the gather kernel
  entH.clear();
  grpH.clear();
  bnH.clear();
  tabH.clear();
  cueH.clear();
  uint32_t ndone = 0;
  for (uint32_t n = 0; n < (uint32_t)act.size(); ++n) {
    const std::vector<Active>& A = act[n];
    if (A.empty()) continue;
    const bool batched = A.size() >= kServeBatchMin;
    if (batched) bnH.push_back(ServeBNet{n, (uint32_t)A.size(), (uint32_t)tabH.size(), 0u});
    uint32_t cont = 0;
    for (const Active& a : A) {
      ServeEntry e{};
      e.slot = a.slot;
      e.net = n;
      e.tloc = a.tloc;
      e.clamp = a.req.clamp;
      if (a.tloc < a.req.clamp) {
        e.ncue = (uint32_t)a.req.cue.size();
        e.cueOff = (uint32_t)cueH.size();
        cueH.insert(cueH.end(), a.req.cue.begin(), a.req.cue.end());
      }
      const bool last = a.tloc + 1 == a.req.steps;
      e.done = last ? ndone++ : 0xFFFFFFFFu;
      e.nextIdx = last ? 0xFFFFFFFFu : cont++;
      if (batched) {
        tabH.push_back(make_uint2(a.slot, a.tloc));
      } else {
        if (grpH.empty() || grpH.back().net != n || grpH.back().n == kServeGroup) {
          ServeGroup gr{};
          gr.net = n;
          grpH.push_back(gr);
        }
        grpH.back().e[grpH.back().n++] = (uint32_t)entH.size();
      }
      entH.push_back(e);
    }
  }
  const uint32_t ne = (uint32_t)entH.size(), ng = (uint32_t)grpH.size(), nb = (uint32_t)bnH.size(),
                 nc = (uint32_t)cueH.size();
  const uint32_t nip = (ncol + kRecallCpi - 1) / kRecallCpi;
  // one upload: [counts, work counter][entries][groups][batched networks][their table][cues]
  const size_t oEnt = 256, oGrp = oEnt + al(ne * sizeof(ServeEntry)), oBn = oGrp + al(ng * sizeof(ServeGroup)),
               oTab = oBn + al(nb * sizeof(ServeBNet)), oCue = oTab + al(tabH.size() * sizeof(uint2)),
               bytes = oCue + (size_t)nc * 4;
  char* h = (char*)hmem;
  uint32_t* cnt = (uint32_t*)h;
  cnt[0] = ne;
  cnt[1] = ng;
  cnt[2] = nb;
  cnt[3] = nb * nip;
  cnt[4] = 0u;  // work counter of the batched kernel
  std::memcpy(h + oEnt, entH.data(), ne * sizeof(ServeEntry));
  if (ng) std::memcpy(h + oGrp, grpH.data(), ng * sizeof(ServeGroup));
  if (nb) std::memcpy(h + oBn, bnH.data(), nb * sizeof(ServeBNet));
  if (!tabH.empty()) std::memcpy(h + oTab, tabH.data(), tabH.size() * sizeof(uint2));
  if (nc) std::memcpy(h + oCue, cueH.data(), (size_t)nc * 4);
  ServeDev td = dev;
  char* ds = (char*)dev.counts;
  td.work = (uint32_t*)(ds + 16);
  td.ent = (const ServeEntry*)(ds + oEnt);
  td.grp = (const ServeGroup*)(ds + oGrp);
  td.bnets = (const ServeBNet*)(ds + oBn);
  td.btab = (const uint2*)(ds + oTab);
  td.cues = (const uint32_t*)(ds + oCue);
  td.par = par;
  // few trajectories: several CTAs share each one's emit (the grid has sms * 2 CTAs)
  td.emitParts = ne * 4u <= (uint32_t)sms * 2u ? 4u : (ne * 2u <= (uint32_t)sms * 2u ? 2u : 1u);
  uint32_t maxBb = 0;
  for (const ServeBNet& bn : bnH) maxBb = std::max(maxBb, bn.B);
  td.dacc = maxBb <= serve_batched_dacc_maxb((!cfg.acc32 && cfg.facil == 0u) ? 1u : 0u) ? 1u : 0u;
  CKS(cudaMemcpyAsync(ds, h, bytes, cudaMemcpyHostToDevice, stream));
  const uint32_t eb = pendingEv ^ 1u;  // this tick's events (the previous tick's are still to be read)
  CKS(cudaEventRecord(ev[eb][0], stream));
  CKS(launch_serve_drive(td, cfg, sms, ng > 0, nb > 0, stream));
  CKS(cudaEventRecord(ev[eb][1], stream));
  CKS(launch_serve_emit(td, cfg, sms, emitSmem, stream, (uint32_t)nets.size()));
  CKS(cudaEventRecord(ev[eb][2], stream));
  // while the GPU runs this tick: the previous tick's results, from the host done buffer
  // (its copy finished before this tick began), then this tick's read-backs into it
  {
    const axon_status st = retire_pending();
    if (st != AXON_OK) return st;
  }
  if (ndone) CKS(cudaMemcpyAsync(hdone, dev.doneBuf, (size_t)ndone * ncol * 4, cudaMemcpyDeviceToHost, stream));
  CKS(cudaMemcpyAsync(herr, dev.err, 4, cudaMemcpyDeviceToHost, stream));
  // the trajectories whose last step runs now leave the tables (retired with the next
  // tick); the others move one step on and keep their order (their next batch indices)
  pending.clear();
  uint32_t ei = 0;
  for (std::vector<Active>& A : act) {
    size_t w = 0;
    for (size_t i = 0; i < A.size(); ++i) {
      Active& a = A[i];
      const ServeEntry& e = entH[ei++];
      if (e.done != 0xFFFFFFFFu) {
        Finished f{};
        f.r.tag = a.req.tag;
        f.r.net = a.req.net;
        f.r.steps = a.req.steps;
        f.r.arrive_s = a.req.arrive;
        f.r.admit_s = a.req.admit;
        f.done = e.done;
        f.slot = a.slot;
        pending.push_back(f);
      } else {
        ++a.tloc;
        if (w != i) A[w] = std::move(a);
        ++w;
      }
    }
    A.resize(w);
  }
  nRunning -= pending.size();
  pendingTick = true;
  pendingNe = ne;
  pendingEv = eb;
  CKS(cudaStreamSynchronize(stream));
  if (herr[0] != 0u) return set_error(AXON_ETIMEOUT, "a copy wait timed out in the serving kernel");
  par ^= 1u;
  return AXON_OK;
}

// Results of the previous tick: final spikes into the result queue, slots back to the
// free list, the tick into the counters.
axon_status axon_server::retire_pending() {
  if (!pendingTick) return AXON_OK;
  pendingTick = false;
  const double t = now_s();
  float msDrive = 0.f, msEmit = 0.f;
  CKS(cudaEventElapsedTime(&msDrive, ev[pendingEv][0], ev[pendingEv][1]));
  CKS(cudaEventElapsedTime(&msEmit, ev[pendingEv][1], ev[pendingEv][2]));
  std::vector<Done> fin(pending.size());
  for (size_t i = 0; i < pending.size(); ++i) {
    fin[i].r = pending[i].r;
    fin[i].r.done_s = t;
    const uint32_t* src = (const uint32_t*)hdone + (size_t)pending[i].done * ncol;
    fin[i].spk.assign(src, src + ncol);
  }
  std::lock_guard<std::mutex> g(mu);
  for (auto& d : fin) done.push_back(std::move(d));
  for (const Finished& f : pending) freeSlots.push_back(f.slot);
  nActive -= pending.size();
  ++ticks;
  driveS += msDrive * 1e-3;
  emitS += msEmit * 1e-3;
  sumActive += pendingNe;
  maxActive = std::max<uint64_t>(maxActive, pendingNe);
  completed += pending.size();
  pending.clear();
  if (nActive == 0 && queue.empty()) cvIdle.notify_all();
  return AXON_OK;
}

extern "C" {

double axon_clock_s(void) { return now_s(); }

axon_status axon_serve_create(axon_net* const* nets, uint32_t n, uint64_t mem_bytes, axon_server** out) {
  if (!nets || !out || n == 0) return set_error(AXON_EINVAL, "null argument or n == 0");
  *out = nullptr;
  axon_server* s = new axon_server();
  const axon_status st = s->start(nets, n, mem_bytes);
  if (st != AXON_OK) {
    delete s;
    return st;
  }
  *out = s;
  return AXON_OK;
}

axon_status axon_serve_submit(axon_server* s, uint32_t net, const uint32_t* cue_cols, uint32_t ncue,
                              uint32_t clamp_steps, uint32_t free_steps, uint64_t tag, double arrive_s) {
  if (!s || (ncue && !cue_cols)) return set_error(AXON_EINVAL, "null argument");
  if (net >= s->nets.size()) return set_error(AXON_EINVAL, "network index out of range");
  if (ncue > s->incols) return set_error(AXON_EINVAL, "more cue columns than input columns");
  for (uint32_t i = 0; i < ncue; ++i)
    if (cue_cols[i] >= s->incols) return set_error(AXON_EINVAL, "cue column outside the input columns");
  if (clamp_steps + free_steps == 0) return set_error(AXON_EINVAL, "a request needs at least one step");
  Request r;
  r.tag = tag;
  r.net = net;
  r.clamp = clamp_steps;
  r.steps = clamp_steps + free_steps;
  r.cue.assign(cue_cols, cue_cols + ncue);
  r.arrive = arrive_s > 0 ? arrive_s : now_s();
  {
    std::lock_guard<std::mutex> g(s->mu);
    if (s->err != AXON_OK) return set_error(s->err, s->errMsg);
    // keep the queue in arrival order (submissions normally come in order)
    auto it = s->queue.end();
    while (it != s->queue.begin() && (it - 1)->arrive > r.arrive) --it;
    s->queue.insert(it, std::move(r));
  }
  s->cv.notify_all();
  return AXON_OK;
}

axon_status axon_serve_poll(axon_server* s, axon_serve_result* res, uint32_t* final_spk, uint32_t max_results,
                            uint32_t* n_out) {
  if (!s || !n_out || (max_results && !res)) return set_error(AXON_EINVAL, "null argument");
  std::lock_guard<std::mutex> g(s->mu);
  uint32_t k = 0;
  while (k < max_results && !s->done.empty()) {
    Done& d = s->done.front();
    res[k] = d.r;
    if (final_spk) std::memcpy(final_spk + (size_t)k * s->ncol, d.spk.data(), (size_t)s->ncol * 4);
    s->done.pop_front();
    ++k;
  }
  *n_out = k;
  if (s->err != AXON_OK) return set_error(s->err, s->errMsg);
  return AXON_OK;
}

axon_status axon_serve_wait_idle(axon_server* s, double timeout_s) {
  if (!s) return set_error(AXON_EINVAL, "null argument");
  std::unique_lock<std::mutex> g(s->mu);
  const auto until = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
  while (s->err == AXON_OK && !(s->queue.empty() && s->freeSlots.size() == s->nslots)) {
    if (s->cvIdle.wait_until(g, until) == std::cv_status::timeout) return set_error(AXON_ETIMEOUT, "server not idle in time");
  }
  if (s->err != AXON_OK) return set_error(s->err, s->errMsg);
  return AXON_OK;
}

axon_status axon_serve_stats(axon_server* s, axon_serve_counters* out) {
  if (!s || !out) return set_error(AXON_EINVAL, "null argument");
  std::lock_guard<std::mutex> g(s->mu);
  std::memset(out, 0, sizeof(*out));
  out->slots = s->nslots;
  out->slot_bytes = s->slotCost;
  out->fixed_bytes = s->fixedCost;
  out->ticks = s->ticks;
  out->completed = s->completed;
  out->mean_batch = s->ticks ? (double)s->sumActive / s->ticks : 0.0;
  out->max_batch = s->maxActive;
  out->busy_s = s->busy;
  out->drive_s = s->driveS;
  out->emit_s = s->emitS;
  out->queued = s->queue.size();
  out->in_flight = s->nslots - (uint32_t)s->freeSlots.size();
  return AXON_OK;
}

axon_status axon_serve_destroy(axon_server* s) {
  delete s;
  return AXON_OK;
}

}  // extern "C"
