// Host side of the batched readout (axon_recall / axon_recall_device).
#include <algorithm>
#include <cstring>

#include "engine.hpp"

using namespace axon;

#define CK(call)                                        \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

axon_status DevArena::ensure(size_t bytes) {
  if (bytes <= cap) return AXON_OK;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  const size_t want = std::max(bytes, cap + cap / 2);
  if (cudaMalloc(&p, want) != cudaSuccess) {
    cudaGetLastError();
    p = nullptr;
    return set_error(AXON_ENOMEM, "device scratch allocation failed");
  }
  cap = want;
  return AXON_OK;
}

void DevArena::release() {
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
}

axon_status axon_net::ensure_w3b() {
  if (w3b_valid) return AXON_OK;
  if (!w3b) {
    if (cudaMalloc(&w3b, plane_words * 4) != cudaSuccess) {
      cudaGetLastError();
      w3b = nullptr;
      return set_error(AXON_ENOMEM, "W3 batch layout allocation failed");
    }
  }
  CK(launch_make_w3r(d.W3, w3b, ncol, stream));
  w3b_valid = true;
  return AXON_OK;
}

namespace {
size_t al(size_t bytes) { return (bytes + 255) & ~(size_t)255; }
}  // namespace

axon_status axon_net::recall(const uint32_t* cues, uint32_t B, const axon_recall_args& a, const uint32_t* refBall,
                             uint32_t* finalOut, uint32_t* hist, uint32_t* stats, uint32_t* driveLog, bool dev,
                             double* ms) {
  if (!initialized) return set_error(AXON_ESTATE, "recall before init");
  if (B == 0) return set_error(AXON_EINVAL, "B must be >= 1");
  // the per-step records (hist, stats, driveLog) and the plain path's network buffers hold
  // 64 steps, as the reference's do; a batched readout that keeps none of them runs longer
  const bool records = hist || stats || driveLog || refBall || a.method == AXON_RECALL_PLAIN;
  if (a.T == 0 || a.T > (records ? 64u : kRecallMaxT))
    return set_error(AXON_EINVAL, records ? "T must be in 1..64 (per-step records or the plain method)"
                                          : "T must be in 1..1024");
  if (a.use_bias > 1 || a.method > 1 || a.contraction > 1 || a.slab > AXON_SLAB_FULL)
    return set_error(AXON_EINVAL, "bad use_bias, method, contraction or slab");
  CK(cudaSetDevice(device));

  // ---- device views of the caller's arrays (copied in when they are host arrays)
  const size_t bn = (size_t)B * ncol;
  const uint32_t* dCues = cues;
  const uint32_t* dRef = refBall;
  uint32_t *dFinal = finalOut, *dHist = hist, *dStats = stats, *dLog = driveLog;
  if (!dev) {
    size_t need = al(bn * 4) + (refBall ? al(bn * 4) : 0) + (finalOut ? al(bn * 4) : 0) +
                  (hist ? al(bn * a.T * 4) : 0) + (stats ? al((size_t)B * 4096) : 0) + (driveLog ? al((size_t)B * 1024) : 0);
    axon_status st = io.ensure(need);
    if (st != AXON_OK) return st;
    char* p = (char*)io.p;
    auto take = [&](size_t bytes) { uint32_t* r = (uint32_t*)p; p += al(bytes); return r; };
    uint32_t* c = take(bn * 4);
    // the clamp reads a cue's input columns only (the first incols words of each row)
    if (cfg.incols > 0)
      CK(cudaMemcpy2DAsync(c, ncol * 4, cues, ncol * 4, cfg.incols * 4, B, cudaMemcpyHostToDevice, stream));
    dCues = c;
    if (refBall) {
      uint32_t* r = take(bn * 4);
      CK(cudaMemcpyAsync(r, refBall, bn * 4, cudaMemcpyHostToDevice, stream));
      dRef = r;
    }
    if (finalOut) dFinal = take(bn * 4);
    if (hist) dHist = take(bn * a.T * 4);
    if (stats) dStats = take((size_t)B * 4096);
    if (driveLog) {
      dLog = take((size_t)B * 1024);
      CK(cudaMemcpyAsync(dLog, driveLog, (size_t)B * 1024, cudaMemcpyHostToDevice, stream));
    }
  }
  if (dStats) CK(cudaMemsetAsync(dStats, 0, (size_t)B * 4096, stream));

  float gpu_ms = 0.f;
  if (a.method == AXON_RECALL_PLAIN) {
    // one persistent presentation launch per trajectory
    const size_t zbytes = al(ncol * 4);
    axon_status st = scratch.ensure(zbytes + al(1024 * 4));
    if (st != AXON_OK) return st;
    uint32_t* zeros = (uint32_t*)scratch.p;
    uint32_t* statsTmp = (uint32_t*)((char*)scratch.p + zbytes);
    CK(cudaMemsetAsync(zeros, 0, ncol * 4, stream));
    const PresentCfg pc = present_cfg(a.T, a.clamp_steps, false, a.use_bias);
    CK(cudaEventRecord(ev0, stream));
    for (uint32_t b = 0; b < B; ++b) {
      NetDev dd = d;
      dd.stim = const_cast<uint32_t*>(dCues) + (size_t)b * ncol;
      dd.refBall = dRef ? const_cast<uint32_t*>(dRef) + (size_t)b * ncol : zeros;
      if (dHist) dd.hist = dHist + (size_t)b * a.T * ncol;
      dd.stats = dStats ? dStats + (size_t)b * 1024 : statsTmp;
      if (!dStats) CK(cudaMemsetAsync(statsTmp, 0, 1024 * 4, stream));
      if (dLog) dd.driveLog = dLog + (size_t)b * 256;
      dd.finalOut = dFinal ? dFinal + (size_t)b * ncol : nullptr;
      CK(launch_present(dd, pc, shape, stream));
    }
    CK(cudaEventRecord(ev1, stream));
  } else {
    if (ncol > 8192) return set_error(AXON_EINVAL, "batched recall supports ncol <= 8192; use the plain method");
    axon_status st = ensure_w3b();
    if (st != AXON_OK) return st;
    const uint32_t ngrp = ncol / 8u;
    const PresentCfg pc = present_cfg(a.T, a.clamp_steps, false, a.use_bias);
    RecallCfg rc{};
    rc.ncol = ncol; rc.incols = cfg.incols; rc.T = a.T; rc.clampSteps = a.clamp_steps;
    rc.useBias = pc.useBias; rc.k = pc.k; rc.dthr = pc.dthr; rc.boost = pc.boost; rc.mode = pc.mode;
    rc.targetCols = pc.targetCols; rc.facil = pc.facil; rc.biasShift = pc.biasShift; rc.topkPar = pc.topkPar;
    rc.waitNs = wait_ns;
    // per-neuron drive fits 16 bits (and two of them one 32-bit shared counter) unless the
    // branches of one neuron can add up to more than 65535
    const uint64_t maxAcc = (cfg.mode == 2 ? 32ull : 32ull * (256ull + cfg.boost)) + cfg.facil;
    rc.acc32 = maxAcc > 65535ull ? 1u : 0u;
    rc.bst = cfg.mode == 1 ? cfg.boost : 0u;
    rc.mma = a.contraction == AXON_CONTRACT_TENSOR ? 1u : 0u;
    rc.slabAllStep = a.slab == AXON_SLAB_FLOOR ? a.clamp_steps + 1u : 0xFFFFFFFFu;
    rc.slabFull = a.slab == AXON_SLAB_FULL ? 1u : 0u;
    const uint32_t maxB = rc.acc32 ? 300u : kRecallMaxB;
    const uint32_t Bc = std::min(B, maxB);  // trajectories per launch
    const size_t bnc = (size_t)Bc * ncol;
    const size_t accBytes = bnc * 32 * (rc.acc32 ? 4 : 2);
    // the afferent cache of the clamped steps: the packed counters' fast write-back path only
    // (no bias, facilitation or drive log), when steps 2.. are clamped and the input columns
    // fill whole groups (a group holding input and recurrent columns changes while clamped)
    const bool useAff = !rc.acc32 && !rc.useBias && rc.facil == 0u && dRef == nullptr && a.clamp_steps >= 2u &&
                        a.T >= 3u && cfg.incols % 8u == 0u;
    const size_t affBytes = useAff ? bnc * 16 * 4 : 0;
    const size_t need = al(2 * bnc * 4) + al(2ull * ngrp * Bc * 8) + al(2ull * ngrp * Bc * 16) + al(4ull * ngrp * 4) + al(bnc * 4) +
                        al(accBytes) + al((size_t)std::max(a.T, 64u) * 4) + al(3ull * Bc * kHistWords * 4) + al((size_t)Bc * 4) +
                        al(affBytes);
    st = scratch.ensure(need);
    if (st != AXON_OK) return st;
    char* p = (char*)scratch.p;
    auto take = [&](size_t bytes) { char* r = p; p += al(bytes); return r; };
    RecallDev rd{};
    rd.W3R = w3b;
    rd.conn = d.conn;
    rd.bias = d.bias;
    rd.mult = d.mult;
    rd.spk = (uint32_t*)take(2 * bnc * 4);
    rd.ent1 = (uint2*)take(2ull * ngrp * Bc * 8);
    rd.entM = (uint4*)take(2ull * ngrp * Bc * 16);
    rd.ecnt = (uint32_t*)take(4ull * ngrp * 4);
    rd.drv = (uint32_t*)take(bnc * 4);
    rd.acc = take(accBytes);
    rd.work = (uint32_t*)take((size_t)std::max(a.T, 64u) * 4);
    rd.thHist = (uint32_t*)take(3ull * Bc * kHistWords * 4);
    rd.thPrev = (uint32_t*)take((size_t)Bc * 4);
    rd.aff = useAff ? (uint32_t*)take(affBytes) : nullptr;
    rd.theta = nullptr;
    rd.bar = d.bar;
    rd.err = d.err;
    RecallShape rs{};
    rs.threads = 896;
    rc.dacc = recall_smem_bytes(ncol, Bc, rc.acc32, 1u) <= kSmemLimitBytes ? 1u : 0u;
    rs.smem = recall_smem_bytes(ncol, Bc, rc.acc32, rc.dacc);
    int per_sm = 0;
    CK(recall_max_blocks_per_sm(rc.acc32, rs.threads, rs.smem, &per_sm));
    if (per_sm < 1) return set_error(AXON_EINVAL, "batched recall kernel does not fit one SM");
    rs.grid = sm_count * per_sm;
    // everything the launches depend on: a captured graph is replayed only for the same key
    const std::vector<uint64_t> key = {(uint64_t)dCues, (uint64_t)dRef, (uint64_t)dFinal, (uint64_t)dHist,
                                       (uint64_t)dStats, (uint64_t)dLog, (uint64_t)scratch.p, (uint64_t)w3b, B, a.T,
                                       a.clamp_steps, a.use_bias, (uint64_t)rs.grid, wait_ns, a.contraction, a.slab};
    const bool graph = a.graph != 0u;
    const bool replay = graph && recallGraph && key == recallKey;
    if (graph && !replay) {
      if (recallGraph) cudaGraphExecDestroy(recallGraph);
      recallGraph = nullptr;
      recallKey.clear();
      CK(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    }
    if (!graph) CK(cudaEventRecord(ev0, stream));
    cudaError_t e = cudaSuccess;  // a failure inside a capture still ends the capture
    for (uint32_t b0 = 0; replay == false && b0 < B; b0 += Bc) {  // one launch per chunk of trajectories
      const uint32_t nb = std::min(Bc, B - b0);
      rc.B = nb;
      rd.stims = dCues + (size_t)b0 * ncol;
      rd.refBall = dRef ? dRef + (size_t)b0 * ncol : nullptr;
      rd.finalOut = dFinal ? dFinal + (size_t)b0 * ncol : nullptr;
      rd.hist = dHist ? dHist + (size_t)b0 * a.T * ncol : nullptr;
      rd.stats = dStats ? dStats + (size_t)b0 * 1024 : nullptr;
      rd.driveLog = dLog ? dLog + (size_t)b0 * 256 : nullptr;
      if (e == cudaSuccess) e = cudaMemsetAsync(rd.spk, 0, (size_t)nb * ncol * 4, stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(rd.ecnt, 0, 2ull * ngrp * 4, stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(rd.work, 0, (size_t)std::max(a.T, 64u) * 4, stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(rd.thHist, 0, 3ull * nb * kHistWords * 4, stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(rd.thPrev, 0, (size_t)nb * 4, stream);
      if (e == cudaSuccess) e = cudaMemsetAsync(d.bar, 0, 4, stream);
      if (e == cudaSuccess) e = launch_recall(rd, rc, rs, stream);
      if (e != cudaSuccess) break;
    }
    if (graph && !replay) {
      cudaGraph_t g = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(stream, &g);
      if (e == cudaSuccess) e = ec;
      if (e == cudaSuccess) e = cudaGraphInstantiate(&recallGraph, g, 0);
      if (g) cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        recallGraph = nullptr;
        return cuda_fail(e, "batched recall graph capture");
      }
      recallKey = key;
    }
    if (e != cudaSuccess) return cuda_fail(e, "launch_recall");
    if (graph) {
      CK(cudaEventRecord(ev0, stream));
      CK(cudaGraphLaunch(recallGraph, stream));
    }
    CK(cudaEventRecord(ev1, stream));
  }
  axon_status st = check_device_error();
  if (st != AXON_OK) return st;
  CK(cudaEventElapsedTime(&gpu_ms, ev0, ev1));
  if (ms) *ms = gpu_ms;
  if (!dev) {
    if (finalOut) CK(cudaMemcpyAsync(finalOut, dFinal, bn * 4, cudaMemcpyDeviceToHost, stream));
    if (hist) CK(cudaMemcpyAsync(hist, dHist, bn * a.T * 4, cudaMemcpyDeviceToHost, stream));
    if (stats) CK(cudaMemcpyAsync(stats, dStats, (size_t)B * 4096, cudaMemcpyDeviceToHost, stream));
    if (driveLog) CK(cudaMemcpyAsync(driveLog, dLog, (size_t)B * 1024, cudaMemcpyDeviceToHost, stream));
    CK(cudaStreamSynchronize(stream));
  }
  return AXON_OK;
}
