// C ABI of the B200 AXON engine: network objects, device memory and launches.
// Declarations and per-function reference citations: include/axon_capi.h.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/axon_capi.h"
#include "engine.hpp"
#include "plain.cuh"
#include "stimulus.hpp"

using namespace axon;

namespace {
thread_local std::string g_err;
axon_status fail(axon_status s, const std::string& msg) {
  g_err = msg;
  return s;
}
}  // namespace

namespace axon {
axon_status cuda_fail(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return AXON_ECUDA;
}
axon_status set_error(axon_status s, const std::string& msg) { return fail(s, msg); }
}  // namespace axon

#define CK(call)                                      \
  do {                                                \
    cudaError_t _e = (call);                          \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

extern "C" {

void axon_cfg_defaults(axon_cfg* c) {
  std::memset(c, 0, sizeof(*c));
  c->ncol = 4096; c->incols = 512; c->inbr = 8; c->nand = 4; c->target = 256; c->k = 6; c->ktest = 0;
  c->dthr = 2; c->boost = 4; c->mode = 1; c->biasup = 0; c->biasdown = 1; c->biasshift = 4;
  c->biasdownevery = 1; c->bandlo = 5; c->bandhi = 11; c->contrast = 0; c->margingate = 1; c->hetero = 0;
  c->ltdrep = 1; c->ltdevery = 1; c->facil = 0; c->topkpar = 1;
}

const char* axon_last_error(void) { return g_err.c_str(); }

axon_status axon_create(const axon_cfg* cfg, int device, axon_net** out) {
  if (!cfg || !out) return fail(AXON_EINVAL, "null argument");
  *out = nullptr;
  std::string why = validate_cfg(*cfg);
  if (!why.empty()) return fail(AXON_EINVAL, why);
  axon_net* n = new axon_net();
  axon_status st = n->create(*cfg, device);
  if (st != AXON_OK) { delete n; return st; }
  *out = n;
  return AXON_OK;
}

axon_status axon_destroy(axon_net* net) {
  if (!net) return AXON_OK;
  net->release();
  delete net;
  return AXON_OK;
}

axon_status axon_init(axon_net* net, uint32_t seed) {
  if (!net) return fail(AXON_EINVAL, "null net");
  return net->init(seed);
}

axon_status axon_present(axon_net* net, const uint32_t* stim, uint32_t T, uint32_t clamp_steps, int learn, int freeze,
                         uint32_t use_bias, double* ms_per_step) {
  if (!net || !stim) return fail(AXON_EINVAL, "null argument");
  return net->present(stim, T, clamp_steps, learn != 0, freeze != 0, use_bias, ms_per_step);
}

uint64_t axon_buf_words(const axon_net* net, axon_buf which) {
  if (!net) return 0;
  return net->buf_words(which);
}

axon_status axon_read(axon_net* net, axon_buf which, uint32_t* host, uint64_t words) {
  if (!net || !host) return fail(AXON_EINVAL, "null argument");
  return net->read(which, host, words);
}

axon_status axon_write(axon_net* net, axon_buf which, const uint32_t* host, uint64_t words) {
  if (!net || !host) return fail(AXON_EINVAL, "null argument");
  return net->write(which, host, words);
}

axon_status axon_wstat(axon_net* net, uint32_t* count) {
  if (!net || !count) return fail(AXON_EINVAL, "null argument");
  return net->wstat(count);
}

axon_status axon_within(axon_net* net, const uint32_t* ball, uint32_t use_mask, const uint32_t* post_mask,
                        const uint32_t* mult, uint32_t out[10]) {
  if (!net || !ball || !out || (use_mask && !post_mask)) return fail(AXON_EINVAL, "null argument");
  return net->within(ball, use_mask, post_mask, mult, out);
}

axon_status axon_indeg(axon_net* net, uint32_t* out_n) {
  if (!net || !out_n) return fail(AXON_EINVAL, "null argument");
  return net->indeg_untouched(0, out_n);
}

axon_status axon_untouched(axon_net* net, uint32_t* out_n) {
  if (!net || !out_n) return fail(AXON_EINVAL, "null argument");
  return net->indeg_untouched(1, out_n);
}

axon_status axon_wdiag(axon_net* net, const uint32_t* memb, const uint32_t* asm_spk, uint32_t nstim, uint32_t sel,
                       uint32_t hist48[48]) {
  if (!net || !memb || !asm_spk || !hist48) return fail(AXON_EINVAL, "null argument");
  return net->wdiag(memb, asm_spk, nstim, sel, hist48);
}

axon_status axon_bstest(int device, uint32_t op, uint32_t lo, uint32_t hi, uint32_t* a0, uint32_t* a1, uint32_t* a2,
                        uint32_t* a3, const uint32_t* m, uint64_t n) {
  if (!a0 || !a1 || !a2 || !a3 || !m || n == 0 || op > 2) return fail(AXON_EINVAL, "bad argument");
  CK(cudaSetDevice(device));
  uint32_t* d = nullptr;
  CK(cudaMalloc(&d, 5 * n * sizeof(uint32_t)));
  uint32_t* planes[4] = {a0, a1, a2, a3};
  cudaError_t e = cudaSuccess;
  for (int p = 0; p < 4 && e == cudaSuccess; ++p) e = cudaMemcpy(d + p * n, planes[p], n * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + 4 * n, m, n * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = launch_bstest(d, d + n, d + 2 * n, d + 3 * n, d + 4 * n, op, lo, hi, n, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  for (int p = 0; p < 4 && e == cudaSuccess; ++p) e = cudaMemcpy(planes[p], d + p * n, n * 4, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "axon_bstest");
  return AXON_OK;
}

axon_status axon_kwtatest(int device, const uint32_t* v, const uint32_t* k, uint32_t* out, uint32_t n) {
  if (!v || !k || !out || n == 0) return fail(AXON_EINVAL, "bad argument");
  CK(cudaSetDevice(device));
  uint32_t* d = nullptr;
  CK(cudaMalloc(&d, (size_t)n * 36u * sizeof(uint32_t)));
  cudaError_t e = cudaMemcpy(d, v, (size_t)n * 32u * 4u, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d + (size_t)n * 32u, k, (size_t)n * 4u, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = launch_kwtatest(d, d + (size_t)n * 32u, d + (size_t)n * 33u, n, 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(out, d + (size_t)n * 33u, (size_t)n * 12u, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "axon_kwtatest");
  return AXON_OK;
}

axon_status axon_clone(const axon_net* src, axon_net** out) {
  if (!src || !out) return fail(AXON_EINVAL, "null argument");
  *out = nullptr;
  axon_net* n = new axon_net();
  axon_status st = n->create(src->cfg, src->device);
  if (st == AXON_OK) st = n->clone_from(*src);
  if (st != AXON_OK) { delete n; return st; }
  *out = n;
  return AXON_OK;
}

axon_status axon_profile_present(axon_net* net, const uint32_t* stim, uint32_t T, uint32_t clamp_steps, int learn,
                                 uint32_t use_bias, double out[6]) {
  if (!net || !stim || !out) return fail(AXON_EINVAL, "null argument");
  if (use_bias > 2) return fail(AXON_EINVAL, "use_bias must be 0, 1 or 2");
  return net->profile_present(stim, T, clamp_steps, learn != 0, use_bias, out);
}

axon_status axon_set_wait_limit(axon_net* net, uint64_t ns) {
  if (!net || ns == 0) return fail(AXON_EINVAL, "bad argument");
  net->wait_ns = ns;
  return AXON_OK;
}

axon_status axon_inject_missing_arrival(axon_net* net, uint32_t missing) {
  if (!net || missing == 0 || missing > 1024) return fail(AXON_EINVAL, "bad argument");
  net->inject_missing = missing;
  return AXON_OK;
}

axon_status axon_stimuli(uint32_t seed, uint32_t nstim, uint32_t incols, uint32_t stimcols, uint32_t* out) {
  if (!out || stimcols > incols) return fail(AXON_EINVAL, "bad argument");
  const auto pats = make_patterns(seed, nstim, incols, stimcols);
  for (uint32_t p = 0; p < nstim; ++p) std::memcpy(out + (size_t)p * stimcols, pats[p].data(), (size_t)stimcols * 4);
  return AXON_OK;
}

axon_status axon_load_stim(const uint32_t* cols, uint32_t ncols, double keep, uint32_t seed, uint32_t ncol,
                           uint32_t* out_ncol) {
  if ((!cols && ncols) || !out_ncol) return fail(AXON_EINVAL, "bad argument");
  for (uint32_t i = 0; i < ncols; ++i)
    if (cols[i] >= ncol) return fail(AXON_EINVAL, "pattern column out of range");
  make_clamp(std::vector<uint32_t>(cols, cols + ncols), keep, seed, ncol, out_ncol);
  return AXON_OK;
}

axon_status axon_noisy_cue(const uint32_t* cols, uint32_t ncols, double frac, uint32_t seed, uint32_t ncol,
                           uint32_t* out_ncol) {
  if ((!cols && ncols) || !out_ncol) return fail(AXON_EINVAL, "bad argument");
  if (!(frac >= 0.0 && frac <= 1.0)) return fail(AXON_EINVAL, "frac must be in [0, 1]");
  std::vector<uint32_t> pat(cols, cols + ncols), sorted(pat);
  std::sort(sorted.begin(), sorted.end());
  for (uint32_t i = 0; i < ncols; ++i) {
    if (sorted[i] >= ncol) return fail(AXON_EINVAL, "pattern column out of range");
    if (i && sorted[i] == sorted[i - 1]) return fail(AXON_EINVAL, "pattern columns must be distinct");
  }
  make_noisy_clamp(pat, frac, seed, ncol, out_ncol);
  return AXON_OK;
}

uint32_t axon_noisy_cue_seed(uint32_t q, uint32_t pct, uint32_t draw) { return noisy_cue_seed(q, pct, draw); }

axon_status axon_recall(axon_net* net, const uint32_t* cues, uint32_t B, const axon_recall_args* args,
                        const uint32_t* ref_ball, uint32_t* final_spk, uint32_t* hist, uint32_t* stats,
                        uint32_t* drive_log, double* gpu_ms) {
  if (!net || !cues || !args) return fail(AXON_EINVAL, "null argument");
  return net->recall(cues, B, *args, ref_ball, final_spk, hist, stats, drive_log, false, gpu_ms);
}

axon_status axon_recall_device(axon_net* net, const uint32_t* cues, uint32_t B, const axon_recall_args* args,
                               const uint32_t* ref_ball, uint32_t* final_spk, uint32_t* hist, uint32_t* stats,
                               uint32_t* drive_log, double* gpu_ms) {
  if (!net || !cues || !args) return fail(AXON_EINVAL, "null argument");
  return net->recall(cues, B, *args, ref_ball, final_spk, hist, stats, drive_log, true, gpu_ms);
}

}  // extern "C"
