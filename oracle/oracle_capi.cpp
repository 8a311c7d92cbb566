// AXON CPU oracle: C entry points for the Python tests (ctypes). TEST INFRASTRUCTURE ONLY.
//
// Mirrors the engine's C ABI (include/axon_capi.h) on the CPU restatement so a test can
// drive both with the same calls and compare every buffer word for word. The per-present
// Params resolution follows present(), src/axon.mm:815-845.
#include <cstring>
#include <random>
#include <vector>

#include "../include/axon_capi.h"
#include "oracle_engine.hpp"
#include "oracle_protocol.hpp"
#include "oracle_rng.hpp"

namespace {

struct OracleNet {
  axon_cfg cfg;
  oracle::Pool pool;
  oracle::Engine E;
  oracle::Params P;
  OracleNet(const axon_cfg& c, unsigned threads) : cfg(c), pool(threads), E(c.ncol, c.incols, &pool) {
    E.topkPar = c.topkpar ? 1u : 0u;
    P.k = c.k; P.dthr = c.dthr; P.boost = c.boost; P.mode = c.mode; P.inCols = c.incols;
    P.targetCols = c.target; P.biasUp = c.biasup; P.biasDown = c.biasdown; P.biasShift = c.biasshift;
    P.bandLo = c.bandlo; P.bandHi = c.contrast ? c.bandhi : 0u; P.marginGate = c.margingate;
    P.hetero = c.hetero; P.ltdRep = c.ltdrep; P.biasDownEvery = c.biasdownevery;
  }
  std::vector<uint32_t>* buf(int which) {
    switch (which) {
      case AXON_BUF_W0: return &E.W[0];
      case AXON_BUF_W1: return &E.W[1];
      case AXON_BUF_W2: return &E.W[2];
      case AXON_BUF_W3: return &E.W[3];
      case AXON_BUF_CONN: return &E.conn;
      case AXON_BUF_SPK_A: return &E.spk[0];
      case AXON_BUF_SPK_B: return &E.spk[1];
      case AXON_BUF_DRIVE: return &E.drive;
      case AXON_BUF_BBITS: return &E.bbits;
      case AXON_BUF_ACC: return &E.acc;
      case AXON_BUF_BIAS: return &E.bias;
      case AXON_BUF_MARG: return &E.marg;
      case AXON_BUF_REFBALL: return &E.refBall;
      case AXON_BUF_DRIVELOG: return &E.driveLog;
      case AXON_BUF_MULT: return &E.mult;
      case AXON_BUF_STIM: return &E.stim;
      case AXON_BUF_STATS: return &E.stats;
      case AXON_BUF_HIST: return &E.hist;
      case AXON_BUF_THETA: return &E.theta;
    }
    return nullptr;
  }
};

}  // namespace

extern "C" {

void* oracle_create(const axon_cfg* cfg, unsigned threads) { return new OracleNet(*cfg, threads ? threads : 1); }
void oracle_destroy(void* h) { delete (OracleNet*)h; }

void oracle_init(void* h, uint32_t seed) {
  OracleNet* o = (OracleNet*)h;
  o->E.init(o->cfg.nand, seed, o->cfg.inbr);
  std::fill(o->E.bias.begin(), o->E.bias.end(), 0u);
  std::fill(o->E.theta.begin(), o->E.theta.end(), 0u);
  std::fill(o->E.stats.begin(), o->E.stats.end(), 0u);
}

// present(), src/axon.mm:815-888, with the stimulus given directly
void oracle_present(void* h, const uint32_t* stim, uint32_t T, uint32_t clampSteps, int learn, int freeze,
                    uint32_t useBias) {
  OracleNet* o = (OracleNet*)h;
  oracle::Engine& E = o->E;
  oracle::Params& P = o->P;
  const axon_cfg& c = o->cfg;
  P.k = learn ? c.k : (c.ktest ? c.ktest : c.k);
  P.facil = learn ? 0u : c.facil;
  P.useBias = (useBias == 2u) ? (learn ? 1u : 0u) : useBias;
  std::copy(stim, stim + c.ncol, E.stim.begin());
  std::fill(E.stats.begin(), E.stats.end(), 0u);
  P.histOn = 1u;
  std::fill(E.spk[0].begin(), E.spk[0].end(), 0u);
  std::fill(E.spk[1].begin(), E.spk[1].end(), 0u);
  for (uint32_t t = 0; t < T; ++t) {
    uint32_t* in = (t & 1) ? E.spk[1].data() : E.spk[0].data();
    uint32_t* out = (t & 1) ? E.spk[0].data() : E.spk[1].data();
    P.step = t; P.learn = learn ? 1u : 0u; P.freeze = freeze ? 1u : 0u;
    P.clamp = (t < clampSteps) ? 1u : 0u;
    P.depress = (learn && (t % 2 == 1)) ? 1u : 0u;
    P.phase = (!learn || !c.contrast) ? 0u
              : ((t < clampSteps) ? 1u : (((t - clampSteps) % c.ltdevery == 0u) ? 2u : 3u));
    E.k_drive(in, P);
    E.k_topk(P);
    E.k_emit(out, P);
    if (learn) E.k_bias(out, P);
    if (learn) E.k_learn(in, out, P);
  }
}

uint64_t oracle_buf_words(void* h, int which) {
  auto* v = ((OracleNet*)h)->buf(which);
  return v ? v->size() : 0;
}
int oracle_read(void* h, int which, uint32_t* host, uint64_t words) {
  auto* v = ((OracleNet*)h)->buf(which);
  if (!v || v->size() != words) return 1;
  std::memcpy(host, v->data(), words * 4);
  return 0;
}
int oracle_write(void* h, int which, const uint32_t* host, uint64_t words) {
  auto* v = ((OracleNet*)h)->buf(which);
  if (!v || v->size() != words) return 1;
  std::memcpy(v->data(), host, words * 4);
  return 0;
}

uint32_t oracle_wstat(void* h) { return ((OracleNet*)h)->E.wstat_count(); }

void oracle_within(void* h, const uint32_t* ball, uint32_t useMask, const uint32_t* postMask, const uint32_t* mult,
                   uint32_t out[10]) {
  OracleNet* o = (OracleNet*)h;
  std::vector<uint32_t> zeros(o->E.N, 0u);
  o->E.k_within(ball, o->cfg.inbr, o->cfg.incols, useMask, postMask ? postMask : zeros.data(),
                mult ? mult : zeros.data(), out);
}
void oracle_indeg(void* h, uint32_t* out) { ((OracleNet*)h)->E.k_indeg(((OracleNet*)h)->cfg.inbr, out); }
void oracle_untouched(void* h, uint32_t* out) { ((OracleNet*)h)->E.k_untouched(((OracleNet*)h)->cfg.inbr, out); }
void oracle_wdiag(void* h, const uint32_t* memb, const uint32_t* asmSpk, uint32_t nstim, uint32_t sel,
                  uint32_t hist48[48]) {
  OracleNet* o = (OracleNet*)h;
  o->E.k_wdiag(memb, asmSpk, nstim, o->cfg.inbr, sel, hist48);
}

// bit-serial ops on n words per plane (k_bstest, src/axon.mm:424-434)
void oracle_bstest(uint32_t op, uint32_t lo, uint32_t hi, uint32_t* a0, uint32_t* a1, uint32_t* a2, uint32_t* a3,
                   const uint32_t* m, uint64_t n) {
  for (uint64_t i = 0; i < n; ++i) {
    if (op == 0) oracle::bs_inc(a0[i], a1[i], a2[i], a3[i], m[i]);
    else if (op == 1) oracle::bs_dec(a0[i], a1[i], a2[i], a3[i], m[i]);
    else oracle::bs_clip(a0[i], a1[i], a2[i], a3[i], lo, hi);
  }
}

// k-of-32 ranking on n columns of 32 values (kwta_ballot_margin, src/axon.mm:134-144):
// out[3i..3i+2] = winners ballot, vk, vk1
void oracle_kwtatest(const uint32_t* v, const uint32_t* k, uint32_t* out, uint32_t n) {
  for (uint32_t i = 0; i < n; ++i) out[3u * i] = oracle::kwta_ballot_margin(v + 32ull * i, k[i], out[3u * i + 1], out[3u * i + 2]);
}

// stimulus patterns of src/axon.mm:793-799: nstim x stimcols column indices
void oracle_stimuli(uint32_t seed, uint32_t nstim, uint32_t incols, uint32_t stimcols, uint32_t* out) {
  std::mt19937 rng(7u + seed * 104729u);
  for (uint32_t p = 0; p < nstim; ++p) {
    std::vector<uint32_t> all(incols);
    for (uint32_t i = 0; i < incols; ++i) all[i] = i;
    oracle::libcxx_shuffle(all, rng);
    std::copy(all.begin(), all.begin() + stimcols, out + (size_t)p * stimcols);
  }
}
// loadStim of src/axon.mm:800-804 over one pattern's column list
void oracle_load_stim(const uint32_t* cols, uint32_t ncols, double keep, uint32_t seed, uint32_t ncol, uint32_t* out) {
  std::fill(out, out + ncol, 0u);
  std::mt19937 r(seed);
  for (uint32_t i = 0; i < ncols; ++i)
    if (oracle::libcxx_canonical(r) <= keep) out[cols[i]] = 0xFFFFFFFFu;
}
// the noisy cue (see oracle::noisy_clamp) of one pattern's column list
void oracle_noisy_cue(const uint32_t* cols, uint32_t ncols, double frac, uint32_t seed, uint32_t ncol, uint32_t* out) {
  std::vector<uint32_t> stim(ncol);
  oracle::noisy_clamp(std::vector<uint32_t>(cols, cols + ncols), frac, seed, stim);
  std::copy(stim.begin(), stim.end(), out);
}
uint32_t oracle_noisy_seed(uint32_t q, uint32_t pct, uint32_t draw) { return oracle::noisy_seed(q, pct, draw); }

// The reference's built-in defaults (src/axon.mm:688-735, restated by the oracle's own
// key parser with no keys given) overridden by `argc` key=value strings, resolved into
// the network configuration struct the oracle and the engine share.
void oracle_cfg(int argc, char** argv, axon_cfg* out) {
  std::vector<char*> av(1 + (size_t)argc);
  static char prog[] = "axon_oracle";
  av[0] = prog;
  for (int i = 0; i < argc; ++i) av[1 + (size_t)i] = argv[i];
  const oracle::Cfg c = oracle::Cfg::parse(argc + 1, av.data());
  std::memset(out, 0, sizeof(*out));
  out->ncol = c.NCOL; out->incols = c.IN_COLS; out->inbr = c.inBranches; out->nand = c.nAnd; out->target = c.targetC;
  out->k = c.K; out->ktest = c.kTest; out->dthr = c.dthr; out->boost = c.boost; out->mode = c.mode;
  out->biasup = c.biasUp; out->biasdown = c.biasDown; out->biasshift = c.biasShift;
  out->biasdownevery = c.biasDownEvery; out->bandlo = c.bandLo; out->bandhi = c.bandHi; out->contrast = c.contrast;
  out->margingate = c.margGate; out->hetero = c.hetero; out->ltdrep = c.ltdRep; out->ltdevery = c.ltdEvery;
  out->facil = c.facil; out->topkpar = c.topkPar;
}

// raw draws of the restated distributions, for known-answer checks
void oracle_uniform_int(uint32_t seed, uint64_t a, uint64_t b, uint32_t n, uint64_t* out) {
  std::mt19937 r(seed);
  for (uint32_t i = 0; i < n; ++i) out[i] = oracle::libcxx_uniform_int(r, a, b);
}
void oracle_canonical(uint32_t seed, uint32_t n, double* out) {
  std::mt19937 r(seed);
  for (uint32_t i = 0; i < n; ++i) out[i] = oracle::libcxx_canonical(r);
}

}  // extern "C"
