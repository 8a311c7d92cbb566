// AXON CPU oracle: the experiment protocol and every printed block.
// TEST INFRASTRUCTURE ONLY (see oracle_engine.hpp).
//
// Restates the host side of rakib-nyc/axon src/axon.mm:660-1909: the key=value parser,
// present(), the training schedule and each readout/analysis block, printing the same
// lines with the same printf formats (the stdout lines are the reference's interface,
// scraped by its bench/*.sh scripts). Timing figures are this CPU's own.
#pragma once
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "oracle_engine.hpp"
#include "oracle_rng.hpp"

namespace oracle {

// argu, src/axon.mm:660-667: exact key followed by '=', last occurrence wins, atoi.
inline uint32_t argu(int argc, char** argv, const char* key, uint32_t dflt) {
  size_t kl = std::strlen(key);
  uint32_t v = dflt;
  for (int i = 1; i < argc; ++i)
    if (!std::strncmp(argv[i], key, kl) && argv[i][kl] == '=') v = (uint32_t)std::atoi(argv[i] + kl + 1);
  return v;
}

// Tunables with the reference defaults, src/axon.mm:688-735.
struct Cfg {
  uint32_t nAnd, targetC, K, dthr, boost, mode, EPOCHS, T, CLAMP, NSTIM, quiet, seed, split,
      unionchar, biasUp, biasDown, biasShift, biasDownEvery, inBranches, STIM_COLS, IN_COLS,
      NCOL, diag, profile, topkPar, vtopk, contrast, bandLo, bandHi, margGate, hetero, vbs,
      ltdRep, ltdEvery, kTest, facil, deep, wave, waveT, trainClamp, cueflip;
  static Cfg parse(int argc, char** argv) {
    Cfg c;
    c.nAnd = argu(argc, argv, "nand", 4);
    c.targetC = argu(argc, argv, "target", 256);
    c.K = argu(argc, argv, "k", 6);
    c.dthr = argu(argc, argv, "dthr", 2);
    c.boost = argu(argc, argv, "boost", 4);
    c.mode = argu(argc, argv, "mode", 1);
    c.EPOCHS = argu(argc, argv, "epochs", 30);
    c.T = argu(argc, argv, "T", 10);
    c.CLAMP = argu(argc, argv, "clampsteps", 5);
    c.NSTIM = argu(argc, argv, "stim", 12);
    c.quiet = argu(argc, argv, "quiet", 0);
    c.seed = argu(argc, argv, "seed", 0);
    c.split = argu(argc, argv, "split", 0);
    c.unionchar = argu(argc, argv, "unionchar", 0);
    c.biasUp = argu(argc, argv, "biasup", 0);
    c.biasDown = argu(argc, argv, "biasdown", 1);
    c.biasShift = argu(argc, argv, "biasshift", 4);
    c.biasDownEvery = argu(argc, argv, "biasdownevery", 1);
    c.inBranches = argu(argc, argv, "inbr", 8);
    c.STIM_COLS = argu(argc, argv, "stimcols", 128);
    c.IN_COLS = argu(argc, argv, "incols", 512);
    c.NCOL = argu(argc, argv, "ncol", 4096);
    c.diag = argu(argc, argv, "diag", 0);
    c.profile = argu(argc, argv, "profile", 0);
    c.topkPar = argu(argc, argv, "topkpar", 1);
    c.vtopk = argu(argc, argv, "vtopk", 0);
    c.contrast = argu(argc, argv, "contrast", 0);
    c.bandLo = argu(argc, argv, "bandlo", 5);
    c.bandHi = argu(argc, argv, "bandhi", 11);
    c.margGate = argu(argc, argv, "margingate", 1);
    c.hetero = argu(argc, argv, "hetero", 0);
    c.vbs = argu(argc, argv, "vbs", 0);
    c.ltdRep = argu(argc, argv, "ltdrep", 1);
    c.ltdEvery = argu(argc, argv, "ltdevery", 1);
    c.kTest = argu(argc, argv, "ktest", 0);
    c.facil = argu(argc, argv, "facil", 0);
    c.deep = argu(argc, argv, "deep", 0);
    c.wave = argu(argc, argv, "wave", 0);
    c.waveT = argu(argc, argv, "wavet", 35);
    c.cueflip = argu(argc, argv, "cueflip", 0);  // not a reference key: noisy-cue recall row
    c.trainClamp = argu(argc, argv, "trainclamp", c.contrast ? c.CLAMP : c.T);
    if (c.biasUp == 1u) {  // "auto" (src/axon.mm:732-735)
      double pr = (double)c.targetC * c.K / (double)(c.NCOL - c.IN_COLS) / NPC;
      c.biasUp = (uint32_t)std::max(2.0, (1.0 - pr) / pr * c.biasDown);
    }
    return c;
  }
  // Inputs the reference accepts but that would index past its fixed buffers or divide
  // by zero. The reference has no guard; the oracle refuses them. Empty = accepted.
  std::string reject_reason() const {
    if (NCOL == 0 || NCOL % 8 != 0) return "ncol must be a positive multiple of 8";
    if (IN_COLS % 8 != 0 || IN_COLS >= NCOL) return "incols must be a multiple of 8 below ncol";
    if (IN_COLS == 0) return "incols must be positive";
    if (inBranches > NSLOT) return "inbr must be <= 32";
    if (ltdEvery == 0 && contrast) return "ltdevery must be >= 1";
    if (T == 0 || T > MAXT) return "T must be in 1..64";
    if (STIM_COLS > IN_COLS) return "stimcols must be <= incols";
    if (NSTIM == 0) return "stim must be >= 1";
    if (cueflip > 100) return "cueflip must be a percentage in 0..100";
    return "";
  }
};

using Cols = std::vector<uint32_t>;

// overlap, src/axon.mm:896-901 (sorted column lists)
inline double overlap(const Cols& a, const Cols& b) {
  if (a.empty() || b.empty()) return 0.0;
  Cols in;
  std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(in));
  return (double)in.size() / std::sqrt((double)a.size() * b.size());
}
inline double jaccard(const Cols& a, const Cols& b) {
  if (a.empty() || b.empty()) return 0.0;
  Cols i, u;
  std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(i));
  std::set_union(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(u));
  return (double)i.size() / u.size();
}

class Protocol {
 public:
  Cfg C;
  Pool pool;
  Engine E;
  Params P;
  std::vector<Cols> stimCols;
  double trainSeconds = 0.0;

  Protocol(const Cfg& c, unsigned threads)
      : C(c), pool(threads), E(c.NCOL, c.IN_COLS, &pool) {
    E.topkPar = C.topkPar ? 1u : 0u;
    P.k = C.K; P.dthr = C.dthr; P.boost = C.boost; P.mode = C.mode; P.inCols = C.IN_COLS;
    P.targetCols = C.targetC; P.biasUp = C.biasUp; P.biasDown = C.biasDown;
    P.biasShift = C.biasShift; P.bandLo = C.bandLo; P.bandHi = C.contrast ? C.bandHi : 0u;
    P.marginGate = C.margGate; P.hetero = C.hetero; P.ltdRep = C.ltdRep;
    P.biasDownEvery = C.biasDownEvery;
  }

  uint32_t N() const { return C.NCOL * NPC; }

  // stimulus patterns, src/axon.mm:793-799
  void make_stimuli() {
    std::mt19937 rng(7u + C.seed * 104729u);
    stimCols.assign(C.NSTIM, {});
    for (uint32_t p = 0; p < C.NSTIM; ++p) {
      std::vector<uint32_t> all(C.IN_COLS);
      for (uint32_t i = 0; i < C.IN_COLS; ++i) all[i] = i;
      libcxx_shuffle(all, rng);
      stimCols[p].assign(all.begin(), all.begin() + C.STIM_COLS);
    }
  }
  // loadStim, src/axon.mm:800-804
  void load_stim(uint32_t p, double keep, uint32_t sd) {
    std::fill(E.stim.begin(), E.stim.end(), 0u);
    std::mt19937 r(sd);
    for (uint32_t c : stimCols[p])
      if (libcxx_canonical(r) <= keep) E.stim[c] = 0xFFFFFFFFu;
  }

  // a readout presentation from a noisy cue (noisy_clamp) instead of loadStim; otherwise
  // present(..., learn = false, freeze = true, useBias = 0)
  void present_noisy(uint32_t p, double frac, uint32_t T_, uint32_t clampSteps, uint32_t sd) {
    P.k = (C.kTest != 0u) ? C.kTest : C.K;
    P.facil = C.facil;
    P.useBias = 0u;
    noisy_clamp(stimCols[p], frac, sd, E.stim);
    std::fill(E.stats.begin(), E.stats.end(), 0u);
    P.histOn = 1u;
    std::fill(E.spk[0].begin(), E.spk[0].end(), 0u);
    std::fill(E.spk[1].begin(), E.spk[1].end(), 0u);
    for (uint32_t t = 0; t < T_; ++t) step(t, clampSteps, false, true);
  }

  // present(), src/axon.mm:815-888; returns wall ms per step
  double present(uint32_t p, double keep, uint32_t T_, uint32_t clampSteps, bool learn,
                 bool freeze, uint32_t sd, uint32_t useBias = 2u) {
    P.k = learn ? C.K : ((C.kTest != 0u) ? C.kTest : C.K);
    P.facil = learn ? 0u : C.facil;
    P.useBias = (useBias == 2u) ? (learn ? 1u : 0u) : useBias;
    load_stim(p, keep, sd);
    std::fill(E.stats.begin(), E.stats.end(), 0u);
    P.histOn = 1u;
    std::fill(E.spk[0].begin(), E.spk[0].end(), 0u);
    std::fill(E.spk[1].begin(), E.spk[1].end(), 0u);
    auto t0 = std::chrono::steady_clock::now();
    for (uint32_t t = 0; t < T_; ++t) step(t, clampSteps, learn, freeze);
    double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return ms / T_;
  }
  void step(uint32_t t, uint32_t clampSteps, bool learn, bool freeze) {
    uint32_t* in = (t & 1) ? E.spk[1].data() : E.spk[0].data();
    uint32_t* out = (t & 1) ? E.spk[0].data() : E.spk[1].data();
    P.step = t; P.learn = learn ? 1u : 0u; P.freeze = freeze ? 1u : 0u;
    P.clamp = (t < clampSteps) ? 1u : 0u;
    P.depress = (learn && (t % 2 == 1)) ? 1u : 0u;
    P.phase = (!learn || !C.contrast) ? 0u
              : ((t < clampSteps) ? 1u : (((t - clampSteps) % C.ltdEvery == 0u) ? 2u : 3u));
    E.k_drive(in, P);
    E.k_topk(P);
    E.k_emit(out, P);
    if (learn) E.k_bias(out, P);
    if (learn) E.k_learn(in, out, P);
  }
  const uint32_t* final_spk(uint32_t T_) const { return (T_ & 1) ? E.spk[1].data() : E.spk[0].data(); }
  Cols assemblyOf(uint32_t T_) const { return colsOf(final_spk(T_)); }
  Cols colsOf(const uint32_t* sp) const {
    Cols v;
    for (uint32_t c = C.IN_COLS; c < C.NCOL; ++c) if (sp[c]) v.push_back(c);
    return v;
  }
  Cols neuronSet(const uint32_t* bal) const {
    Cols r;
    for (uint32_t c = C.IN_COLS; c < C.NCOL; ++c) {
      uint32_t b = bal[c];
      while (b) { uint32_t l = (uint32_t)__builtin_ctz(b); b &= b - 1; r.push_back(c * NPC + l); }
    }
    return r;
  }
  double wstat() {
    std::fill(E.stats.begin(), E.stats.end(), 0u);
    return 100.0 * E.wstat_count() / ((double)N() * FANIN);
  }

  int run();
  void block_vbs();
  void block_vtopk();
  void block_diag(const std::vector<std::vector<uint32_t>>& asmSpkHost);
};

}  // namespace oracle
