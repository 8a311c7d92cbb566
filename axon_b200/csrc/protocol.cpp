// Host protocol of the `axon` command line (see protocol.hpp). Each block names the
// reference lines it restates; printed formats are the reference's (its stdout is the
// interface its bench/*.sh scripts scrape).
#include "protocol.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <stdexcept>

#include "setops.hpp"
#include "stimulus.hpp"

namespace axon {

namespace {

constexpr uint32_t kNpc = 32, kNslot = 32, kPresyn = 256, kFanin = kNslot * kPresyn;

uint32_t argv_u32(int argc, char** argv, const char* key, uint32_t dflt) {
  const size_t kl = std::strlen(key);
  uint32_t v = dflt;
  for (int i = 1; i < argc; ++i)  // last occurrence wins (src/axon.mm:660-667)
    if (std::strncmp(argv[i], key, kl) == 0 && argv[i][kl] == '=') v = (uint32_t)std::atoi(argv[i] + kl + 1);
  return v;
}

struct AxonFailure : std::runtime_error {
  explicit AxonFailure(const std::string& s) : std::runtime_error(s) {}
};
void ok(axon_status s, const char* what) {
  if (s != AXON_OK) throw AxonFailure(std::string(what) + ": " + axon_last_error());
}

// Results of one batched readout.
struct Readout {
  uint32_t B = 0, T = 0, ncol = 0;
  std::vector<uint32_t> fin, hist, stats, dlog;
  const uint32_t* final_of(uint32_t b) const { return fin.data() + (size_t)b * ncol; }
  const uint32_t* row(uint32_t b, uint32_t t) const { return hist.data() + ((size_t)b * T + t) * ncol; }
  const uint32_t* stats_of(uint32_t b) const { return stats.data() + (size_t)b * 1024; }
  const uint32_t* dlog_of(uint32_t b) const { return dlog.data() + (size_t)b * 256; }
};

struct Cue {
  uint32_t p;
  double keep;
  uint32_t seed;
  double flip = 0.0;  // > 0: the whole pattern with this fraction of its active bits flipped off
};

class Session {
 public:
  explicit Session(const CliArgs& a)
      : A(a), ncol(a.ncol), incols(a.incols), n(a.ncol * kNpc), T(a.T), CLAMP(a.clampsteps), NSTIM(a.stim) {}
  ~Session() {
    if (net) axon_destroy(net);
  }
  int run();

 private:
  const CliArgs& A;
  axon_net* net = nullptr;
  const uint32_t ncol, incols, n, T, CLAMP, NSTIM;
  std::vector<std::vector<uint32_t>> pats;
  std::vector<uint32_t> clampw;

  const uint32_t* clamp_words(uint32_t p, double keep, uint32_t seed) {
    clampw.resize(ncol);
    make_clamp(pats[p], keep, seed, ncol, clampw.data());
    return clampw.data();
  }
  // one presentation through the plain path; wall milliseconds per step (the
  // reference times its command buffer on the host clock, src/axon.mm:834-887)
  double present(uint32_t p, double keep, uint32_t T_, uint32_t clamp_, bool learn, uint32_t seed) {
    const uint32_t* w = clamp_words(p, keep, seed);
    const auto t0 = std::chrono::steady_clock::now();
    ok(axon_present(net, w, T_, clamp_, learn ? 1 : 0, learn ? 0 : 1, 2, nullptr), "axon_present");
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return ms / T_;
  }
  Readout readout(const std::vector<Cue>& cues, uint32_t T_, uint32_t clamp_, uint32_t useBias, bool hist, bool stats,
                  const std::vector<const uint32_t*>* refs = nullptr) {
    Readout r;
    r.B = (uint32_t)cues.size();
    r.T = T_;
    r.ncol = ncol;
    std::vector<uint32_t> words((size_t)r.B * ncol), refw;
    for (uint32_t b = 0; b < r.B; ++b) {
      uint32_t* w = &words[(size_t)b * ncol];
      if (cues[b].flip > 0.0) make_noisy_clamp(pats[cues[b].p], cues[b].flip, cues[b].seed, ncol, w);
      else make_clamp(pats[cues[b].p], cues[b].keep, cues[b].seed, ncol, w);
    }
    if (refs) {
      refw.resize((size_t)r.B * ncol);
      for (uint32_t b = 0; b < r.B; ++b) std::memcpy(&refw[(size_t)b * ncol], (*refs)[b], ncol * 4);
      r.dlog.assign((size_t)r.B * 256, 0u);
    }
    r.fin.resize((size_t)r.B * ncol);
    if (hist) r.hist.resize((size_t)r.B * T_ * ncol);
    if (stats) r.stats.resize((size_t)r.B * 1024);
    axon_recall_args a{};
    a.T = T_;
    a.clamp_steps = clamp_;
    a.use_bias = useBias;
    a.method = AXON_RECALL_BATCHED;
    ok(axon_recall(net, words.data(), r.B, &a, refs ? refw.data() : nullptr, r.fin.data(),
                   hist ? r.hist.data() : nullptr, stats ? r.stats.data() : nullptr, refs ? r.dlog.data() : nullptr,
                   nullptr),
       "axon_recall");
    return r;
  }
  std::vector<uint32_t> buffer(axon_buf which) {
    std::vector<uint32_t> v(axon_buf_words(net, which));
    ok(axon_read(net, which, v.data(), v.size()), "axon_read");
    return v;
  }
  double wstat() {  // src/axon.mm:784-791 (also clears the stats counters)
    uint32_t c = 0;
    ok(axon_wstat(net, &c), "axon_wstat");
    std::vector<uint32_t> z(1024, 0u);
    ok(axon_write(net, AXON_BUF_STATS, z.data(), z.size()), "axon_write");
    return 100.0 * c / ((double)n * kFanin);
  }
  std::vector<uint32_t> within(const uint32_t* ball, uint32_t useMask, const uint32_t* post, const uint32_t* mult) {
    std::vector<uint32_t> out(10, 0u);
    ok(axon_within(net, ball, useMask, post, mult, out.data()), "axon_within");
    return out;
  }
  void block_vbs();
  void block_vtopk(const axon_cfg& cfg);
};

void Session::block_vbs() {  // src/axon.mm:903-956
  printf("\n========== BIT-SERIAL VERIFICATION vs SCALAR REFERENCE ==========\n");
  const uint32_t NW = 1 << 14;
  const size_t nbits = (size_t)NW * 4 * 32, nwords = (size_t)NW * 4;
  std::mt19937 r(424242);
  struct Case { const char* name; uint32_t op, lo, hi; };
  const Case cases[] = {{"bs_inc (carry, saturate 15)", 0, 0, 0}, {"bs_dec (BORROW, saturate 0)", 1, 0, 0},
                        {"bs_clip [5,11]", 2, 5, 11}, {"bs_clip [6,10]", 2, 6, 10}, {"bs_clip [4,12]", 2, 4, 12}};
  for (const Case& cs : cases) {
    std::vector<uint8_t> vin(nbits), mk(nbits);
    std::vector<uint32_t> pl[4], pm(nwords, 0u);
    for (auto& p : pl) p.assign(nwords, 0u);
    for (size_t i = 0; i < nbits; ++i) {
      const uint8_t v = r() & 15u, m = r() & 1u;
      vin[i] = v;
      mk[i] = m;
      for (int b = 0; b < 4; ++b)
        if ((v >> b) & 1) pl[b][i >> 5] |= 1u << (i & 31);
      if (m) pm[i >> 5] |= 1u << (i & 31);
    }
    ok(axon_bstest(A.device, cs.op, cs.lo, cs.hi, pl[0].data(), pl[1].data(), pl[2].data(), pl[3].data(), pm.data(),
                   nwords),
       "axon_bstest");
    size_t bad = 0, first = (size_t)-1;
    uint32_t got_first = 0;
    for (size_t i = 0; i < nbits; ++i) {
      uint32_t got = 0;
      for (int b = 0; b < 4; ++b) got |= ((pl[b][i >> 5] >> (i & 31)) & 1u) << b;
      int exp;
      if (cs.op == 0) exp = mk[i] ? std::min(15, vin[i] + 1) : vin[i];
      else if (cs.op == 1) exp = mk[i] ? std::max(0, vin[i] - 1) : vin[i];
      else exp = std::min((int)cs.hi, std::max((int)cs.lo, (int)vin[i]));
      if (exp != (int)got) {
        if (!bad) { first = i; got_first = got; }
        ++bad;
      }
    }
    printf("  %-30s %9zu values  mismatches %zu  %s\n", cs.name, nbits, bad, bad ? "FAIL" : "EXACT");
    if (bad) printf("      first at i=%zu in=%u mask=%u got=%u\n", first, vin[first], mk[first], got_first);
  }
  printf("================================================================\n");
}

void Session::block_vtopk(const axon_cfg& cfg) {  // src/axon.mm:958-994
  printf("\n=============== STEP B: parallel top-K verification ===============\n");
  printf("  serial TG=256 threads | parallel TG=%u threads (max %lu)\n", 1024u, 1024ul);
  // the serial selection runs on a second network with the same seed (identical weights)
  axon_cfg scfg = cfg;
  scfg.topkpar = 0;
  axon_net* sn = nullptr;
  ok(axon_create(&scfg, A.device, &sn), "axon_create");
  ok(axon_init(sn, A.seed), "axon_init");
  axon_cfg pcfg = cfg;
  pcfg.topkpar = 1;
  axon_net* pn = nullptr;
  ok(axon_create(&pcfg, A.device, &pn), "axon_create");
  ok(axon_init(pn, A.seed), "axon_init");
  std::vector<uint32_t> hs(64ull * ncol), hp(64ull * ncol), th(16);
  uint32_t mism = 0, thMism = 0;
  for (uint32_t q = 0; q < NSTIM; ++q) {
    const uint32_t* w = clamp_words(q, 1.0, 9000 + q);
    ok(axon_present(sn, w, T, CLAMP, 0, 1, 2, nullptr), "axon_present");
    ok(axon_present(pn, w, T, CLAMP, 0, 1, 2, nullptr), "axon_present");
    ok(axon_read(sn, AXON_BUF_HIST, hs.data(), hs.size()), "axon_read");
    ok(axon_read(pn, AXON_BUF_HIST, hp.data(), hp.size()), "axon_read");
    for (size_t i = 0; i < (size_t)T * ncol; ++i) mism += hs[i] != hp[i];
    ok(axon_read(sn, AXON_BUF_THETA, th.data(), 16), "axon_read");
    const uint32_t ts = th[0];
    ok(axon_read(pn, AXON_BUF_THETA, th.data(), 16), "axon_read");
    thMism += ts != th[0];
  }
  printf("  winner-set words compared: %zu   MISMATCHES: %u  -> %s\n", (size_t)T * ncol * NSTIM, mism,
         mism ? "FAIL" : "BIT-IDENTICAL");
  printf("  final theta compared: %u stimuli, mismatches %u\n", NSTIM, thMism);
  auto best_of = [&](axon_net* x) {
    double best = 1e30;
    for (int r = 0; r < 5; ++r) {
      const uint32_t* w = clamp_words(0, 1.0, 9999);
      const auto t0 = std::chrono::steady_clock::now();
      ok(axon_present(x, w, T, CLAMP, 0, 1, 2, nullptr), "axon_present");
      best = std::min(best, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() / T);
    }
    return best;
  };
  const double ts = best_of(sn), tp = best_of(pn);
  printf("  full step: serial %.1f us | parallel %.1f us | saved %.1f us (%.1f%% of step)\n", ts * 1000.0, tp * 1000.0,
         (ts - tp) * 1000.0, 100.0 * (ts - tp) / ts);
  axon_destroy(sn);
  axon_destroy(pn);
  printf("==================================================================\n");
}

int Session::run() {
  const axon_cfg cfg = A.engine_cfg();
  const uint32_t trainClamp = A.trainclamp;
  const double PLANE_MB = (double)ncol * kNslot * 2 * 32 * 16 / 1048576.0;
  if (!A.quiet) {  // src/axon.mm:737-747
    printf("======================================================================\n");
    printf(" AXON v0  -  columnar assembly engine, NVIDIA B200\n");
    printf("======================================================================\n");
    printf("  neurons %u (%u cols x %u) | branches %u x %u presyn | fan-in %u | %.2f G syn\n", n, ncol, kNpc, kNslot,
           kPresyn, kFanin, (double)n * kFanin / 1e9);
    printf("  weights 4 planes x %.0f MB = %.0f MB | groups %u\n", PLANE_MB, 4 * PLANE_MB, ncol / 8);
    printf("  nand=%u target=%u k=%u dthr=%u mode=%u epochs=%u T=%u clamp=%u stim=%u biasUp=%u inbr=%u stimcols=%u\n\n",
           A.nand, A.target, A.k, A.dthr, A.mode, A.epochs, T, CLAMP, NSTIM, A.biasup, A.inbr, A.stimcols);
  }
  ok(axon_create(&cfg, A.device, &net), "axon_create");
  ok(axon_init(net, A.seed), "axon_init");
  pats = make_patterns(A.seed, NSTIM, incols, A.stimcols);
  if (A.vbs) block_vbs();
  if (A.vtopk) block_vtopk(cfg);

  const double d0 = wstat();
  if (!A.quiet) printf("initial functional synapse density: %.3f%%  (fan-in %.0f functional)\n\n", d0, d0 / 100.0 * kFanin);

  // settle (src/axon.mm:1001): ten readouts that change no state; the printed line
  // reports the last one, which is the only one whose effect is observable
  present((10 - 1) % NSTIM, 1.0, T, T, false, 999);
  if (!A.quiet) {
    const auto th = buffer(AXON_BUF_THETA);
    const auto st = buffer(AXON_BUF_STATS);
    printf("settled: theta=%u  activeCols/step=%.0f  activeNeurons/step=%.0f\n\n", th[0], (double)st[0] / T,
           (double)st[1] / T);
  }

  // training, src/axon.mm:1008-1026
  double msAcc = 0;
  int msN = 0;
  for (uint32_t ep = 0; ep < A.epochs; ++ep) {
    for (uint32_t p = 0; p < NSTIM; ++p) {
      msAcc += present(p, 1.0, T, trainClamp, true, 1000 + p);
      ++msN;
    }
    if (!A.quiet && (ep % 5 == 4 || ep == 0)) {
      const auto st = buffer(AXON_BUF_STATS);
      const double ltp = st[8], ltd = st[9];
      const uint32_t tp = st[10], td = st[11];
      const double wd = wstat();
      printf("  ep %3u  wdens %7.3f%%  LTP %10.0f  LTD %10.0f  LTD/LTP %6.3f  learners %u/%u\n", ep + 1, wd, ltp, ltd,
             ltp > 0 ? ltd / ltp : 0.0, tp, td);
    }
  }
  if (msN == 0) {
    msAcc = present(0, 1.0, T, T, false, 777);
    msN = 1;
  }
  const double msStep = msAcc / msN;

  // firing steps per neuron under training conditions, src/axon.mm:1032-1072
  {
    present(0, 1.0, T, trainClamp, true, 31337);
    const auto H = buffer(AXON_BUF_HIST);
    std::vector<uint16_t> all(n, 0), clampedC(n, 0), freeC(n, 0);
    std::vector<uint8_t> member(n, 0);
    for (uint32_t t = 0; t < T; ++t)
      for (uint32_t c = incols; c < ncol; ++c)
        for (uint32_t b = H[(size_t)t * ncol + c]; b; b &= b - 1) {
          const uint32_t id = c * kNpc + (uint32_t)__builtin_ctz(b);
          ++all[id];
          (t < trainClamp ? clampedC : freeC)[id]++;
          if (t == T - 1) member[id] = 1;
        }
    double cnt = 0, s = 0, sC = 0, sF = 0, mc = 0, ms = 0, msC = 0, msF = 0;
    std::vector<uint16_t> v, vm;
    for (uint32_t i = incols * kNpc; i < n; ++i) {
      if (all[i]) { cnt++; s += all[i]; sC += clampedC[i]; sF += freeC[i]; v.push_back(all[i]); }
      if (member[i]) { mc++; ms += all[i]; msC += clampedC[i]; msF += freeC[i]; vm.push_back(all[i]); }
    }
    std::sort(v.begin(), v.end());
    std::sort(vm.begin(), vm.end());
    printf("\n================= FIRING STEPS PER NEURON (training) =================\n");
    printf("  T=%u  trainClamp=%u (clamped) + %u (free)\n", T, trainClamp, T - trainClamp);
    printf("  neurons firing at least once: %.0f\n", cnt);
    printf("  mean firing steps  : %.2f   (clamped %.2f + free %.2f)\n", cnt ? s / cnt : 0.0, cnt ? sC / cnt : 0.0,
           cnt ? sF / cnt : 0.0);
    if (!v.empty())
      printf("  p50 %u | p90 %u | max %u   | as fraction of T: %.3f\n", v[v.size() / 2], v[(size_t)(0.9 * (v.size() - 1))],
             v.back(), cnt ? s / cnt / T : 0.0);
    printf("  --- restricted to FINAL-STATE ASSEMBLY MEMBERS (the allocated ones) ---\n");
    printf("  members: %.0f | mean firing steps %.2f (clamped %.2f + free %.2f) | fraction of T %.3f\n", mc,
           mc ? ms / mc : 0.0, mc ? msC / mc : 0.0, mc ? msF / mc : 0.0, mc ? ms / mc / T : 0.0);
    if (!vm.empty())
      printf("  p50 %u | p90 %u | max %u\n", vm[vm.size() / 2], vm[(size_t)(0.9 * (vm.size() - 1))], vm.back());
    printf("  => bias gain per presentation = biasUp * spikes(members) = %.0f\n", mc ? A.biasup * ms / mc : 0.0);
    printf("======================================================================\n");
  }

  // reference assemblies, src/axon.mm:1080-1105: clamped throughout, and cue then release
  std::vector<Cue> cl, fr;
  for (uint32_t p = 0; p < NSTIM; ++p) {
    cl.push_back({p, 1.0, 2000 + p});
    fr.push_back({p, 1.0, 2100 + p});
  }
  const Readout rc = readout(cl, T, T, 0, false, false);
  const Readout rf = readout(fr, T, CLAMP, 0, false, false);
  std::vector<Ids> refCols(NSTIM), freeCols(NSTIM), refN(NSTIM), freeN(NSTIM);
  std::vector<std::vector<uint32_t>> refBal(NSTIM);
  for (uint32_t p = 0; p < NSTIM; ++p) {
    refBal[p].assign(rc.final_of(p), rc.final_of(p) + ncol);
    refCols[p] = active_columns(rc.final_of(p), incols, ncol);
    freeCols[p] = active_columns(rf.final_of(p), incols, ncol);
    refN[p] = active_neurons(rc.final_of(p), incols, ncol);
    freeN[p] = active_neurons(rf.final_of(p), incols, ncol);
  }
  double sz = 0;
  for (auto& a : refCols) sz += a.size();
  sz /= NSTIM;
  double xtalk = 0, xtalkF = 0;
  int xn = 0;
  for (uint32_t i = 0; i < NSTIM; ++i)
    for (uint32_t j = i + 1; j < NSTIM; ++j) {
      xtalk += cos_overlap(refCols[i], refCols[j]);
      xtalkF += cos_overlap(freeCols[i], freeCols[j]);
      ++xn;
    }
  xtalk = xn ? xtalk / xn : 0;
  xtalkF = xn ? xtalkF / xn : 0;

  if (A.diag) {  // counter histogram, src/axon.mm:1107-1151
    std::vector<uint32_t> memb(n, 0u), asmv((size_t)NSTIM * ncol, 0u);
    for (uint32_t q = 0; q < NSTIM; ++q)
      for (uint32_t c = incols; c < ncol; ++c) asmv[(size_t)q * ncol + c] = refBal[q][c];
    for (uint32_t q = 0; q < std::min(NSTIM, 32u); ++q)
      for (uint32_t c = incols; c < ncol; ++c)
        for (uint32_t b = refBal[q][c]; b; b &= b - 1) memb[c * kNpc + (uint32_t)__builtin_ctz(b)] |= 1u << q;
    uint32_t nMember = 0;
    for (uint32_t x : memb) nMember += x != 0u;
    const char* selName[2] = {"RECURRENT branches", "AFFERENT branches"};
    printf("\n======================= STEP 0 DIAGNOSTIC =======================\n");
    printf("4-bit synaptic counter distribution, %u stimuli, %u assembly-member neurons\n", NSTIM, nMember);
    for (uint32_t sel = 0; sel < 2; ++sel) {
      uint32_t h[48] = {0};
      ok(axon_wdiag(net, memb.data(), asmv.data(), NSTIM, sel, h), "axon_wdiag");
      const char* cat[3] = {"within-assembly", "between-assembly", "all"};
      printf("\n--- %s ---\n", selName[sel]);
      printf("  %-17s %10s  %6s %6s %6s | %s\n", "pair type", "count", "mean", "%at 0", "%at 15", "histogram v=0..15");
      for (uint32_t c = 0; c < 3; ++c) {
        double tot = 0, sum = 0;
        for (uint32_t v = 0; v < 16; ++v) { tot += h[c * 16 + v]; sum += (double)v * h[c * 16 + v]; }
        printf("  %-17s %10.0f  %6.2f %6.1f %6.1f | ", cat[c], tot, tot ? sum / tot : 0.0,
               tot ? 100.0 * h[c * 16] / tot : 0.0, tot ? 100.0 * h[c * 16 + 15] / tot : 0.0);
        for (uint32_t v = 0; v < 16; ++v) printf("%s%.1f", v ? "," : "", tot ? 100.0 * h[c * 16 + v] / tot : 0.0);
        printf("\n");
      }
    }
    printf("================================================================\n");
  }

  if (!A.quiet) {  // src/axon.mm:1153-1160
    printf("\n  %.4f ms/timestep -> %.0f steps/s (%.1fx biological real time), wdens %.3f%%\n", msStep, 1000.0 / msStep,
           1.0 / msStep, wstat());
    printf("  assembly size %.1f cols (%.2f%% of area) | cross-talk CLAMPED %.3f  FREE %.3f  (chance %.3f)\n\n", sz,
           100.0 * sz / (ncol - incols), xtalk, xtalkF, sz / (ncol - incols));
    printf("--- pattern completion: cue %u steps, RELEASED %u.  BOTH reference definitions ---\n", CLAMP, T - CLAMP);
    printf("  cue  |  CLAMPED ref: self  other  margin  |  FREE ref: self  other  margin\n");
  }

  if (A.profile) {  // src/axon.mm:1161-1256: one learning presentation of pattern 0, timed per phase
    axon_net* pn = nullptr;
    ok(axon_clone(net, &pn), "axon_clone");  // on a copy: profiling changes no weight of the run
    const uint32_t* w = clamp_words(0, 1.0, 5555);
    double o[6] = {0, 0, 0, 0, 0, 0};
    const auto t0 = std::chrono::steady_clock::now();
    const axon_status st = axon_profile_present(pn, w, T, CLAMP, 1, 2, o);
    const double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count() / T;
    axon_destroy(pn);
    ok(st, "axon_profile_present");
    const char* rows[4] = {"drive + k-of-32 (k_drive)", "grid barrier", "threshold + emit (k_topk, k_emit)",
                           "records, bias, learn (k_bias, k_learn)"};
    printf("\n============= PER-PHASE GPU PROFILE (device timer, one persistent launch) =============\n");
    printf("  %u timesteps, cue %u steps, learning ON, on a copy of the network\n", T, CLAMP);
    printf("  %-40s %10s %10s\n", "phase", "us/step", "% of step");
    for (int k = 0; k < 4; ++k) printf("  %-40s %10.1f %10.1f\n", rows[k], o[k], o[4] > 0 ? 100.0 * o[k] / o[4] : 0.0);
    printf("  %-40s %10.1f %10.1f\n", "TOTAL", o[4], 100.0);
    printf("  launch %.3f ms/step | wall %.3f ms/step\n", o[5] / T, wall);
    printf("  the five kernels run fused in one launch: a per-kernel ablation does not apply\n");
    printf("========================================================================================\n");
  }

  // STEP A1: in-degree and winner identity, src/axon.mm:1343-1409
  std::vector<uint32_t> indeg(n);
  ok(axon_indeg(net, indeg.data()), "axon_indeg");
  const std::vector<uint32_t> bias = buffer(AXON_BUF_BIAS);
  {
    std::vector<uint32_t> v(indeg.begin() + (size_t)incols * kNpc, indeg.end());
    std::vector<uint32_t> sv = v;
    std::sort(sv.begin(), sv.end());
    auto pct = [&](double q) { return sv[(size_t)(q * (sv.size() - 1))]; };
    const double mean = std::accumulate(v.begin(), v.end(), 0.0) / v.size();
    double var = 0;
    for (uint32_t x : v) var += (x - mean) * (x - mean);
    const double sd = std::sqrt(var / v.size());
    printf("\n=============================== STEP A1 ===============================\n");
    printf("Functional in-degree over the %u RECURRENT branches (popcount of MSB plane)\n", kNslot - A.inbr);
    printf("  n=%zu neurons   mean %.1f   sd %.1f   cv %.3f\n", v.size(), mean, sd, sd / mean);
    printf("  min %u | p10 %u | p25 %u | p50 %u | p75 %u | p90 %u | p99 %u | p99.9 %u | max %u\n", sv.front(), pct(0.10),
           pct(0.25), pct(0.50), pct(0.75), pct(0.90), pct(0.99), pct(0.999), sv.back());
    printf("  tail ratio p99/p50 = %.2f   max/p50 = %.2f\n", (double)pct(0.99) / pct(0.50), (double)sv.back() / pct(0.50));
    for (int which = 0; which < 2; ++which) {
      const auto& sets = which ? refN : freeN;
      double jm = 0, jmax = 0;
      int jn = 0;
      for (uint32_t i = 0; i < NSTIM; ++i)
        for (uint32_t j = i + 1; j < NSTIM; ++j) {
          const double x = jaccard(sets[i], sets[j]);
          jm += x;
          ++jn;
          jmax = std::max(jmax, x);
        }
      std::vector<uint32_t> wins(n, 0);
      for (auto& s : sets) for (uint32_t x : s) ++wins[x];
      uint32_t nAll = 0, nNone = 0, nAny = 0;
      double dAll = 0, dNone = 0, dAny = 0, bAll = 0, bNone = 0, bAny = 0;
      for (uint32_t id = incols * kNpc; id < n; ++id) {
        if (wins[id] >= NSTIM - 1) { ++nAll; dAll += indeg[id]; bAll += bias[id]; }
        if (wins[id] == 0) { ++nNone; dNone += indeg[id]; bNone += bias[id]; }
        if (wins[id] > 0) { ++nAny; dAny += indeg[id]; bAny += bias[id]; }
      }
      printf("\n  --- winner identity, %s endpoint ---\n", which ? "CLAMPED" : "FREE-RUN");
      printf("    mean pairwise Jaccard %.3f (max %.3f) over %d pairs, mean set size %.0f\n", jm / jn, jmax, jn,
             (double)sets[0].size());
      printf("    neurons winning in >=%u/%u stimuli: %6u  in-degree %6.1f  intrinsic-bias %8.1f\n", NSTIM - 1, NSTIM,
             nAll, nAll ? dAll / nAll : 0.0, nAll ? bAll / nAll : 0.0);
      printf("    neurons winning in any stimulus  : %6u  in-degree %6.1f  intrinsic-bias %8.1f\n", nAny,
             nAny ? dAny / nAny : 0.0, nAny ? bAny / nAny : 0.0);
      printf("    neurons never winning            : %6u  in-degree %6.1f  intrinsic-bias %8.1f\n", nNone,
             nNone ? dNone / nNone : 0.0, nNone ? bNone / nNone : 0.0);
      printf("    HUB RATIO (winners-in-all / never) = %.3f\n",
             (nNone && dNone) ? (dAll / std::max(1u, nAll)) / (dNone / nNone) : 0.0);
    }
    printf("======================================================================\n");
  }

  // STEP A3 + A4, src/axon.mm:1412-1511
  {
    const double npool = (double)(ncol - incols) * kNpc;
    double msz = 0;
    for (auto& s : refN) msz += s.size();
    msz /= NSTIM;
    const double eInt = msz * msz / npool, eJac = eInt / (2.0 * msz - eInt);
    double jm = 0, jmax = 0, totInt = 0;
    int jn = 0;
    for (uint32_t i = 0; i < NSTIM; ++i)
      for (uint32_t j = i + 1; j < NSTIM; ++j) {
        const double x = jaccard(refN[i], refN[j]);
        jm += x;
        ++jn;
        jmax = std::max(jmax, x);
        totInt += n_common(refN[i], refN[j]);
      }
    Ids uni;
    for (auto& s : refN) uni.insert(uni.end(), s.begin(), s.end());
    dedup(uni);
    const double sumSz = msz * NSTIM;
    printf("\n=============================== STEP A3 ===============================\n");
    printf("Chance baseline for %u assemblies of %.0f neurons from a pool of %.0f\n", NSTIM, msz, npool);
    printf("  E[|A n B|] = m^2/n            = %.2f neurons\n", eInt);
    printf("  E[Jaccard] = E/(2m-E)         = %.5f      <-- CHANCE\n", eJac);
    printf("  measured mean pairwise Jaccard = %.5f   (max %.5f)\n", jm / jn, jmax);
    printf("  ratio measured/chance          = %.3f\n", eJac > 0 ? (jm / jn) / eJac : 0.0);
    printf("  total pairwise overlap: measured %.0f neurons vs %.0f expected at chance (%.1fx less)\n", totInt,
           eInt * jn, totInt > 0 ? eInt * jn / totInt : 1e9);
    printf("  sum of assembly sizes %.0f | union %zu | excess %.0f  -> %s\n", sumSz, uni.size(),
           sumSz - (double)uni.size(), (sumSz - (double)uni.size()) < 0.02 * sumSz ? "NEAR-EXACT PARTITION" : "overlapping");

    std::vector<Cue> nb;
    for (uint32_t q = 0; q < NSTIM; ++q) nb.push_back({q, 1.0, 2200 + q});
    const Readout rnb = readout(nb, T, T, 0, false, false);
    std::vector<Ids> nbCols(NSTIM);
    for (uint32_t q = 0; q < NSTIM; ++q) nbCols[q] = active_columns(rnb.final_of(q), incols, ncol);
    double preserve = 0;
    for (uint32_t q = 0; q < NSTIM; ++q) preserve += cos_overlap(nbCols[q], refCols[q]);
    preserve /= NSTIM;
    double xNB = 0;
    int xn2 = 0;
    for (uint32_t i = 0; i < NSTIM; ++i)
      for (uint32_t j = i + 1; j < NSTIM; ++j) { xNB += cos_overlap(nbCols[i], nbCols[j]); ++xn2; }
    xNB /= xn2;
    printf("\n=============================== STEP A4 ===============================\n");
    printf("Zero the intrinsic bias at TEST time only. Trained weights unchanged.\n");
    printf("  clamped assembly preserved when bias is zeroed: overlap %.3f\n", preserve);
    printf("  cross-talk of clamped assemblies, bias OFF     : %.3f  (bias ON: %.3f)\n", xNB, xtalk);

    printf("\n  release trajectory, cue 75%%, bias OFF at test (vs bias ON baseline)\n");
    printf("  step  phase   ov(clampRef,biasON)  ov(clampRef,biasOFF)  ov(noBiasRef,biasOFF)\n");
    std::vector<Cue> tr;
    for (uint32_t q = 0; q < NSTIM; ++q) tr.push_back({q, 0.75, 4300 + q});
    const Readout ron = readout(tr, T, CLAMP, 1, true, false);
    const Readout roff = readout(tr, T, CLAMP, 0, true, false);
    std::vector<double> a1(T, 0), a2(T, 0), a3(T, 0);
    for (uint32_t q = 0; q < NSTIM; ++q)
      for (uint32_t t = 0; t < T; ++t) {
        a1[t] += cos_overlap(active_columns(ron.row(q, t), incols, ncol), refCols[q]);
        const Ids x = active_columns(roff.row(q, t), incols, ncol);
        a2[t] += cos_overlap(x, refCols[q]);
        a3[t] += cos_overlap(x, nbCols[q]);
      }
    for (uint32_t t = 0; t < T; ++t)
      printf("  %4u  %-5s %19.3f %21.3f %22.3f\n", t, t < CLAMP ? "cue" : "FREE", a1[t] / NSTIM, a2[t] / NSTIM,
             a3[t] / NSTIM);

    printf("\n  pattern completion with bias OFF at test  (keep=0 is the no-cue control)\n");
    printf("  cue  |  vs CLAMPED ref(biasON): self  other  margin | vs noBias ref: self  other  margin\n");
    const double keeps[] = {1.0, 0.75, 0.5, 0.35, 0.25, 0.15, 0.10, 0.05, 0.02, 0.0};
    std::vector<Cue> comp;
    for (double k : keeps)
      for (uint32_t q = 0; q < NSTIM; ++q) comp.push_back({q, k, 4400 + q});
    // cueflip=P (no counterpart in the reference): one more row, the whole pattern with P%
    // of its active bits flipped off (axon_noisy_cue, draw 0)
    const size_t nrows = A.cueflip ? 11 : 10;
    if (A.cueflip)
      for (uint32_t q = 0; q < NSTIM; ++q) comp.push_back({q, 1.0, noisy_cue_seed(q, A.cueflip, 0), A.cueflip / 100.0});
    const Readout rcp = readout(comp, T, CLAMP, 0, false, false);
    for (size_t ki = 0; ki < nrows; ++ki) {
      double s1 = 0, o1 = 0, s2 = 0, o2 = 0;
      for (uint32_t q = 0; q < NSTIM; ++q) {
        const Ids a = active_columns(rcp.final_of((uint32_t)(ki * NSTIM + q)), incols, ncol);
        s1 += cos_overlap(a, refCols[q]);
        s2 += cos_overlap(a, nbCols[q]);
        double b1 = 0, b2 = 0;
        for (uint32_t r = 0; r < NSTIM; ++r)
          if (r != q) { b1 = std::max(b1, cos_overlap(a, refCols[r])); b2 = std::max(b2, cos_overlap(a, nbCols[r])); }
        o1 += b1;
        o2 += b2;
      }
      if (ki < 10)
        printf("  %3.0f%% |%25.3f %6.3f %+7.3f |%18.3f %6.3f %+7.3f\n", keeps[ki] * 100, s1 / NSTIM, o1 / NSTIM,
               s1 / NSTIM - o1 / NSTIM, s2 / NSTIM, o2 / NSTIM, s2 / NSTIM - o2 / NSTIM);
      else
        printf("  flip%3u%% |%21.3f %6.3f %+7.3f |%18.3f %6.3f %+7.3f\n", A.cueflip, s1 / NSTIM, o1 / NSTIM,
               s1 / NSTIM - o1 / NSTIM, s2 / NSTIM, o2 / NSTIM, s2 / NSTIM - o2 / NSTIM);
    }
    printf("======================================================================\n");
  }

  // A4b + A4c, src/axon.mm:1514-1599
  {
    std::vector<uint32_t> unt(n);
    ok(axon_untouched(net, unt.data()), "axon_untouched");
    const double RECSYN = (double)(kNslot - A.inbr) * kPresyn;
    const double cues[4] = {1.0, 0.75, 0.35, 0.15};
    printf("\n=============================== A4b ===============================\n");
    printf("Is the recalled ~25%% a FIXED subset? (readout gate on: bias off at test)\n");
    std::vector<Cue> cs;
    for (uint32_t q = 0; q < NSTIM; ++q)
      for (int ci = 0; ci < 4; ++ci) cs.push_back({q, cues[ci], 5000 + q * 16 + (uint32_t)ci});
    const Readout r = readout(cs, T, CLAMP, 0, false, false);
    auto rec = [&](uint32_t q, int ci) { return active_neurons(r.final_of(q * 4 + (uint32_t)ci), incols, ncol); };
    std::vector<std::vector<Ids>> R(NSTIM, std::vector<Ids>(4));
    for (uint32_t q = 0; q < NSTIM; ++q)
      for (int ci = 0; ci < 4; ++ci) R[q][ci] = rec(q, ci);
    printf("  pairwise Jaccard of recalled sets ACROSS cue levels, same stimulus:\n    ");
    double jall = 0;
    int jn = 0;
    for (int a = 0; a < 4; ++a)
      for (int b = a + 1; b < 4; ++b) {
        double m = 0;
        for (uint32_t q = 0; q < NSTIM; ++q) m += jaccard(R[q][a], R[q][b]);
        m /= NSTIM;
        printf("%.0f%%/%.0f%%=%.3f  ", cues[a] * 100, cues[b] * 100, m);
        jall += m;
        ++jn;
      }
    printf("\n    mean across cue pairs = %.3f\n", jall / jn);
    double coreSz = 0, periSz = 0, asmSz = 0, dCore = 0, dPeri = 0, uCore = 0, uPeri = 0;
    size_t nCore = 0, nPeri = 0;
    for (uint32_t q = 0; q < NSTIM; ++q) {
      Ids core = R[q][0];
      for (int ci = 1; ci < 4; ++ci) core = common(core, R[q][ci]);
      const Ids& As = refN[q];
      const Ids coreInA = common(core, As), peri = minus(As, core);
      coreSz += coreInA.size();
      periSz += peri.size();
      asmSz += As.size();
      for (uint32_t x : coreInA) { dCore += indeg[x]; uCore += 100.0 * unt[x] / RECSYN; ++nCore; }
      for (uint32_t x : peri) { dPeri += indeg[x]; uPeri += 100.0 * unt[x] / RECSYN; ++nPeri; }
    }
    printf("\n  assembly %.0f neurons | CORE (recalled at all 4 cues) %.0f (%.1f%%) | periphery %.0f\n", asmSz / NSTIM,
           coreSz / NSTIM, 100.0 * coreSz / asmSz, periSz / NSTIM);
    printf("  %-12s %10s %14s %22s\n", "group", "n", "in-degree", "%% synapses still at 5/6");
    printf("  %-12s %10zu %14.1f %22.1f\n", "CORE", nCore, nCore ? dCore / nCore : 0.0, nCore ? uCore / nCore : 0.0);
    printf("  %-12s %10zu %14.1f %22.1f\n", "periphery", nPeri, nPeri ? dPeri / nPeri : 0.0, nPeri ? uPeri / nPeri : 0.0);
    double allD = 0, allU = 0;
    size_t nAll = 0;
    for (uint32_t id = incols * kNpc; id < n; ++id) { allD += indeg[id]; allU += 100.0 * unt[id] / RECSYN; ++nAll; }
    printf("  %-12s %10zu %14.1f %22.1f\n", "all neurons", nAll, allD / nAll, allU / nAll);

    std::vector<uint32_t> bv(bias.begin() + (size_t)incols * kNpc, bias.end());
    std::sort(bv.begin(), bv.end());
    const double bm = std::accumulate(bv.begin(), bv.end(), 0.0) / bv.size();
    printf("\n=============================== A4c ===============================\n");
    printf("Intrinsic bias growth after %u epochs (unbounded, non-leaky, learning-time only)\n", A.epochs);
    printf("  mean %.0f | p50 %u | p99 %u | max %u | UINT32_MAX %u | headroom %.3g x\n", bm, bv[bv.size() / 2],
           bv[(size_t)(0.99 * (bv.size() - 1))], bv.back(), 4294967295u, bv.back() ? 4294967295.0 / bv.back() : 0.0);
    printf("  growth rate ~= %.1f per epoch (max/epochs) -> epochs to saturate ~ %.3g\n",
           A.epochs ? (double)bv.back() / A.epochs : 0.0,
           (bv.back() && A.epochs) ? 4294967295.0 / ((double)bv.back() / A.epochs) : 0.0);
    printf("==================================================================\n");
  }

  // assembly multiplicity, as the reference writes it into its mult buffer (src/axon.mm:1604-1607)
  std::vector<uint32_t> mult(n, 0u);
  auto set_mult = [&]() {
    std::fill(mult.begin(), mult.end(), 0u);
    for (uint32_t q = 0; q < NSTIM; ++q) for (uint32_t x : refN[q]) ++mult[x];
    ok(axon_write(net, AXON_BUF_MULT, mult.data(), n), "axon_write");
  };
  const uint32_t NQ12 = std::min(NSTIM, 12u);
  std::vector<const uint32_t*> refp(NSTIM);
  for (uint32_t q = 0; q < NSTIM; ++q) refp[q] = refBal[q].data();

  if (A.unionchar) {  // visited-union characterisation, src/axon.mm:1602-1652
    set_mult();
    std::vector<Cue> cs;
    for (uint32_t q = 0; q < NQ12; ++q) cs.push_back({q, 1.0, 9500 + q});
    const Readout r = readout(cs, 35, CLAMP, 0, true, false);
    Ids allRec;
    for (uint32_t id = incols * kNpc; id < n; ++id) allRec.push_back(id);
    double nIn = 0, nOut = 0, fI = 0, pI = 0, fO = 0, pO = 0, fA = 0, pA = 0, mOut = 0, mAll = 0, nAllR = 0;
    std::vector<uint32_t> post(n);
    auto runW = [&](const uint32_t* ball, const Ids& ps, double& f, double& pp) {
      std::fill(post.begin(), post.end(), 0u);
      for (uint32_t x : ps) post[x] = 1u;
      const auto w = within(ball, 1, post.data(), mult.data());
      f += w[0];
      pp += w[1];
    };
    for (uint32_t q = 0; q < NQ12; ++q) {
      Ids uni;
      for (uint32_t t = CLAMP; t < 35u; ++t) {
        const Ids x = active_neurons(r.row(q, t), incols, ncol);
        uni.insert(uni.end(), x.begin(), x.end());
      }
      dedup(uni);
      const Ids in_ = common(uni, refN[q]), out_ = minus(uni, refN[q]);
      nIn += in_.size();
      nOut += out_.size();
      runW(refp[q], in_, fI, pI);
      runW(refp[q], out_, fO, pO);
      runW(refp[q], allRec, fA, pA);
      for (uint32_t x : out_) mOut += mult[x];
      for (uint32_t x : allRec) mAll += mult[x];
      nAllR += allRec.size();
    }
    printf("\nUNIONCHAR %.0f %.0f %.4f %.4f %.4f %.4f %.4f\n", nIn / NQ12, nOut / NQ12, 100.0 * fI / pI, 100.0 * fO / pO,
           100.0 * fA / pA, nOut > 0 ? mOut / nOut : 0.0, nAllR > 0 ? mAll / nAllR : 0.0);
  }

  if (A.split) {  // shared vs exclusive members, src/axon.mm:1655-1692
    set_mult();
    double fS = 0, pS = 0, fE = 0, pE = 0, nS = 0, nE = 0;
    for (uint32_t q = 0; q < NQ12; ++q) {
      const auto w = within(refp[q], 0, nullptr, mult.data());
      fS += w[4]; pS += w[5]; fE += w[6]; pE += w[7]; nS += w[8]; nE += w[9];
    }
    std::vector<Cue> cs;
    std::vector<const uint32_t*> refs;
    for (uint32_t q = 0; q < NQ12; ++q) { cs.push_back({q, 1.0, 8800 + q}); refs.push_back(refp[q]); }
    const Readout r = readout(cs, 35, CLAMP, 0, false, false, &refs);
    std::vector<double> dS(35, 0), cS(35, 0), dE(35, 0), cE(35, 0);
    for (uint32_t q = 0; q < NQ12; ++q)
      for (uint32_t t = 0; t < 35u; ++t) {
        const uint32_t* dl = r.dlog_of(q) + t * 4;
        dS[t] += dl[0]; cS[t] += dl[1]; dE[t] += dl[2]; cE[t] += dl[3];
      }
    printf("\n===== SHARED vs EXCLUSIVE assembly members (NSTIM=%u) =====\n", NSTIM);
    printf("  shared fraction of assembly : %.3f  (%.0f shared / %.0f exclusive neurons)\n",
           (nS + nE) > 0 ? nS / (nS + nE) : 0.0, nS / NQ12, nE / NQ12);
    printf("  within-assembly density  SHARED    %.4f%%  (%.0f/%.0f)\n", 100.0 * fS / pS, fS, pS);
    printf("  within-assembly density  EXCLUSIVE %.4f%%  (%.0f/%.0f)\n", 100.0 * fE / pE, fE, pE);
    printf("  free-phase drive  SHARED   :");
    for (uint32_t t = CLAMP; t < 35u; ++t) printf(" %.0f", cS[t] ? dS[t] / cS[t] : 0.0);
    printf("\n  free-phase drive  EXCLUSIVE:");
    for (uint32_t t = CLAMP; t < 35u; ++t) printf(" %.0f", cE[t] ? dE[t] / cE[t] : 0.0);
    printf("\n==========================================================\n");
  }

  if (A.deep) {  // within-assembly scaffold and drive trace, src/axon.mm:1695-1730
    const uint32_t TT = std::min(T + 20u, 40u);
    double fIn = 0, pIn = 0, fOut = 0, pOut = 0;
    for (uint32_t q = 0; q < NQ12; ++q) {
      const auto w = within(refp[q], 0, nullptr, mult.data());
      fIn += w[0]; pIn += w[1]; fOut += w[2]; pOut += w[3];
    }
    std::vector<Cue> cs;
    std::vector<const uint32_t*> refs;
    for (uint32_t q = 0; q < NQ12; ++q) { cs.push_back({q, 1.0, 8600 + q}); refs.push_back(refp[q]); }
    const Readout r = readout(cs, TT, CLAMP, 0, false, false, &refs);
    std::vector<double> drvSum(40, 0), drvCnt(40, 0);
    for (uint32_t q = 0; q < NQ12; ++q)
      for (uint32_t t = 0; t < TT; ++t) {
        const uint32_t* dl = r.dlog_of(q) + t * 4;
        drvSum[t] += dl[0] + dl[2];
        drvCnt[t] += dl[1] + dl[3];
      }
    printf("\n========= WITHIN-ASSEMBLY RECURRENT SCAFFOLD (NSTIM=%u) =========\n", NSTIM);
    printf("  within-assembly : %.0f functional of %.0f possible = %.4f%%\n", fIn, pIn, 100.0 * fIn / pIn);
    printf("  between         : %.0f functional of %.0f possible = %.4f%%\n", fOut, pOut, 100.0 * fOut / pOut);
    printf("  enrichment within/between = %.2fx\n", (fOut > 0 && pIn > 0) ? (fIn / pIn) / (fOut / pOut) : 0.0);
    printf("  free-phase drive to assembly members, per step:\n   ");
    for (uint32_t t = 0; t < TT; ++t)
      if (t < CLAMP + 12) printf(" t%u:%.0f", t, drvCnt[t] ? drvSum[t] / drvCnt[t] : 0.0);
    printf("\n================================================================\n");
  }

  if (A.deep) {  // retrieved-population multiplicity and heavy tail, src/axon.mm:1733-1801
    std::vector<uint16_t> m(n, 0);
    for (uint32_t q = 0; q < NSTIM; ++q) for (uint32_t x : refN[q]) ++m[x];
    double popSum = 0;
    uint32_t popN = 0, maxMult = 0;
    for (uint32_t id = incols * kNpc; id < n; ++id)
      if (m[id]) { popSum += m[id]; ++popN; maxMult = std::max<uint32_t>(maxMult, m[id]); }
    const double popMean = popN ? popSum / popN : 0.0;
    const uint32_t NQ = std::min(NSTIM, 30u);
    std::vector<Cue> cs;
    for (uint32_t q = 0; q < NQ; ++q) cs.push_back({q, 1.0, 8100 + q});
    const Readout r = readout(cs, T, CLAMP, 0, false, false);
    double mIn = 0, mOut = 0, nIn = 0, nOut = 0, sumBest = 0, sumMean = 0, sumSelf = 0;
    for (uint32_t q = 0; q < NQ; ++q) {
      const Ids recn = active_neurons(r.final_of(q), incols, ncol);
      for (uint32_t x : common(recn, refN[q])) { mIn += m[x]; ++nIn; }
      for (uint32_t x : minus(recn, refN[q])) { mOut += m[x]; ++nOut; }
      const Ids rc2 = active_columns(r.final_of(q), incols, ncol);
      sumSelf += cos_overlap(rc2, refCols[q]);
      double best = 0, tot = 0;
      uint32_t cnt = 0;
      for (uint32_t o = 0; o < NSTIM; ++o)
        if (o != q) { const double x = cos_overlap(rc2, refCols[o]); best = std::max(best, x); tot += x; ++cnt; }
      sumBest += best;
      sumMean += cnt ? tot / cnt : 0.0;
    }
    printf("\n============ RETRIEVED-POPULATION MULTIPLICITY (NSTIM=%u) ============\n", NSTIM);
    printf("  population: %u neurons used, mean multiplicity %.2f, max %u\n", popN, popMean, maxMult);
    printf("  recalled AND in reference    : n=%.0f  mean multiplicity %.2f\n", nIn, nIn ? mIn / nIn : 0.0);
    printf("  recalled but NOT in reference: n=%.0f  mean multiplicity %.2f  (%.2fx population)\n", nOut,
           nOut ? mOut / nOut : 0.0, (nOut && popMean) ? (mOut / nOut) / popMean : 0.0);
    printf("  self %.3f | best-other %.3f | MEAN-over-others %.3f  -> %s\n", sumSelf / NQ, sumBest / NQ, sumMean / NQ,
           (sumMean / NQ > 0.5 * sumBest / NQ) ? "UNIFORM contamination" : "TAIL-dominated");
    std::vector<double> J, IO, IX;
    for (uint32_t i = 0; i < NSTIM; ++i)
      for (uint32_t j = i + 1; j < NSTIM; ++j) {
        const size_t in = n_common(refN[i], refN[j]), un = refN[i].size() + refN[j].size() - in;
        J.push_back(un ? (double)in / un : 0.0);
        Ids a = pats[i], b = pats[j];
        std::sort(a.begin(), a.end());
        std::sort(b.begin(), b.end());
        IO.push_back((double)n_common(a, b));
        IX.push_back((double)std::max(i, j));
      }
    auto pearson = [](const std::vector<double>& x, const std::vector<double>& y) {
      double mx = 0, my = 0;
      for (size_t i = 0; i < x.size(); ++i) { mx += x[i]; my += y[i]; }
      mx /= x.size();
      my /= y.size();
      double sxy = 0, sxx = 0, syy = 0;
      for (size_t i = 0; i < x.size(); ++i) {
        const double dx = x[i] - mx, dy = y[i] - my;
        sxy += dx * dy; sxx += dx * dx; syy += dy * dy;
      }
      return (sxx > 0 && syy > 0) ? sxy / std::sqrt(sxx * syy) : 0.0;
    };
    std::vector<double> Js = J;
    std::sort(Js.begin(), Js.end());
    printf("  heavy tail: %zu pairs | mean J %.5f | p99 %.5f | max %.5f\n", J.size(),
           std::accumulate(J.begin(), J.end(), 0.0) / J.size(), Js[(size_t)(0.99 * (Js.size() - 1))], Js.back());
    printf("  corr(assemblyJaccard, INPUT overlap)      r = %+.3f\n", pearson(J, IO));
    printf("  corr(assemblyJaccard, allocation index)   r = %+.3f\n", pearson(J, IX));
    printf("======================================================================\n");
  }

  if (A.wave) {  // long free-run wave, src/axon.mm:1804-1858
    const uint32_t TW = std::min(A.wavet, 60u);
    std::vector<Cue> cs;
    for (uint32_t q = 0; q < NQ12; ++q) cs.push_back({q, 1.0, 7000 + q});
    const Readout r = readout(cs, TW, CLAMP, 0, true, false);
    std::vector<double> ovR(TW, 0), nCol(TW, 0), nNeu(TW, 0), jPrev(TW, 0), fracA(TW, 0), jPrev2(TW, 0);
    double unionSz = 0, unionE = 0, unionO = 0, unionX = 0;
    for (uint32_t q = 0; q < NQ12; ++q) {
      const Ids& ref = refN[q];
      Ids prev, prev2, uni, uniE, uniO;
      for (uint32_t t = 0; t < TW; ++t) {
        const uint32_t* row = r.row(q, t);
        const Ids cur = active_neurons(row, incols, ncol);
        nCol[t] += active_columns(row, incols, ncol).size();
        nNeu[t] += cur.size();
        const size_t ii = n_common(cur, ref);
        ovR[t] += (cur.empty() || ref.empty()) ? 0.0 : (double)ii / std::sqrt((double)cur.size() * ref.size());
        fracA[t] += ref.empty() ? 0.0 : (double)ii / ref.size();
        if (t >= CLAMP) {
          uni.insert(uni.end(), cur.begin(), cur.end());
          Ids& half = (t % 2u == 0u) ? uniE : uniO;
          half.insert(half.end(), cur.begin(), cur.end());
        }
        jPrev[t] += t ? jaccard(cur, prev) : 0.0;
        jPrev2[t] += t > 1 ? jaccard(cur, prev2) : 0.0;
        prev2 = prev;
        prev = cur;
      }
      dedup(uni);
      dedup(uniE);
      dedup(uniO);
      unionSz += uni.size();
      unionE += uniE.size();
      unionO += uniO.size();
      unionX += (uniE.empty() || uniO.empty()) ? 0.0
                                               : (double)n_common(uniE, uniO) / std::sqrt((double)uniE.size() * uniO.size());
    }
    printf("\nPARITY %.0f %.4f %.0f %.4f %.0f %.4f %.4f\n", unionSz / NQ12, unionSz / NQ12 / 1536.0, unionE / NQ12,
           unionE / NQ12 / 1536.0, unionO / NQ12, unionO / NQ12 / 1536.0, unionX / NQ12);
    printf("\n================= WAVE: %u free steps after a %u-step cue =================\n", TW - CLAMP, CLAMP);
    printf("  step  phase   cols  neurons   ov(clampRef)  fracOfAssembly  J(t,t-1)   J(t,t-2)\n");
    for (uint32_t t = 0; t < TW; ++t)
      printf("  %4u  %-5s %6.0f %8.0f %13.3f %15.3f %10.3f %10.3f\n", t, t < CLAMP ? "cue" : "FREE", nCol[t] / NQ12,
             nNeu[t] / NQ12, ovR[t] / NQ12, fracA[t] / NQ12, jPrev[t] / NQ12, jPrev2[t] / NQ12);
    printf("==========================================================================\n");
  }

  {  // free-run diagnostic, src/axon.mm:1861-1887
    printf("\n============ FREE-RUN DIAGNOSTIC (cue %u steps, then released) ============\n", CLAMP);
    printf("  cue=75%%, averaged over %u stimuli.  'margin' = k-th minus (k+1)-th drive\n", NSTIM);
    printf("  step  phase  cols  drive_k  margin  %%marg=0   ov(CLAMPED ref)  ov(FREE ref)\n");
    std::vector<Cue> cs;
    for (uint32_t q = 0; q < NSTIM; ++q) cs.push_back({q, 0.75, 4000 + q});
    const Readout r = readout(cs, T, CLAMP, 0, true, true);
    std::vector<double> ovt(T, 0), ovf(T, 0), mg(T, 0), dk(T, 0), tie(T, 0), nc(T, 0);
    for (uint32_t q = 0; q < NSTIM; ++q)
      for (uint32_t t = 0; t < T; ++t) {
        const Ids a = active_columns(r.row(q, t), incols, ncol);
        ovt[t] += cos_overlap(a, refCols[q]);
        ovf[t] += cos_overlap(a, freeCols[q]);
        const uint32_t* sb = r.stats_of(q) + 64 + t * 8;
        const double cnt = sb[2];
        nc[t] += cnt;
        if (cnt > 0) { mg[t] += sb[0] / cnt; dk[t] += sb[1] / cnt; tie[t] += 100.0 * sb[3] / cnt; }
      }
    for (uint32_t t = 0; t < T; ++t)
      printf("  %4u  %-5s %5.0f %8.1f %7.1f %8.1f   %14.3f  %12.3f\n", t, t < CLAMP ? "cue" : "FREE", nc[t] / NSTIM,
             dk[t] / NSTIM, mg[t] / NSTIM, tie[t] / NSTIM, ovt[t] / NSTIM, ovf[t] / NSTIM);
    printf("==========================================================================\n");
  }

  // final completion table, src/axon.mm:1889-1908
  double m50 = 0;
  {
    const double keeps[] = {1.0, 0.75, 0.5, 0.35, 0.25};
    std::vector<Cue> cs;
    for (double k : keeps)
      for (uint32_t p = 0; p < NSTIM; ++p) cs.push_back({p, k, 3000 + p});
    const Readout r = readout(cs, T, CLAMP, 0, false, false);
    for (size_t ki = 0; ki < 5; ++ki) {
      double self = 0, other = 0, selfF = 0, otherF = 0;
      for (uint32_t p = 0; p < NSTIM; ++p) {
        const Ids a = active_columns(r.final_of((uint32_t)(ki * NSTIM + p)), incols, ncol);
        self += cos_overlap(a, refCols[p]);
        selfF += cos_overlap(a, freeCols[p]);
        double best = 0, bestF = 0;
        for (uint32_t q = 0; q < NSTIM; ++q)
          if (q != p) { best = std::max(best, cos_overlap(a, refCols[q])); bestF = std::max(bestF, cos_overlap(a, freeCols[q])); }
        other += best;
        otherF += bestF;
      }
      self /= NSTIM; other /= NSTIM; selfF /= NSTIM; otherF /= NSTIM;
      if (keeps[ki] == 0.5) m50 = self - other;
      if (!A.quiet)
        printf("  %3.0f%% |  %16.3f %6.3f %+7.3f  |  %11.3f %6.3f %+7.3f\n", keeps[ki] * 100, self, other, self - other,
               selfF, otherF, selfF - otherF);
    }
  }
  if (A.quiet)
    printf("tgt=%-4u k=%-3u inbr=%-3u stimc=%-4u bias=%-4u nand=%u | %7.4f ms %6.0f st/s asm=%-5.0f xtalk=%.3f margin50=%+.3f wd=%.2f\n",
           A.target, A.k, A.inbr, A.stimcols, A.biasup, A.nand, msStep, 1000.0 / msStep, sz, xtalk, m50, wstat());
  else
    printf("\n=== DONE ===\n");
  return 0;
}

}  // namespace

CliArgs CliArgs::parse(int argc, char** argv) {
  CliArgs a;
  auto g = [&](const char* k, uint32_t& v) { v = argv_u32(argc, argv, k, v); };
  g("nand", a.nand); g("target", a.target); g("k", a.k); g("dthr", a.dthr); g("boost", a.boost); g("mode", a.mode);
  g("epochs", a.epochs); g("T", a.T); g("clampsteps", a.clampsteps); g("stim", a.stim); g("quiet", a.quiet);
  g("seed", a.seed); g("split", a.split); g("unionchar", a.unionchar); g("biasup", a.biasup); g("biasdown", a.biasdown);
  g("biasshift", a.biasshift); g("biasdownevery", a.biasdownevery); g("inbr", a.inbr); g("stimcols", a.stimcols);
  g("incols", a.incols); g("ncol", a.ncol); g("diag", a.diag); g("profile", a.profile); g("topkpar", a.topkpar);
  g("vtopk", a.vtopk); g("contrast", a.contrast); g("bandlo", a.bandlo); g("bandhi", a.bandhi);
  g("margingate", a.margingate); g("hetero", a.hetero); g("vbs", a.vbs); g("ltdrep", a.ltdrep);
  g("ltdevery", a.ltdevery); g("ktest", a.ktest); g("facil", a.facil); g("deep", a.deep); g("wave", a.wave);
  g("wavet", a.wavet); g("cueflip", a.cueflip);
  a.trainclamp = argv_u32(argc, argv, "trainclamp", a.contrast ? a.clampsteps : a.T);
  uint32_t dev = argv_u32(argc, argv, "device", 0);
  a.device = (int)dev;
  if (a.biasup == 1u) {  // "auto" from the implied firing rate (src/axon.mm:732-735)
    const double pr = (double)a.target * a.k / (double)(a.ncol - a.incols) / kNpc;
    a.biasup = (uint32_t)std::max(2.0, (1.0 - pr) / pr * a.biasdown);
  }
  return a;
}

std::string CliArgs::check() const {
  if (T == 0 || T > 64) return "T must be in 1..64";
  if (stim == 0) return "stim must be >= 1";
  if (stimcols > incols) return "stimcols must be <= incols";
  if (trainclamp > 64) return "trainclamp must be <= 64";
  if (cueflip > 100) return "cueflip must be a percentage in 0..100";
  return "";
}

axon_cfg CliArgs::engine_cfg() const {
  axon_cfg c;
  axon_cfg_defaults(&c);
  c.ncol = ncol; c.incols = incols; c.inbr = inbr; c.nand = nand; c.target = target; c.k = k; c.ktest = ktest;
  c.dthr = dthr; c.boost = boost; c.mode = mode; c.biasup = biasup; c.biasdown = biasdown; c.biasshift = biasshift;
  c.biasdownevery = biasdownevery; c.bandlo = bandlo; c.bandhi = bandhi; c.contrast = contrast;
  c.margingate = margingate; c.hetero = hetero; c.ltdrep = ltdrep; c.ltdevery = ltdevery; c.facil = facil;
  c.topkpar = topkpar;
  return c;
}

int run_protocol(const CliArgs& a) {
  try {
    Session s(a);
    return s.run();
  } catch (const AxonFailure& e) {
    fflush(stdout);
    fprintf(stderr, "axon: %s\n", e.what());
    return 3;
  }
}

}  // namespace axon
