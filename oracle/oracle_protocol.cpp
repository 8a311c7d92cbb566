// AXON CPU oracle: main protocol and printed blocks. TEST INFRASTRUCTURE ONLY.
// Block-by-block restatement of rakib-nyc/axon src/axon.mm:737-1909 (cited per block).
#include "oracle_protocol.hpp"

#include <thread>

namespace oracle {

// vbs=1 bit-serial known-answer test, src/axon.mm:903-956
void Protocol::block_vbs() {
  printf("\n========== BIT-SERIAL VERIFICATION vs SCALAR REFERENCE ==========\n");
  const uint32_t NW = 1 << 14;
  const size_t nbits = (size_t)NW * 4 * 32;
  std::mt19937 r(424242);
  struct T { const char* n; uint32_t op, lo, hi; };
  const T tests[] = {{"bs_inc (carry, saturate 15)", 0, 0, 0}, {"bs_dec (BORROW, saturate 0)", 1, 0, 0},
                     {"bs_clip [5,11]", 2, 5, 11}, {"bs_clip [6,10]", 2, 6, 10}, {"bs_clip [4,12]", 2, 4, 12}};
  for (const auto& t : tests) {
    std::vector<uint8_t> vin(nbits), mk(nbits), vout(nbits);
    std::vector<uint32_t> p0(NW * 4, 0), p1(NW * 4, 0), p2(NW * 4, 0), p3(NW * 4, 0), pm(NW * 4, 0);
    for (size_t i = 0; i < nbits; ++i) {
      uint8_t v = r() & 15u, m = r() & 1u;
      vin[i] = v; mk[i] = m;
      size_t w = i >> 5, b = i & 31;
      if (v & 1) p0[w] |= 1u << b;
      if (v & 2) p1[w] |= 1u << b;
      if (v & 4) p2[w] |= 1u << b;
      if (v & 8) p3[w] |= 1u << b;
      if (m) pm[w] |= 1u << b;
    }
    for (size_t w = 0; w < (size_t)NW * 4; ++w) {
      if (t.op == 0) bs_inc(p0[w], p1[w], p2[w], p3[w], pm[w]);
      else if (t.op == 1) bs_dec(p0[w], p1[w], p2[w], p3[w], pm[w]);
      else bs_clip(p0[w], p1[w], p2[w], p3[w], t.lo, t.hi);
    }
    for (size_t i = 0; i < nbits; ++i) {
      size_t w = i >> 5, b = i & 31;
      vout[i] = ((p0[w] >> b) & 1) | (((p1[w] >> b) & 1) << 1) | (((p2[w] >> b) & 1) << 2) | (((p3[w] >> b) & 1) << 3);
    }
    size_t bad = 0, firstBad = (size_t)-1;
    for (size_t i = 0; i < nbits; ++i) {
      int exp;
      if (t.op == 0) exp = mk[i] ? std::min(15, (int)vin[i] + 1) : vin[i];
      else if (t.op == 1) exp = mk[i] ? std::max(0, (int)vin[i] - 1) : vin[i];
      else exp = std::min((int)t.hi, std::max((int)t.lo, (int)vin[i]));
      if (exp != (int)vout[i]) { if (bad == 0) firstBad = i; bad++; }
    }
    printf("  %-30s %9zu values  mismatches %zu  %s\n", t.n, nbits, bad, bad ? "FAIL" : "EXACT");
    if (bad) printf("      first at i=%zu in=%u mask=%u got=%u\n", firstBad, vin[firstBad], mk[firstBad], vout[firstBad]);
  }
  printf("================================================================\n");
}

// vtopk=1 serial-vs-parallel selection check, src/axon.mm:958-994
void Protocol::block_vtopk() {
  printf("\n=============== STEP B: parallel top-K verification ===============\n");
  printf("  serial TG=256 threads | parallel TG=%u threads (max %lu)\n", 1024u, 1024ul);
  std::vector<uint32_t> hs((size_t)C.T * C.NCOL), hp((size_t)C.T * C.NCOL);
  uint32_t mismatch = 0, thetaMismatch = 0;
  for (uint32_t q = 0; q < C.NSTIM; ++q) {
    E.topkPar = 0;
    present(q, 1.0, C.T, C.CLAMP, false, true, 9000 + q);
    std::copy(E.hist.begin(), E.hist.begin() + hs.size(), hs.begin());
    uint32_t thS = E.theta[0];
    E.topkPar = 1;
    present(q, 1.0, C.T, C.CLAMP, false, true, 9000 + q);
    std::copy(E.hist.begin(), E.hist.begin() + hp.size(), hp.begin());
    uint32_t thP = E.theta[0];
    for (size_t i = 0; i < hs.size(); ++i) if (hs[i] != hp[i]) mismatch++;
    if (thS != thP) thetaMismatch++;
  }
  printf("  winner-set words compared: %zu   MISMATCHES: %u  -> %s\n", (size_t)C.T * C.NCOL * C.NSTIM,
         mismatch, mismatch ? "FAIL" : "BIT-IDENTICAL");
  printf("  final theta compared: %u stimuli, mismatches %u\n", C.NSTIM, thetaMismatch);
  auto timeIt = [&](bool par) -> double {
    E.topkPar = par ? 1u : 0u;
    double best = 1e30;
    for (int rr = 0; rr < 5; ++rr) best = std::min(best, present(0, 1.0, C.T, C.CLAMP, false, true, 9999));
    return best;
  };
  double ts = timeIt(false), tp = timeIt(true);
  printf("  full step: serial %.1f us | parallel %.1f us | saved %.1f us (%.1f%% of step)\n", ts * 1000.0,
         tp * 1000.0, (ts - tp) * 1000.0, 100.0 * (ts - tp) / ts);
  E.topkPar = C.topkPar ? 1u : 0u;
  printf("==================================================================\n");
}

// diag=1 counter histogram, src/axon.mm:1107-1151
void Protocol::block_diag(const std::vector<std::vector<uint32_t>>& asmSpkHost) {
  const uint32_t n = N();
  std::vector<uint32_t> memb(n, 0u), asmv((size_t)C.NSTIM * C.NCOL);
  for (uint32_t q = 0; q < C.NSTIM; ++q) std::copy(asmSpkHost[q].begin(), asmSpkHost[q].end(), asmv.begin() + (size_t)q * C.NCOL);
  for (uint32_t c = C.IN_COLS; c < C.NCOL; ++c)
    for (uint32_t l = 0; l < NPC; ++l) {
      uint32_t m = 0;
      for (uint32_t q = 0; q < std::min(C.NSTIM, 32u); ++q) if ((asmSpkHost[q][c] >> l) & 1u) m |= (1u << q);
      memb[c * NPC + l] = m;
    }
  uint32_t nMember = 0;
  for (uint32_t i = 0; i < n; ++i) if (memb[i]) nMember++;
  const char* selName[2] = {"RECURRENT branches", "AFFERENT branches"};
  printf("\n======================= STEP 0 DIAGNOSTIC =======================\n");
  printf("4-bit synaptic counter distribution, %u stimuli, %u assembly-member neurons\n", C.NSTIM, nMember);
  for (uint32_t sel = 0; sel < 2; ++sel) {
    uint32_t h[48] = {0};
    E.k_wdiag(memb.data(), asmv.data(), C.NSTIM, C.inBranches, sel, h);
    const char* cat[3] = {"within-assembly", "between-assembly", "all"};
    printf("\n--- %s ---\n", selName[sel]);
    printf("  %-17s %10s  %6s %6s %6s | %s\n", "pair type", "count", "mean", "%at 0", "%at 15", "histogram v=0..15");
    for (uint32_t c = 0; c < 3; ++c) {
      double tot = 0, sum = 0;
      for (uint32_t v = 0; v < 16; ++v) { tot += h[c * 16 + v]; sum += (double)v * h[c * 16 + v]; }
      printf("  %-17s %10.0f  %6.2f %6.1f %6.1f | ", cat[c], tot, tot ? sum / tot : 0.0,
             tot ? 100.0 * h[c * 16 + 0] / tot : 0.0, tot ? 100.0 * h[c * 16 + 15] / tot : 0.0);
      for (uint32_t v = 0; v < 16; ++v) printf("%s%.1f", v ? "," : "", tot ? 100.0 * h[c * 16 + v] / tot : 0.0);
      printf("\n");
    }
  }
  printf("================================================================\n");
}

int Protocol::run() {
  const uint32_t NCOL = C.NCOL, IN_COLS = C.IN_COLS, NSTIM = C.NSTIM, T = C.T, CLAMP = C.CLAMP;
  const uint32_t Nn = N();
  const uint32_t NGRP = NCOL / COLS_PER_GRP;
  const double PLANE_B = (double)NCOL * NSLOT * SLOT_U4 * 32 * 16;
  if (!C.quiet) {  // banner, src/axon.mm:737-747
    printf("======================================================================\n");
    printf(" AXON v0  -  columnar assembly engine, CPU oracle\n");
    printf("======================================================================\n");
    printf("  neurons %u (%u cols x %u) | branches %u x %u presyn | fan-in %u | %.2f G syn\n", Nn, NCOL, NPC,
           NSLOT, PRESYN, FANIN, (double)Nn * FANIN / 1e9);
    printf("  weights 4 planes x %.0f MB = %.0f MB | groups %u\n", PLANE_B / 1048576.0, 4 * PLANE_B / 1048576.0, NGRP);
    printf("  nand=%u target=%u k=%u dthr=%u mode=%u epochs=%u T=%u clamp=%u stim=%u biasUp=%u inbr=%u stimcols=%u\n\n",
           C.nAnd, C.targetC, C.K, C.dthr, C.mode, C.EPOCHS, T, CLAMP, NSTIM, C.biasUp, C.inBranches, C.STIM_COLS);
  }
  E.init(C.nAnd, C.seed, C.inBranches);  // src/axon.mm:770-782
  std::fill(E.theta.begin(), E.theta.end(), 0u);
  std::fill(E.stats.begin(), E.stats.end(), 0u);
  make_stimuli();

  if (C.vbs) block_vbs();
  if (C.vtopk) block_vtopk();

  double d0 = wstat();  // src/axon.mm:996-998
  if (!C.quiet) printf("initial functional synapse density: %.3f%%  (fan-in %.0f functional)\n\n", d0, d0 / 100.0 * FANIN);

  for (uint32_t i = 0; i < 10; ++i) present(i % NSTIM, 1.0, T, T, false, false, 999);  // settle, :1001
  if (!C.quiet)
    printf("settled: theta=%u  activeCols/step=%.0f  activeNeurons/step=%.0f\n\n", E.theta[0],
           (double)E.stats[0] / T, (double)E.stats[1] / T);

  // training, src/axon.mm:1008-1026
  double msAcc = 0; int msN = 0;
  auto tr0 = std::chrono::steady_clock::now();
  for (uint32_t ep = 0; ep < C.EPOCHS; ++ep) {
    for (uint32_t p = 0; p < NSTIM; ++p) { msAcc += present(p, 1.0, T, C.trainClamp, true, false, 1000 + p); msN++; }
    if (!C.quiet && (ep % 5 == 4 || ep == 0)) {
      double ltp = E.stats[8], ltd = E.stats[9];
      uint32_t tp = E.stats[10], td = E.stats[11];
      double wd = wstat();
      printf("  ep %3u  wdens %7.3f%%  LTP %10.0f  LTD %10.0f  LTD/LTP %6.3f  learners %u/%u\n", ep + 1, wd, ltp,
             ltd, ltp > 0 ? ltd / ltp : 0.0, tp, td);
    }
  }
  trainSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - tr0).count();
  if (msN == 0) { msAcc = present(0, 1.0, T, T, false, true, 777); msN = 1; }
  double msStep = msAcc / msN;

  // firing steps per neuron under training conditions, src/axon.mm:1032-1072
  {
    present(0, 1.0, T, C.trainClamp, true, false, 31337);
    const uint32_t* H = E.hist.data();
    std::vector<uint16_t> cnt(Nn, 0), cntC(Nn, 0), cntF(Nn, 0);
    for (uint32_t t = 0; t < T; ++t)
      for (uint32_t c = IN_COLS; c < NCOL; ++c) {
        uint32_t b = H[(size_t)t * NCOL + c];
        while (b) {
          uint32_t l = (uint32_t)__builtin_ctz(b); b &= b - 1;
          cnt[c * NPC + l]++;
          if (t < C.trainClamp) cntC[c * NPC + l]++; else cntF[c * NPC + l]++;
        }
      }
    const uint32_t* Hlast = H + (size_t)(T - 1) * NCOL;
    std::vector<uint8_t> isMember(Nn, 0);
    uint32_t nMem = 0;
    for (uint32_t c = IN_COLS; c < NCOL; ++c) {
      uint32_t b = Hlast[c];
      while (b) { uint32_t l = (uint32_t)__builtin_ctz(b); b &= b - 1; isMember[c * NPC + l] = 1; nMem++; }
    }
    (void)nMem;
    double n = 0, sum = 0, sumC = 0, sumF = 0, nm = 0, sm = 0, smC = 0, smF = 0;
    std::vector<uint16_t> v, vm;
    for (uint32_t i = IN_COLS * NPC; i < Nn; ++i) {
      if (cnt[i]) { n++; sum += cnt[i]; sumC += cntC[i]; sumF += cntF[i]; v.push_back(cnt[i]); }
      if (isMember[i]) { nm++; sm += cnt[i]; smC += cntC[i]; smF += cntF[i]; vm.push_back(cnt[i]); }
    }
    std::sort(v.begin(), v.end()); std::sort(vm.begin(), vm.end());
    printf("\n================= FIRING STEPS PER NEURON (training) =================\n");
    printf("  T=%u  trainClamp=%u (clamped) + %u (free)\n", T, C.trainClamp, T - C.trainClamp);
    printf("  neurons firing at least once: %.0f\n", n);
    printf("  mean firing steps  : %.2f   (clamped %.2f + free %.2f)\n", n ? sum / n : 0.0, n ? sumC / n : 0.0,
           n ? sumF / n : 0.0);
    if (!v.empty())
      printf("  p50 %u | p90 %u | max %u   | as fraction of T: %.3f\n", v[v.size() / 2],
             v[(size_t)(0.9 * (v.size() - 1))], v.back(), n ? sum / n / T : 0.0);
    printf("  --- restricted to FINAL-STATE ASSEMBLY MEMBERS (the allocated ones) ---\n");
    printf("  members: %.0f | mean firing steps %.2f (clamped %.2f + free %.2f) | fraction of T %.3f\n", nm,
           nm ? sm / nm : 0.0, nm ? smC / nm : 0.0, nm ? smF / nm : 0.0, nm ? sm / nm / T : 0.0);
    if (!vm.empty())
      printf("  p50 %u | p90 %u | max %u\n", vm[vm.size() / 2], vm[(size_t)(0.9 * (vm.size() - 1))], vm.back());
    printf("  => bias gain per presentation = biasUp * spikes(members) = %.0f\n", nm ? C.biasUp * sm / nm : 0.0);
    printf("======================================================================\n");
  }

  // reference assemblies, src/axon.mm:1080-1105
  std::vector<Cols> refClampCols(NSTIM), refFreeCols(NSTIM);
  std::vector<std::vector<uint32_t>> refClampBal(NSTIM), refFreeBal(NSTIM);
  std::vector<std::vector<uint32_t>> asmSpkHost(NSTIM, std::vector<uint32_t>(NCOL, 0));
  for (uint32_t p = 0; p < NSTIM; ++p) {
    present(p, 1.0, T, T, false, true, 2000 + p);
    refClampCols[p] = assemblyOf(T);
    refClampBal[p].assign(final_spk(T), final_spk(T) + NCOL);
    asmSpkHost[p] = refClampBal[p];
    for (uint32_t c = 0; c < IN_COLS; ++c) asmSpkHost[p][c] = 0u;
    present(p, 1.0, T, CLAMP, false, true, 2100 + p);
    refFreeCols[p] = assemblyOf(T);
    refFreeBal[p].assign(final_spk(T), final_spk(T) + NCOL);
  }
  double sz = 0;
  for (auto& a : refClampCols) sz += a.size();
  sz /= NSTIM;
  double xtalk = 0, xtalkF = 0; int xn = 0;
  for (uint32_t i = 0; i < NSTIM; ++i)
    for (uint32_t j = i + 1; j < NSTIM; ++j) {
      xtalk += overlap(refClampCols[i], refClampCols[j]);
      xtalkF += overlap(refFreeCols[i], refFreeCols[j]);
      xn++;
    }
  xtalk = xn ? xtalk / xn : 0; xtalkF = xn ? xtalkF / xn : 0;

  if (C.diag) block_diag(asmSpkHost);

  if (!C.quiet) {  // src/axon.mm:1153-1160
    printf("\n  %.4f ms/timestep -> %.0f steps/s (%.1fx biological real time), wdens %.3f%%\n", msStep,
           1000.0 / msStep, 1.0 / msStep, wstat());
    printf("  assembly size %.1f cols (%.2f%% of area) | cross-talk CLAMPED %.3f  FREE %.3f  (chance %.3f)\n\n", sz,
           100.0 * sz / (NCOL - IN_COLS), xtalk, xtalkF, sz / (NCOL - IN_COLS));
    printf("--- pattern completion: cue %u steps, RELEASED %u.  BOTH reference definitions ---\n", CLAMP, T - CLAMP);
    printf("  cue  |  CLAMPED ref: self  other  margin  |  FREE ref: self  other  margin\n");
  }
  if (C.profile) printf("\n[profile] GPU timestamps unavailable on this device\n");

  // STEP A1, src/axon.mm:1343-1409
  {
    std::vector<uint32_t> ind(Nn, 0u);
    E.k_indeg(C.inBranches, ind.data());
    std::vector<uint32_t> v;
    v.reserve(Nn);
    for (uint32_t c = IN_COLS; c < NCOL; ++c) for (uint32_t l = 0; l < NPC; ++l) v.push_back(ind[c * NPC + l]);
    std::vector<uint32_t> sv = v;
    std::sort(sv.begin(), sv.end());
    auto pct = [&](double q) { return sv[(size_t)(q * (sv.size() - 1))]; };
    double mean = 0;
    for (uint32_t x : v) mean += x;
    mean /= v.size();
    double sd = 0;
    for (uint32_t x : v) sd += (x - mean) * (x - mean);
    sd = std::sqrt(sd / v.size());
    printf("\n=============================== STEP A1 ===============================\n");
    printf("Functional in-degree over the %u RECURRENT branches (popcount of MSB plane)\n", NSLOT - C.inBranches);
    printf("  n=%zu neurons   mean %.1f   sd %.1f   cv %.3f\n", v.size(), mean, sd, sd / mean);
    printf("  min %u | p10 %u | p25 %u | p50 %u | p75 %u | p90 %u | p99 %u | p99.9 %u | max %u\n", sv.front(),
           pct(0.10), pct(0.25), pct(0.50), pct(0.75), pct(0.90), pct(0.99), pct(0.999), sv.back());
    printf("  tail ratio p99/p50 = %.2f   max/p50 = %.2f\n", (double)pct(0.99) / pct(0.50),
           (double)sv.back() / pct(0.50));
    for (int which = 0; which < 2; ++which) {
      const auto& src = which ? refClampBal : refFreeBal;
      std::vector<Cols> ns(NSTIM);
      for (uint32_t q = 0; q < NSTIM; ++q) ns[q] = neuronSet(src[q].data());
      double jm = 0; int jn = 0; double jmax = 0;
      for (uint32_t i = 0; i < NSTIM; ++i)
        for (uint32_t j = i + 1; j < NSTIM; ++j) { double x = jaccard(ns[i], ns[j]); jm += x; jn++; jmax = std::max(jmax, x); }
      std::vector<uint32_t> cnt(Nn, 0);
      for (auto& a : ns) for (uint32_t x : a) cnt[x]++;
      const uint32_t* bias = E.bias.data();
      uint32_t nAll = 0, nNone = 0, nAny = 0;
      double dAll = 0, dNone = 0, dAny = 0, bAll = 0, bNone = 0, bAny = 0;
      for (uint32_t c = IN_COLS; c < NCOL; ++c)
        for (uint32_t l = 0; l < NPC; ++l) {
          uint32_t id = c * NPC + l;
          if (cnt[id] >= NSTIM - 1) { nAll++; dAll += ind[id]; bAll += bias[id]; }
          if (cnt[id] == 0) { nNone++; dNone += ind[id]; bNone += bias[id]; }
          if (cnt[id] > 0) { nAny++; dAny += ind[id]; bAny += bias[id]; }
        }
      printf("\n  --- winner identity, %s endpoint ---\n", which ? "CLAMPED" : "FREE-RUN");
      printf("    mean pairwise Jaccard %.3f (max %.3f) over %d pairs, mean set size %.0f\n", jm / jn, jmax, jn,
             (double)ns[0].size());
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
    const double npool = (double)(NCOL - IN_COLS) * NPC;
    std::vector<Cols> cns(NSTIM);
    for (uint32_t q = 0; q < NSTIM; ++q) cns[q] = neuronSet(refClampBal[q].data());
    double msz = 0;
    for (auto& a : cns) msz += a.size();
    msz /= NSTIM;
    double eInt = msz * msz / npool;
    double eJac = eInt / (2.0 * msz - eInt);
    double jm = 0, jmax = 0; int jn = 0; double totInt = 0;
    for (uint32_t i = 0; i < NSTIM; ++i)
      for (uint32_t j = i + 1; j < NSTIM; ++j) {
        double x = jaccard(cns[i], cns[j]);
        jm += x; jn++; jmax = std::max(jmax, x);
        Cols ii;
        std::set_intersection(cns[i].begin(), cns[i].end(), cns[j].begin(), cns[j].end(), std::back_inserter(ii));
        totInt += ii.size();
      }
    Cols uni;
    for (auto& a : cns) uni.insert(uni.end(), a.begin(), a.end());
    std::sort(uni.begin(), uni.end());
    size_t uniqN = std::unique(uni.begin(), uni.end()) - uni.begin();
    double sumSz = msz * NSTIM;
    printf("\n=============================== STEP A3 ===============================\n");
    printf("Chance baseline for %u assemblies of %.0f neurons from a pool of %.0f\n", NSTIM, msz, npool);
    printf("  E[|A n B|] = m^2/n            = %.2f neurons\n", eInt);
    printf("  E[Jaccard] = E/(2m-E)         = %.5f      <-- CHANCE\n", eJac);
    printf("  measured mean pairwise Jaccard = %.5f   (max %.5f)\n", jm / jn, jmax);
    printf("  ratio measured/chance          = %.3f\n", eJac > 0 ? (jm / jn) / eJac : 0.0);
    printf("  total pairwise overlap: measured %.0f neurons vs %.0f expected at chance (%.1fx less)\n", totInt,
           eInt * jn, totInt > 0 ? eInt * jn / totInt : 1e9);
    printf("  sum of assembly sizes %.0f | union %zu | excess %.0f  -> %s\n", sumSz, uniqN, sumSz - (double)uniqN,
           (sumSz - (double)uniqN) < 0.02 * sumSz ? "NEAR-EXACT PARTITION" : "overlapping");

    std::vector<Cols> refNBCols(NSTIM);
    for (uint32_t q = 0; q < NSTIM; ++q) {
      present(q, 1.0, T, T, false, true, 2200 + q, 0u);
      refNBCols[q] = assemblyOf(T);
    }
    double preserve = 0;
    for (uint32_t q = 0; q < NSTIM; ++q) preserve += overlap(refNBCols[q], refClampCols[q]);
    preserve /= NSTIM;
    double xNB = 0; int xn2 = 0;
    for (uint32_t i = 0; i < NSTIM; ++i)
      for (uint32_t j = i + 1; j < NSTIM; ++j) { xNB += overlap(refNBCols[i], refNBCols[j]); xn2++; }
    xNB /= xn2;
    printf("\n=============================== STEP A4 ===============================\n");
    printf("Zero the intrinsic bias at TEST time only. Trained weights unchanged.\n");
    printf("  clamped assembly preserved when bias is zeroed: overlap %.3f\n", preserve);
    printf("  cross-talk of clamped assemblies, bias OFF     : %.3f  (bias ON: %.3f)\n", xNB, xtalk);

    printf("\n  release trajectory, cue 75%%, bias OFF at test (vs bias ON baseline)\n");
    printf("  step  phase   ov(clampRef,biasON)  ov(clampRef,biasOFF)  ov(noBiasRef,biasOFF)\n");
    std::vector<double> a1(T, 0), a2(T, 0), a3(T, 0);
    for (uint32_t q = 0; q < NSTIM; ++q) {
      present(q, 0.75, T, CLAMP, false, true, 4300 + q, 1u);
      for (uint32_t t = 0; t < T; ++t) a1[t] += overlap(colsOf(E.hist.data() + (size_t)t * NCOL), refClampCols[q]);
      present(q, 0.75, T, CLAMP, false, true, 4300 + q, 0u);
      for (uint32_t t = 0; t < T; ++t) {
        Cols a = colsOf(E.hist.data() + (size_t)t * NCOL);
        a2[t] += overlap(a, refClampCols[q]);
        a3[t] += overlap(a, refNBCols[q]);
      }
    }
    for (uint32_t t = 0; t < T; ++t)
      printf("  %4u  %-5s %19.3f %21.3f %22.3f\n", t, t < CLAMP ? "cue" : "FREE", a1[t] / NSTIM, a2[t] / NSTIM,
             a3[t] / NSTIM);

    printf("\n  pattern completion with bias OFF at test  (keep=0 is the no-cue control)\n");
    printf("  cue  |  vs CLAMPED ref(biasON): self  other  margin | vs noBias ref: self  other  margin\n");
    // cueflip=P adds an 11th row (no counterpart in the reference): keep = -P/100 marks the
    // whole pattern with P% of its active bits flipped off (noisy_clamp, draw 0)
    std::vector<double> rows = {1.0, 0.75, 0.5, 0.35, 0.25, 0.15, 0.10, 0.05, 0.02, 0.0};
    if (C.cueflip) rows.push_back(-(double)C.cueflip / 100.0);
    for (double keep : rows) {
      double s1 = 0, o1 = 0, s2 = 0, o2 = 0;
      for (uint32_t q = 0; q < NSTIM; ++q) {
        if (keep < 0) present_noisy(q, -keep, T, CLAMP, noisy_seed(q, C.cueflip, 0));
        else present(q, keep, T, CLAMP, false, true, 4400 + q, 0u);
        Cols a = assemblyOf(T);
        s1 += overlap(a, refClampCols[q]);
        s2 += overlap(a, refNBCols[q]);
        double b1 = 0, b2 = 0;
        for (uint32_t r = 0; r < NSTIM; ++r)
          if (r != q) { b1 = std::max(b1, overlap(a, refClampCols[r])); b2 = std::max(b2, overlap(a, refNBCols[r])); }
        o1 += b1; o2 += b2;
      }
      if (keep >= 0)
        printf("  %3.0f%% |%25.3f %6.3f %+7.3f |%18.3f %6.3f %+7.3f\n", keep * 100, s1 / NSTIM, o1 / NSTIM,
               s1 / NSTIM - o1 / NSTIM, s2 / NSTIM, o2 / NSTIM, s2 / NSTIM - o2 / NSTIM);
      else
        printf("  flip%3u%% |%21.3f %6.3f %+7.3f |%18.3f %6.3f %+7.3f\n", C.cueflip, s1 / NSTIM, o1 / NSTIM,
               s1 / NSTIM - o1 / NSTIM, s2 / NSTIM, o2 / NSTIM, s2 / NSTIM - o2 / NSTIM);
    }
    printf("======================================================================\n");
  }

  // A4b + A4c, src/axon.mm:1514-1599
  {
    std::vector<uint32_t> ind(Nn, 0u), unt(Nn, 0u);
    E.k_indeg(C.inBranches, ind.data());
    E.k_untouched(C.inBranches, unt.data());
    const double RECSYN = (double)(NSLOT - C.inBranches) * PRESYN;
    const double cues[4] = {1.0, 0.75, 0.35, 0.15};
    printf("\n=============================== A4b ===============================\n");
    printf("Is the recalled ~25%% a FIXED subset? (readout gate on: bias off at test)\n");
    std::vector<std::vector<Cols>> rec(NSTIM, std::vector<Cols>(4));
    for (uint32_t q = 0; q < NSTIM; ++q)
      for (int ci = 0; ci < 4; ++ci) {
        present(q, cues[ci], T, CLAMP, false, true, 5000 + q * 16 + ci);
        rec[q][ci] = neuronSet(final_spk(T));
      }
    printf("  pairwise Jaccard of recalled sets ACROSS cue levels, same stimulus:\n    ");
    double jall = 0; int jn = 0;
    for (int a = 0; a < 4; ++a)
      for (int b = a + 1; b < 4; ++b) {
        double m = 0;
        for (uint32_t q = 0; q < NSTIM; ++q) m += jaccard(rec[q][a], rec[q][b]);
        m /= NSTIM;
        printf("%.0f%%/%.0f%%=%.3f  ", cues[a] * 100, cues[b] * 100, m);
        jall += m; jn++;
      }
    printf("\n    mean across cue pairs = %.3f\n", jall / jn);
    double coreSz = 0, periSz = 0, asmSz = 0, dCore = 0, dPeri = 0, uCore = 0, uPeri = 0;
    size_t nCore = 0, nPeri = 0;
    for (uint32_t q = 0; q < NSTIM; ++q) {
      Cols core = rec[q][0];
      for (int ci = 1; ci < 4; ++ci) {
        Cols t;
        std::set_intersection(core.begin(), core.end(), rec[q][ci].begin(), rec[q][ci].end(), std::back_inserter(t));
        core = t;
      }
      Cols A = neuronSet(refClampBal[q].data());
      Cols coreInA, peri;
      std::set_intersection(core.begin(), core.end(), A.begin(), A.end(), std::back_inserter(coreInA));
      std::set_difference(A.begin(), A.end(), core.begin(), core.end(), std::back_inserter(peri));
      coreSz += coreInA.size(); periSz += peri.size(); asmSz += A.size();
      for (uint32_t x : coreInA) { dCore += ind[x]; uCore += 100.0 * unt[x] / RECSYN; nCore++; }
      for (uint32_t x : peri) { dPeri += ind[x]; uPeri += 100.0 * unt[x] / RECSYN; nPeri++; }
    }
    printf("\n  assembly %.0f neurons | CORE (recalled at all 4 cues) %.0f (%.1f%%) | periphery %.0f\n",
           asmSz / NSTIM, coreSz / NSTIM, 100.0 * coreSz / asmSz, periSz / NSTIM);
    printf("  %-12s %10s %14s %22s\n", "group", "n", "in-degree", "%% synapses still at 5/6");
    printf("  %-12s %10zu %14.1f %22.1f\n", "CORE", nCore, nCore ? dCore / nCore : 0.0, nCore ? uCore / nCore : 0.0);
    printf("  %-12s %10zu %14.1f %22.1f\n", "periphery", nPeri, nPeri ? dPeri / nPeri : 0.0, nPeri ? uPeri / nPeri : 0.0);
    double allD = 0, allU = 0; size_t nAll = 0;
    for (uint32_t c = IN_COLS; c < NCOL; ++c)
      for (uint32_t l = 0; l < NPC; ++l) { allD += ind[c * NPC + l]; allU += 100.0 * unt[c * NPC + l] / RECSYN; nAll++; }
    printf("  %-12s %10zu %14.1f %22.1f\n", "all neurons", nAll, allD / nAll, allU / nAll);

    std::vector<uint32_t> bv;
    bv.reserve(Nn);
    for (uint32_t c = IN_COLS; c < NCOL; ++c) for (uint32_t l = 0; l < NPC; ++l) bv.push_back(E.bias[c * NPC + l]);
    std::sort(bv.begin(), bv.end());
    double bm = 0;
    for (uint32_t x : bv) bm += x;
    bm /= bv.size();
    printf("\n=============================== A4c ===============================\n");
    printf("Intrinsic bias growth after %u epochs (unbounded, non-leaky, learning-time only)\n", C.EPOCHS);
    printf("  mean %.0f | p50 %u | p99 %u | max %u | UINT32_MAX %u | headroom %.3g x\n", bm, bv[bv.size() / 2],
           bv[(size_t)(0.99 * (bv.size() - 1))], bv.back(), 4294967295u, bv.back() ? 4294967295.0 / bv.back() : 0.0);
    printf("  growth rate ~= %.1f per epoch (max/epochs) -> epochs to saturate ~ %.3g\n",
           C.EPOCHS ? (double)bv.back() / C.EPOCHS : 0.0,
           (bv.back() && C.EPOCHS) ? 4294967295.0 / ((double)bv.back() / C.EPOCHS) : 0.0);
    printf("==================================================================\n");
  }

  // visited-union characterisation, src/axon.mm:1602-1652
  if (C.unionchar) {
    std::fill(E.mult.begin(), E.mult.end(), 0u);
    for (uint32_t q = 0; q < NSTIM; ++q)
      for (uint32_t c = IN_COLS; c < NCOL; ++c) {
        uint32_t b = refClampBal[q][c];
        while (b) { uint32_t l = (uint32_t)__builtin_ctz(b); b &= b - 1; E.mult[c * NPC + l]++; }
      }
    uint32_t NQ = std::min(NSTIM, 12u);
    double nIn = 0, nOut = 0, fI = 0, pI = 0, fO = 0, pO = 0, fA = 0, pA = 0, mOut = 0, mAll = 0, nAllR = 0;
    std::vector<uint32_t> post(Nn, 0u);
    auto runW = [&](const Cols& ps, double& f, double& pp) {
      std::fill(post.begin(), post.end(), 0u);
      for (uint32_t x : ps) post[x] = 1u;
      uint32_t w[10] = {0};
      E.k_within(E.refBall.data(), C.inBranches, IN_COLS, 1u, post.data(), E.mult.data(), w);
      f += w[0]; pp += w[1];
    };
    Cols allRec;
    for (uint32_t c = IN_COLS; c < NCOL; ++c) for (uint32_t l = 0; l < NPC; ++l) allRec.push_back(c * NPC + l);
    for (uint32_t q = 0; q < NQ; ++q) {
      E.refBall = refClampBal[q];
      present(q, 1.0, 35u, CLAMP, false, true, 9500 + q);
      Cols uni;
      for (uint32_t t = CLAMP; t < 35u; ++t)
        for (uint32_t c = IN_COLS; c < NCOL; ++c) {
          uint32_t b = E.hist[(size_t)t * NCOL + c];
          while (b) { uint32_t l = (uint32_t)__builtin_ctz(b); b &= b - 1; uni.push_back(c * NPC + l); }
        }
      std::sort(uni.begin(), uni.end());
      uni.erase(std::unique(uni.begin(), uni.end()), uni.end());
      Cols ref = neuronSet(refClampBal[q].data());
      Cols in_, out_;
      std::set_intersection(uni.begin(), uni.end(), ref.begin(), ref.end(), std::back_inserter(in_));
      std::set_difference(uni.begin(), uni.end(), ref.begin(), ref.end(), std::back_inserter(out_));
      nIn += in_.size(); nOut += out_.size();
      runW(in_, fI, pI); runW(out_, fO, pO); runW(allRec, fA, pA);
      for (uint32_t x : out_) mOut += E.mult[x];
      for (uint32_t x : allRec) mAll += E.mult[x];
      nAllR += allRec.size();
    }
    printf("\nUNIONCHAR %.0f %.0f %.4f %.4f %.4f %.4f %.4f\n", nIn / NQ, nOut / NQ, 100.0 * fI / pI, 100.0 * fO / pO,
           100.0 * fA / pA, nOut > 0 ? mOut / nOut : 0.0, nAllR > 0 ? mAll / nAllR : 0.0);
  }

  // shared vs exclusive members, src/axon.mm:1655-1692
  if (C.split) {
    std::fill(E.mult.begin(), E.mult.end(), 0u);
    for (uint32_t q = 0; q < NSTIM; ++q)
      for (uint32_t c = IN_COLS; c < NCOL; ++c) {
        uint32_t b = refClampBal[q][c];
        while (b) { uint32_t l = (uint32_t)__builtin_ctz(b); b &= b - 1; E.mult[c * NPC + l]++; }
      }
    uint32_t NQ = std::min(NSTIM, 12u);
    double fS = 0, pS = 0, fE = 0, pE = 0, nS = 0, nE = 0;
    std::vector<double> dS(64, 0), cS(64, 0), dE(64, 0), cE(64, 0);
    for (uint32_t q = 0; q < NQ; ++q) {
      E.refBall = refClampBal[q];
      uint32_t w[10] = {0};
      E.k_within(E.refBall.data(), C.inBranches, IN_COLS, 0u, E.mult.data(), E.mult.data(), w);
      fS += w[4]; pS += w[5]; fE += w[6]; pE += w[7]; nS += w[8]; nE += w[9];
      std::fill(E.driveLog.begin(), E.driveLog.end(), 0u);
      present(q, 1.0, 35u, CLAMP, false, true, 8800 + q);
      for (uint32_t t = 0; t < 35u; ++t) {
        dS[t] += E.driveLog[t * 4 + 0]; cS[t] += E.driveLog[t * 4 + 1];
        dE[t] += E.driveLog[t * 4 + 2]; cE[t] += E.driveLog[t * 4 + 3];
      }
    }
    printf("\n===== SHARED vs EXCLUSIVE assembly members (NSTIM=%u) =====\n", NSTIM);
    printf("  shared fraction of assembly : %.3f  (%.0f shared / %.0f exclusive neurons)\n",
           (nS + nE) > 0 ? nS / (nS + nE) : 0.0, nS / NQ, nE / NQ);
    printf("  within-assembly density  SHARED    %.4f%%  (%.0f/%.0f)\n", 100.0 * fS / pS, fS, pS);
    printf("  within-assembly density  EXCLUSIVE %.4f%%  (%.0f/%.0f)\n", 100.0 * fE / pE, fE, pE);
    printf("  free-phase drive  SHARED   :");
    for (uint32_t t = CLAMP; t < 35u; ++t) printf(" %.0f", cS[t] ? dS[t] / cS[t] : 0.0);
    printf("\n  free-phase drive  EXCLUSIVE:");
    for (uint32_t t = CLAMP; t < 35u; ++t) printf(" %.0f", cE[t] ? dE[t] / cE[t] : 0.0);
    printf("\n==========================================================\n");
  }

  // within-assembly scaffold and drive trace, src/axon.mm:1695-1730
  if (C.deep) {
    uint32_t NQ = std::min(NSTIM, 12u);
    double fIn = 0, pIn = 0, fOut = 0, pOut = 0;
    std::vector<double> drvSum(40, 0), drvCnt(40, 0);
    const uint32_t TT = std::min(T + 20u, 40u);
    for (uint32_t q = 0; q < NQ; ++q) {
      E.refBall = refClampBal[q];
      uint32_t w[10] = {0};
      // the reference leaves buffers 6-8 unbound here; only out[0..3] are read
      E.k_within(E.refBall.data(), C.inBranches, IN_COLS, 0u, E.mult.data(), E.mult.data(), w);
      fIn += w[0]; pIn += w[1]; fOut += w[2]; pOut += w[3];
      std::fill(E.driveLog.begin(), E.driveLog.end(), 0u);
      present(q, 1.0, TT, CLAMP, false, true, 8600 + q);
      for (uint32_t t = 0; t < TT; ++t) {
        drvSum[t] += E.driveLog[t * 4 + 0] + E.driveLog[t * 4 + 2];
        drvCnt[t] += E.driveLog[t * 4 + 1] + E.driveLog[t * 4 + 3];
      }
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

  // retrieved-population multiplicity and heavy tail, src/axon.mm:1733-1801
  if (C.deep) {
    std::vector<uint16_t> mult(Nn, 0);
    for (uint32_t q = 0; q < NSTIM; ++q) for (uint32_t x : neuronSet(refClampBal[q].data())) mult[x]++;
    double popSum = 0; uint32_t popN = 0, maxMult = 0;
    for (uint32_t i = IN_COLS * NPC; i < Nn; ++i)
      if (mult[i]) { popSum += mult[i]; popN++; maxMult = std::max<uint32_t>(maxMult, mult[i]); }
    double popMean = popN ? popSum / popN : 0.0;
    uint32_t NQ = std::min(NSTIM, 30u);
    double mIn = 0, mOut = 0, nIn = 0, nOut = 0, sumBest = 0, sumMeanOther = 0, sumSelf = 0;
    for (uint32_t q = 0; q < NQ; ++q) {
      present(q, 1.0, T, CLAMP, false, true, 8100 + q);
      const uint32_t* sp = final_spk(T);
      Cols recn = neuronSet(sp), refN = neuronSet(refClampBal[q].data());
      Cols in_, out_;
      std::set_intersection(recn.begin(), recn.end(), refN.begin(), refN.end(), std::back_inserter(in_));
      std::set_difference(recn.begin(), recn.end(), refN.begin(), refN.end(), std::back_inserter(out_));
      for (uint32_t x : in_) { mIn += mult[x]; nIn++; }
      for (uint32_t x : out_) { mOut += mult[x]; nOut++; }
      Cols recCols = colsOf(sp);
      sumSelf += overlap(recCols, refClampCols[q]);
      double best = 0, tot = 0; uint32_t cnt = 0;
      for (uint32_t r = 0; r < NSTIM; ++r)
        if (r != q) { double o = overlap(recCols, refClampCols[r]); best = std::max(best, o); tot += o; cnt++; }
      sumBest += best; sumMeanOther += cnt ? tot / cnt : 0.0;
    }
    printf("\n============ RETRIEVED-POPULATION MULTIPLICITY (NSTIM=%u) ============\n", NSTIM);
    printf("  population: %u neurons used, mean multiplicity %.2f, max %u\n", popN, popMean, maxMult);
    printf("  recalled AND in reference    : n=%.0f  mean multiplicity %.2f\n", nIn, nIn ? mIn / nIn : 0.0);
    printf("  recalled but NOT in reference: n=%.0f  mean multiplicity %.2f  (%.2fx population)\n", nOut,
           nOut ? mOut / nOut : 0.0, (nOut && popMean) ? (mOut / nOut) / popMean : 0.0);
    printf("  self %.3f | best-other %.3f | MEAN-over-others %.3f  -> %s\n", sumSelf / NQ, sumBest / NQ,
           sumMeanOther / NQ, (sumMeanOther / NQ > 0.5 * sumBest / NQ) ? "UNIFORM contamination" : "TAIL-dominated");
    auto jac2 = [&](const Cols& a, const Cols& b) {
      Cols i, u;
      std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(i));
      std::set_union(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(u));
      return u.empty() ? 0.0 : (double)i.size() / u.size();
    };
    std::vector<Cols> ns(NSTIM);
    for (uint32_t q = 0; q < NSTIM; ++q) ns[q] = neuronSet(refClampBal[q].data());
    std::vector<double> J, IO, IX;
    for (uint32_t i = 0; i < NSTIM; ++i)
      for (uint32_t j = i + 1; j < NSTIM; ++j) {
        J.push_back(jac2(ns[i], ns[j]));
        Cols a = stimCols[i], b = stimCols[j];
        std::sort(a.begin(), a.end()); std::sort(b.begin(), b.end());
        Cols ii;
        std::set_intersection(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(ii));
        IO.push_back((double)ii.size());
        IX.push_back((double)std::max(i, j));
      }
    auto pear = [&](std::vector<double>& x, std::vector<double>& y) {
      double mx = 0, my = 0;
      for (size_t i = 0; i < x.size(); ++i) { mx += x[i]; my += y[i]; }
      mx /= x.size(); my /= y.size();
      double sxy = 0, sxx = 0, syy = 0;
      for (size_t i = 0; i < x.size(); ++i) { double dx = x[i] - mx, dy = y[i] - my; sxy += dx * dy; sxx += dx * dx; syy += dy * dy; }
      return (sxx > 0 && syy > 0) ? sxy / std::sqrt(sxx * syy) : 0.0;
    };
    std::vector<double> Js = J;
    std::sort(Js.begin(), Js.end());
    printf("  heavy tail: %zu pairs | mean J %.5f | p99 %.5f | max %.5f\n", J.size(),
           std::accumulate(J.begin(), J.end(), 0.0) / J.size(), Js[(size_t)(0.99 * (Js.size() - 1))], Js.back());
    printf("  corr(assemblyJaccard, INPUT overlap)      r = %+.3f\n", pear(J, IO));
    printf("  corr(assemblyJaccard, allocation index)   r = %+.3f\n", pear(J, IX));
    printf("======================================================================\n");
  }

  // long free-run wave characterisation, src/axon.mm:1804-1858
  if (C.wave) {
    uint32_t TW = std::min(C.waveT, 60u);
    uint32_t NQ = std::min(NSTIM, 12u);
    std::vector<double> ovR(TW, 0), nCol(TW, 0), nNeu(TW, 0), jPrev(TW, 0), fracA(TW, 0), jPrev2(TW, 0);
    double unionSz = 0, unionE = 0, unionO = 0, unionX = 0;
    for (uint32_t q = 0; q < NQ; ++q) {
      present(q, 1.0, TW, CLAMP, false, true, 7000 + q);
      Cols refN = neuronSet(refClampBal[q].data());
      Cols prev, prev2, uni, uniE, uniO;
      for (uint32_t t = 0; t < TW; ++t) {
        const uint32_t* row = E.hist.data() + (size_t)t * NCOL;
        Cols cur = neuronSet(row);
        uint32_t nc = 0;
        for (uint32_t c = IN_COLS; c < NCOL; ++c) if (row[c]) nc++;
        nCol[t] += nc; nNeu[t] += cur.size();
        Cols ii;
        std::set_intersection(cur.begin(), cur.end(), refN.begin(), refN.end(), std::back_inserter(ii));
        ovR[t] += (cur.empty() || refN.empty()) ? 0.0 : (double)ii.size() / std::sqrt((double)cur.size() * refN.size());
        fracA[t] += refN.empty() ? 0.0 : (double)ii.size() / refN.size();
        if (t >= CLAMP) {
          uni.insert(uni.end(), cur.begin(), cur.end());
          if (t % 2u == 0u) uniE.insert(uniE.end(), cur.begin(), cur.end());
          else uniO.insert(uniO.end(), cur.begin(), cur.end());
        }
        jPrev[t] += t ? jaccard(cur, prev) : 0.0;
        jPrev2[t] += t > 1 ? jaccard(cur, prev2) : 0.0;
        prev2 = prev; prev = cur;
      }
      std::sort(uni.begin(), uni.end());
      uni.erase(std::unique(uni.begin(), uni.end()), uni.end());
      unionSz += (double)uni.size();
      std::sort(uniE.begin(), uniE.end()); uniE.erase(std::unique(uniE.begin(), uniE.end()), uniE.end());
      std::sort(uniO.begin(), uniO.end()); uniO.erase(std::unique(uniO.begin(), uniO.end()), uniO.end());
      Cols ii;
      std::set_intersection(uniE.begin(), uniE.end(), uniO.begin(), uniO.end(), std::back_inserter(ii));
      unionE += (double)uniE.size(); unionO += (double)uniO.size();
      unionX += (uniE.empty() || uniO.empty()) ? 0.0 : (double)ii.size() / std::sqrt((double)uniE.size() * uniO.size());
    }
    printf("\nPARITY %.0f %.4f %.0f %.4f %.0f %.4f %.4f\n", unionSz / NQ, unionSz / NQ / 1536.0, unionE / NQ,
           unionE / NQ / 1536.0, unionO / NQ, unionO / NQ / 1536.0, unionX / NQ);
    printf("\n================= WAVE: %u free steps after a %u-step cue =================\n", TW - CLAMP, CLAMP);
    printf("  step  phase   cols  neurons   ov(clampRef)  fracOfAssembly  J(t,t-1)   J(t,t-2)\n");
    for (uint32_t t = 0; t < TW; ++t)
      printf("  %4u  %-5s %6.0f %8.0f %13.3f %15.3f %10.3f %10.3f\n", t, t < CLAMP ? "cue" : "FREE", nCol[t] / NQ,
             nNeu[t] / NQ, ovR[t] / NQ, fracA[t] / NQ, jPrev[t] / NQ, jPrev2[t] / NQ);
    printf("==========================================================================\n");
  }

  // free-run diagnostic, src/axon.mm:1861-1887
  {
    printf("\n============ FREE-RUN DIAGNOSTIC (cue %u steps, then released) ============\n", CLAMP);
    printf("  cue=75%%, averaged over %u stimuli.  'margin' = k-th minus (k+1)-th drive\n", NSTIM);
    printf("  step  phase  cols  drive_k  margin  %%marg=0   ov(CLAMPED ref)  ov(FREE ref)\n");
    std::vector<double> ovc(T, 0), ovt(T, 0), mg(T, 0), dk(T, 0), tie(T, 0), zer(T, 0), nc(T, 0), ovf(T, 0);
    for (uint32_t q = 0; q < NSTIM; ++q) {
      present(q, 0.75, T, CLAMP, false, true, 4000 + q);
      const uint32_t* H = E.hist.data();
      const uint32_t* S = E.stats.data();
      Cols ref = colsOf(H + (size_t)(CLAMP - 1) * NCOL);
      for (uint32_t t = 0; t < T; ++t) {
        Cols a = colsOf(H + (size_t)t * NCOL);
        ovc[t] += overlap(a, ref); ovt[t] += overlap(a, refClampCols[q]); ovf[t] += overlap(a, refFreeCols[q]);
        const uint32_t* sb = S + 64 + t * 8;
        double n = sb[2];
        nc[t] += n;
        if (n > 0) { mg[t] += sb[0] / n; dk[t] += sb[1] / n; tie[t] += 100.0 * sb[3] / n; zer[t] += 100.0 * sb[4] / n; }
      }
    }
    for (uint32_t t = 0; t < T; ++t)
      printf("  %4u  %-5s %5.0f %8.1f %7.1f %8.1f   %14.3f  %12.3f\n", t, t < CLAMP ? "cue" : "FREE", nc[t] / NSTIM,
             dk[t] / NSTIM, mg[t] / NSTIM, tie[t] / NSTIM, ovt[t] / NSTIM, ovf[t] / NSTIM);
    printf("==========================================================================\n");
  }

  // final completion table, src/axon.mm:1889-1908
  double m50 = 0;
  for (double keep : {1.0, 0.75, 0.5, 0.35, 0.25}) {
    double self = 0, other = 0, selfF = 0, otherF = 0;
    for (uint32_t p = 0; p < NSTIM; ++p) {
      present(p, keep, T, CLAMP, false, true, 3000 + p);
      Cols a = assemblyOf(T);
      self += overlap(a, refClampCols[p]); selfF += overlap(a, refFreeCols[p]);
      double best = 0, bestF = 0;
      for (uint32_t q = 0; q < NSTIM; ++q)
        if (q != p) { best = std::max(best, overlap(a, refClampCols[q])); bestF = std::max(bestF, overlap(a, refFreeCols[q])); }
      other += best; otherF += bestF;
    }
    self /= NSTIM; other /= NSTIM; selfF /= NSTIM; otherF /= NSTIM;
    if (keep == 0.5) m50 = self - other;
    if (!C.quiet)
      printf("  %3.0f%% |  %16.3f %6.3f %+7.3f  |  %11.3f %6.3f %+7.3f\n", keep * 100, self, other, self - other,
             selfF, otherF, selfF - otherF);
  }
  if (C.quiet)
    printf("tgt=%-4u k=%-3u inbr=%-3u stimc=%-4u bias=%-4u nand=%u | %7.4f ms %6.0f st/s asm=%-5.0f xtalk=%.3f margin50=%+.3f wd=%.2f\n",
           C.targetC, C.K, C.inBranches, C.STIM_COLS, C.biasUp, C.nAnd, msStep, 1000.0 / msStep, sz, xtalk, m50, wstat());
  else
    printf("\n=== DONE ===\n");
  return 0;
}

}  // namespace oracle
