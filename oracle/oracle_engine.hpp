// AXON CPU oracle: engine state and the per-timestep kernel rules.
//
// TEST INFRASTRUCTURE ONLY. This file is the CPU restatement that the CUDA engine is
// checked against. It is never linked into the product library or the product CLI;
// only tests/, the smoke check and bench.py's cpu_baseline leg use it, as the checker.
//
// Every rule here restates a Metal kernel of rakib-nyc/axon src/axon.mm (cited per
// function). Integer semantics are kept exactly: 32-bit unsigned wrap-around for the
// atomic counters, the reference's tie rules, its skip conditions and its clip-on-all-
// lanes quirk. Work is split over columns across a small thread pool; counters that the
// reference accumulates with relaxed atomics are summed per thread and reduced after,
// which is order-independent for unsigned addition.
#pragma once
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace oracle {

// ---------------------------------------------------------------- geometry constants
// src/axon.mm:31-43. NCOL and IN_COLS are runtime values (ncol=, incols=).
constexpr uint32_t NPC = 32;      // neurons per column
constexpr uint32_t NSLOT = 32;    // dendritic branches per neuron
constexpr uint32_t SLOT_U4 = 2;   // uint4 per branch per lane (256 presynaptic)
constexpr uint32_t PRESYN = 256;
constexpr uint32_t FANIN = NSLOT * PRESYN;
constexpr uint32_t COLS_PER_GRP = 8;
constexpr uint32_t MAXT = 64;     // hist rows (src/axon.mm:766)

// hash32, src/axon.mm:54
inline uint32_t hash32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
  return x;
}

inline uint32_t popc(uint32_t x) { return (uint32_t)__builtin_popcount(x); }

// Per-dispatch control block, src/axon.mm:56-83 (same fields, same meaning).
struct Params {
  uint32_t k = 0, theta = 0, dthr = 0, boost = 0, mode = 0, inCols = 0, step = 0,
           learn = 0, depress = 0, targetCols = 0, clamp = 0, freeze = 0, biasUp = 0,
           biasDown = 0, biasShift = 0, histOn = 0, useBias = 0, phase = 0, bandLo = 0,
           bandHi = 0, marginGate = 0, hetero = 0, ltdRep = 0, biasDownEvery = 0,
           facil = 0;
};

// ---------------------------------------------------------------- thread pool
class Pool {
 public:
  explicit Pool(unsigned n) : n_(n ? n : 1) {
    for (unsigned i = 1; i < n_; ++i) th_.emplace_back([this, i] { worker(i); });
  }
  ~Pool() {
    { std::lock_guard<std::mutex> g(m_); stop_ = true; ++gen_; }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  unsigned size() const { return n_; }
  // fn(begin, end, worker_index) over [0, n) split into contiguous chunks.
  void run(uint32_t n, const std::function<void(uint32_t, uint32_t, unsigned)>& fn) {
    if (n_ == 1 || n < 2) { fn(0, n, 0); return; }
    {
      std::lock_guard<std::mutex> g(m_);
      fn_ = &fn; total_ = n; pending_ = n_ - 1; ++gen_;
    }
    cv_.notify_all();
    chunk(0);
    std::unique_lock<std::mutex> lk(m_);
    done_cv_.wait(lk, [this] { return pending_ == 0; });
    fn_ = nullptr;
  }

 private:
  void chunk(unsigned w) {
    uint32_t per = (total_ + n_ - 1) / n_;
    uint32_t b = std::min(total_, per * w), e = std::min(total_, b + per);
    if (b < e) (*fn_)(b, e, w);
  }
  void worker(unsigned w) {
    uint64_t seen = 0;
    for (;;) {
      std::unique_lock<std::mutex> lk(m_);
      cv_.wait(lk, [&] { return gen_ != seen; });
      seen = gen_;
      if (stop_) return;
      lk.unlock();
      chunk(w);
      lk.lock();
      if (--pending_ == 0) done_cv_.notify_one();
    }
  }
  unsigned n_;
  std::vector<std::thread> th_;
  std::mutex m_;
  std::condition_variable cv_, done_cv_;
  const std::function<void(uint32_t, uint32_t, unsigned)>* fn_ = nullptr;
  uint32_t total_ = 0;
  unsigned pending_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};

// ---------------------------------------------------------------- bit-serial counter ops
// src/axon.mm:371-420. Each operates on one 32-bit word of each plane (32 synapses);
// the reference applies the same ops component-wise to uint4.
inline void bs_inc(uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t& a3, uint32_t m) {
  uint32_t c = m, t;
  t = a0 ^ c; c = a0 & c; a0 = t;
  t = a1 ^ c; c = a1 & c; a1 = t;
  t = a2 ^ c; c = a2 & c; a2 = t;
  t = a3 ^ c; c = a3 & c; a3 = t;
  a0 |= c; a1 |= c; a2 |= c; a3 |= c;  // carry out of bit 3: value was 15, saturate
}
inline void bs_dec(uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t& a3, uint32_t m) {
  uint32_t b = m, t;
  t = a0 ^ b; b = ~a0 & b; a0 = t;
  t = a1 ^ b; b = ~a1 & b; a1 = t;
  t = a2 ^ b; b = ~a2 & b; a2 = t;
  t = a3 ^ b; b = ~a3 & b; a3 = t;
  uint32_t keep = ~b;  // borrow out of bit 3: value was 0, saturate
  a0 &= keep; a1 &= keep; a2 &= keep; a3 &= keep;
}
// mask of synapses whose 4-bit value is < K (resp. > K), MSB-first compare
inline uint32_t bs_lt(uint32_t a3, uint32_t a2, uint32_t a1, uint32_t a0, uint32_t K) {
  const uint32_t a[4] = {a0, a1, a2, a3};
  uint32_t lt = 0, eq = ~0u;
  for (int i = 3; i >= 0; --i) {
    uint32_t kb = (K >> i) & 1u;
    if (kb) lt |= eq & ~a[i];
    if (i) eq &= kb ? a[i] : ~a[i];
  }
  return lt;
}
inline uint32_t bs_gt(uint32_t a3, uint32_t a2, uint32_t a1, uint32_t a0, uint32_t K) {
  const uint32_t a[4] = {a0, a1, a2, a3};
  uint32_t gt = 0, eq = ~0u;
  for (int i = 3; i >= 0; --i) {
    uint32_t kb = (K >> i) & 1u;
    if (!kb) gt |= eq & a[i];
    if (i) eq &= kb ? a[i] : ~a[i];
  }
  return gt;
}
inline void bs_set(uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t& a3, uint32_t m, uint32_t C) {
  uint32_t keep = ~m;
  a0 = (a0 & keep) | (((C >> 0) & 1u) ? m : 0u);
  a1 = (a1 & keep) | (((C >> 1) & 1u) ? m : 0u);
  a2 = (a2 & keep) | (((C >> 2) & 1u) ? m : 0u);
  a3 = (a3 & keep) | (((C >> 3) & 1u) ? m : 0u);
}
// both masks are taken before either is applied (src/axon.mm:413-420)
inline void bs_clip(uint32_t& a0, uint32_t& a1, uint32_t& a2, uint32_t& a3, uint32_t lo, uint32_t hi) {
  uint32_t l = bs_lt(a3, a2, a1, a0, lo);
  uint32_t g = bs_gt(a3, a2, a1, a0, hi);
  bs_set(a0, a1, a2, a3, l, lo);
  bs_set(a0, a1, a2, a3, g, hi);
}

// Exact k-of-32 ranking, src/axon.mm:134-144: rank = #{j: v_j > v_i or (v_j == v_i and
// j < i)}; fire if rank < k; vk / vk1 are the values ranked k-1 and k (0 if none).
inline uint32_t kwta_ballot_margin(const uint32_t v[32], uint32_t k, uint32_t& vk, uint32_t& vk1) {
  uint32_t ball = 0;
  vk = 0; vk1 = 0;
  for (uint32_t i = 0; i < 32; ++i) {
    uint32_t rank = 0;
    for (uint32_t j = 0; j < 32; ++j) rank += (v[j] > v[i] || (v[j] == v[i] && j < i)) ? 1u : 0u;
    if (rank == k - 1u) vk = std::max(vk, v[i]);
    if (rank == k) vk1 = std::max(vk1, v[i]);
    if (rank < k) ball |= 1u << i;
  }
  return ball;
}

// ---------------------------------------------------------------- engine
struct Engine {
  uint32_t NCOL, IN_COLS, N, NGRP;
  size_t PLANE_WORDS;  // 32-bit words per plane = NCOL*NSLOT*SLOT_U4*32*4
  Pool* pool;
  std::vector<uint32_t> W[4];
  std::vector<uint32_t> conn, spk[2], drive, bbits, acc, bias, marg, refBall, driveLog, mult,
      stim, stats, hist, theta;
  uint32_t topkPar = 1;  // 1 = k_topk_par semantics (default), 0 = k_topk_serial

  Engine(uint32_t ncol, uint32_t incols, Pool* p)
      : NCOL(ncol), IN_COLS(incols), N(ncol * NPC), NGRP(ncol / COLS_PER_GRP), pool(p) {
    PLANE_WORDS = (size_t)NCOL * NSLOT * SLOT_U4 * 32 * 4;
    for (auto& w : W) w.assign(PLANE_WORDS, 0u);
    conn.assign((size_t)NCOL * NSLOT, 0u);
    spk[0].assign(NCOL, 0u); spk[1].assign(NCOL, 0u);
    drive.assign(NCOL, 0u); bbits.assign(N, 0u); acc.assign(N, 0u); bias.assign(N, 0u);
    marg.assign(NCOL, 0u); refBall.assign(NCOL, 0u); driveLog.assign(256, 0u);
    mult.assign(N, 0u); stim.assign(NCOL, 0u); stats.assign(1024, 0u);
    hist.assign((size_t)MAXT * NCOL, 0u); theta.assign(16, 0u);
  }

  // word index of component comp of uint4 number ((col*NSLOT+s)*SLOT_U4+j)*32+lane
  static size_t widx(uint32_t col, uint32_t s, uint32_t j, uint32_t lane, uint32_t comp) {
    return ((((size_t)col * NSLOT + s) * SLOT_U4 + j) * 32 + lane) * 4 + comp;
  }

  // k_init_w, src/axon.mm:86-104, and k_init_conn, src/axon.mm:109-117 (cfg at :778)
  void init(uint32_t nAnd, uint32_t seed, uint32_t inBr) {
    size_t nU4 = PLANE_WORDS / 4;
    pool->run((uint32_t)(nU4 / 1024), [&](uint32_t b, uint32_t e, unsigned) {
      for (size_t gg = (size_t)b * 1024; gg < (size_t)e * 1024; ++gg) {
        uint32_t g = (uint32_t)gg ^ (seed * 0x9E3779B9u);
        uint32_t m[4] = {~0u, ~0u, ~0u, ~0u};
        for (uint32_t i = 0; i < nAnd; ++i)
          for (uint32_t c = 0; c < 4; ++c) m[c] &= hash32(g * 32u + i * 4u + c);
        const uint32_t cadd[4] = {11, 13, 17, 19};
        for (uint32_t c = 0; c < 4; ++c) {
          uint32_t cc = hash32(g * 8u + cadd[c]);
          W[3][gg * 4 + c] = m[c];
          W[2][gg * 4 + c] = ~m[c] | cc;
          W[1][gg * 4 + c] = cc;
          W[0][gg * 4 + c] = ~cc;
        }
      }
    });
    uint32_t nGrp = NGRP, nInGrp = IN_COLS / COLS_PER_GRP;
    for (uint32_t g = 0; g < NCOL * NSLOT; ++g) {
      uint32_t s = g % NSLOT;
      uint32_t h = hash32(g * 2246822519u + 7u + seed * 2654435761u);
      conn[g] = (s < inBr) ? (h % nInGrp) : (nInGrp + h % (nGrp - nInGrp));
    }
  }

  // k_drive, src/axon.mm:150-190
  void k_drive(const uint32_t* spkIn, const Params& P) {
    pool->run(NCOL, [&](uint32_t cb, uint32_t ce, unsigned) {
      for (uint32_t col = cb; col < ce; ++col) {
        uint32_t dsum = 0;
        for (uint32_t lane = 0; lane < 32; ++lane) {
          uint32_t a = 0, bb = 0, base = col * NSLOT;
          for (uint32_t s = 0; s < NSLOT; ++s) {
            uint32_t g = conn[base + s];
            const uint32_t* sw = spkIn + (size_t)g * 8;
            uint32_t any = sw[0] | sw[1] | sw[2] | sw[3] | sw[4] | sw[5] | sw[6] | sw[7];
            if (any == 0u) continue;
            uint32_t c = 0;
            for (uint32_t j = 0; j < 2; ++j)
              for (uint32_t q = 0; q < 4; ++q) c += popc(W[3][widx(col, s, j, lane, q)] & sw[j * 4 + q]);
            bool nmda = c >= P.dthr;
            if (nmda) bb |= 1u << s;
            if (P.mode == 0u) a += c;
            else if (P.mode == 1u) a += nmda ? (c + P.boost) : c;
            else a += nmda ? 1u : 0u;
          }
          if (P.facil != 0u && ((spkIn[col] >> lane) & 1u) != 0u) a += P.facil;
          uint32_t bi = (P.useBias != 0u) ? (bias[col * 32 + lane] >> P.biasShift) : 0u;
          a = (a > bi) ? (a - bi) : 0u;
          acc[col * 32 + lane] = a;
          bbits[col * 32 + lane] = bb;
          dsum += a;
        }
        drive[col] = dsum;
      }
    });
  }

  // k_topk_par, src/axon.mm:301-352 (default), and k_topk_serial, src/axon.mm:259-292.
  // theta[0] = max(prefix, 1), theta[1] = residual need.
  void k_topk(const Params& P) {
    uint32_t need = P.targetCols, prefix = 0;
    for (int by = 2; by >= 0; --by) {
      uint32_t h[256] = {0};
      uint32_t shHi = (uint32_t)(by + 1) * 8u, shLo = (uint32_t)by * 8u;
      for (uint32_t c = P.inCols; c < NCOL; ++c) {
        uint32_t d = drive[c];
        if ((d >> shHi) == (prefix >> shHi)) h[(d >> shLo) & 255u]++;
      }
      if (topkPar) {
        uint32_t scan[257];
        scan[256] = 0;
        for (int i = 255; i >= 0; --i) scan[i] = scan[i + 1] + h[i];
        uint32_t sel = 0;
        for (uint32_t t = 0; t < 256; ++t)
          if (scan[t] >= need && scan[t + 1] < need) sel = t;
        need = need - scan[sel + 1];
        prefix |= sel << shLo;
      } else {
        uint32_t cum = 0, b = 0, above = 0;
        for (int i = 255; i >= 0; --i) {
          if (cum + h[i] >= need) { b = (uint32_t)i; above = cum; break; }
          cum += h[i];
        }
        need = need - above;
        prefix |= b << shLo;
      }
    }
    theta[0] = std::max(prefix, 1u);
    theta[1] = need;
  }

  // k_emit, src/axon.mm:192-236
  void k_emit(uint32_t* spkOut, const Params& P) {
    unsigned nt = pool->size();
    std::vector<uint32_t> part((size_t)nt * 1024 + (size_t)nt * 256, 0u);
    pool->run(NCOL, [&](uint32_t cb, uint32_t ce, unsigned w) {
      uint32_t* st = part.data() + (size_t)w * 1024;
      uint32_t* dl = part.data() + (size_t)nt * 1024 + (size_t)w * 256;
      for (uint32_t col = cb; col < ce; ++col) {
        uint32_t vk, vk1;
        uint32_t b = kwta_ballot_margin(&acc[col * 32], P.k, vk, vk1);
        if (drive[col] < std::max(theta[0], 1u)) b = 0u;
        if (P.clamp != 0u && col < P.inCols) b = stim[col];
        for (uint32_t lane = 0; lane < 32; ++lane) {
          uint32_t gid = col * 32 + lane;
          if (((b >> lane) & 1u) != 0u && col >= P.inCols) st[2] += popc(bbits[gid]);
          if (col >= P.inCols && ((refBall[col] >> lane) & 1u) != 0u) {
            uint32_t o = (mult[gid] > 1u) ? 0u : 2u;
            dl[P.step * 4u + o + 0u] += acc[gid];
            dl[P.step * 4u + o + 1u] += 1u;
          }
        }
        spkOut[col] = b;
        marg[col] = (vk > vk1) ? 1u : 0u;
        if (P.histOn != 0u) hist[(size_t)P.step * NCOL + col] = b;
        if (b != 0u && col >= P.inCols) {
          uint32_t sb = 64u + P.step * 8u;
          st[0] += 1u;
          st[1] += popc(b);
          st[sb + 0u] += vk - vk1;
          st[sb + 1u] += vk;
          st[sb + 2u] += 1u;
          if (vk == vk1) st[sb + 3u] += 1u;
          if (vk == 0u) st[sb + 4u] += 1u;
        }
      }
    });
    for (unsigned w = 0; w < nt; ++w) {
      for (uint32_t i = 0; i < 1024; ++i) stats[i] += part[(size_t)w * 1024 + i];
      for (uint32_t i = 0; i < 256; ++i) driveLog[i] += part[(size_t)nt * 1024 + (size_t)w * 256 + i];
    }
  }

  // k_bias, src/axon.mm:240-253
  void k_bias(const uint32_t* spkOut, const Params& P) {
    for (uint32_t col = P.inCols; col < NCOL; ++col)
      for (uint32_t lane = 0; lane < 32; ++lane) {
        uint32_t gid = col * 32 + lane;
        bool fired = ((spkOut[col] >> lane) & 1u) != 0u;
        int dec = ((P.step % std::max(P.biasDownEvery, 1u)) == 0u) ? (int)P.biasDown : 0;
        int b = (int)bias[gid] + (fired ? (int)P.biasUp : -dec);
        bias[gid] = (uint32_t)std::max(0, b);
      }
  }

  // k_learn, src/axon.mm:436-495
  void k_learn(const uint32_t* spkIn, const uint32_t* spkOut, const Params& P) {
    if (P.phase == 3u) return;
    unsigned nt = pool->size();
    std::vector<uint32_t> part((size_t)nt * 4, 0u);
    pool->run(NCOL, [&](uint32_t cb, uint32_t ce, unsigned w) {
      uint32_t* st = part.data() + (size_t)w * 4;
      for (uint32_t col = cb; col < ce; ++col) {
        uint32_t b = spkOut[col];
        if (b == 0u) continue;
        if (P.marginGate != 0u && marg[col] == 0u) continue;
        uint32_t nLTP[32] = {0}, nLTD[32] = {0};
        for (uint32_t s = 0; s < NSLOT; ++s) {
          uint32_t vote = 0;
          for (uint32_t lane = 0; lane < 32; ++lane)
            if (((b >> lane) & 1u) && ((bbits[col * 32 + lane] >> s) & 1u)) vote |= 1u << lane;
          if (vote == 0u) continue;
          uint32_t g = conn[col * NSLOT + s];
          for (uint32_t lane = 0; lane < 32; ++lane) {
            bool want = (vote >> lane) & 1u;
            for (uint32_t j = 0; j < SLOT_U4; ++j)
              for (uint32_t q = 0; q < 4; ++q) {
                uint32_t sp = spkIn[(size_t)g * 8 + j * 4 + q];
                size_t ix = widx(col, s, j, lane, q);
                uint32_t a0 = W[0][ix], a1 = W[1][ix], a2 = W[2][ix], a3 = W[3][ix];
                uint32_t co = want ? sp : 0u;
                uint32_t nco = popc(co);
                if (P.phase == 1u) { bs_inc(a0, a1, a2, a3, co); nLTP[lane] += nco; }
                else if (P.phase == 2u) {
                  for (uint32_t r = 0; r < P.ltdRep; ++r) bs_dec(a0, a1, a2, a3, co);
                  nLTD[lane] += nco * P.ltdRep;
                } else {
                  bs_inc(a0, a1, a2, a3, co);
                  bs_dec(a0, a1, a2, a3, (want && P.depress != 0u) ? ~sp : 0u);
                }
                if (P.hetero != 0u && P.phase == 1u) bs_dec(a0, a1, a2, a3, want ? ~sp : 0u);
                if (P.bandHi != 0u) bs_clip(a0, a1, a2, a3, P.bandLo, P.bandHi);
                W[0][ix] = a0; W[1][ix] = a1; W[2][ix] = a2; W[3][ix] = a3;
              }
          }
        }
        for (uint32_t lane = 0; lane < 32; ++lane) {
          st[0] += nLTP[lane];
          st[1] += nLTD[lane];
          if (nLTP[lane]) st[2] += 1u;
          if (nLTD[lane]) st[3] += 1u;
        }
      }
    });
    for (unsigned w = 0; w < nt; ++w)
      for (uint32_t i = 0; i < 4; ++i) stats[8 + i] += part[(size_t)w * 4 + i];
  }

  // k_wstat, src/axon.mm:641-646 (u32 atomic total) and the wstat() wrapper at :784-791
  uint32_t wstat_count() const {
    uint32_t t = 0;
    for (size_t i = 0; i < PLANE_WORDS; ++i) t += popc(W[3][i]);
    return t;
  }

  // k_within, src/axon.mm:524-562. out[0..9] accumulate (u32).
  void k_within(const uint32_t* ball, uint32_t inBr, uint32_t inCols, uint32_t useMask,
                const uint32_t* postMask, const uint32_t* multv, uint32_t out[10]) {
    unsigned nt = pool->size();
    std::vector<uint32_t> part((size_t)nt * 10, 0u);
    pool->run(NCOL, [&](uint32_t cb, uint32_t ce, unsigned w) {
      uint32_t* o = part.data() + (size_t)w * 10;
      for (uint32_t col = std::max(cb, inCols); col < ce; ++col)
        for (uint32_t lane = 0; lane < 32; ++lane) {
          uint32_t gid = col * 32 + lane;
          if (useMask != 0u) { if (postMask[gid] == 0u) continue; }
          else if (((ball[col] >> lane) & 1u) == 0u) continue;
          uint32_t fIn = 0, pIn = 0, fOut = 0, pOut = 0;
          for (uint32_t s = inBr; s < NSLOT; ++s) {
            uint32_t g = conn[col * NSLOT + s];
            for (uint32_t j = 0; j < SLOT_U4; ++j)
              for (uint32_t q = 0; q < 4; ++q) {
                uint32_t ap = ball[(size_t)g * 8 + j * 4 + q];
                uint32_t wv = W[3][widx(col, s, j, lane, q)];
                fIn += popc(wv & ap); pIn += popc(ap);
                fOut += popc(wv & ~ap); pOut += popc(~ap);
              }
          }
          o[0] += fIn; o[1] += pIn; o[2] += fOut; o[3] += pOut;
          uint32_t bsel = (multv[gid] > 1u) ? 4u : 6u;
          o[bsel] += fIn; o[bsel + 1] += pIn;
          o[(multv[gid] > 1u) ? 8u : 9u] += 1u;
        }
    });
    for (unsigned w = 0; w < nt; ++w)
      for (uint32_t i = 0; i < 10; ++i) out[i] += part[(size_t)w * 10 + i];
  }

  // k_indeg, src/axon.mm:566-581
  void k_indeg(uint32_t inBr, uint32_t* out) const {
    pool->run(NCOL, [&](uint32_t cb, uint32_t ce, unsigned) {
      for (uint32_t col = cb; col < ce; ++col)
        for (uint32_t lane = 0; lane < 32; ++lane) {
          uint32_t d = 0;
          for (uint32_t s = inBr; s < NSLOT; ++s)
            for (uint32_t j = 0; j < SLOT_U4; ++j)
              for (uint32_t q = 0; q < 4; ++q) d += popc(W[3][widx(col, s, j, lane, q)]);
          out[col * 32 + lane] = d;
        }
    });
  }

  // k_untouched, src/axon.mm:501-519
  void k_untouched(uint32_t inBr, uint32_t* out) const {
    pool->run(NCOL, [&](uint32_t cb, uint32_t ce, unsigned) {
      for (uint32_t col = cb; col < ce; ++col)
        for (uint32_t lane = 0; lane < 32; ++lane) {
          uint32_t u = 0;
          for (uint32_t s = inBr; s < NSLOT; ++s)
            for (uint32_t j = 0; j < SLOT_U4; ++j)
              for (uint32_t q = 0; q < 4; ++q) {
                size_t ix = widx(col, s, j, lane, q);
                uint32_t a0 = W[0][ix], a1 = W[1][ix], a2 = W[2][ix], a3 = W[3][ix];
                uint32_t v5 = ~a3 & a2 & ~a1 & a0, v6 = ~a3 & a2 & a1 & ~a0;
                u += popc(v5 | v6);
              }
          out[col * 32 + lane] = u;
        }
    });
  }

  // k_wdiag, src/axon.mm:591-638. hist48 accumulates (u32).
  void k_wdiag(const uint32_t* memb, const uint32_t* asmSpk, uint32_t nstim, uint32_t inBr,
               uint32_t sel, uint32_t hist48[48]) const {
    unsigned nt = pool->size();
    std::vector<uint32_t> part((size_t)nt * 48, 0u);
    pool->run(NCOL, [&](uint32_t cb, uint32_t ce, unsigned w) {
      uint32_t* hh = part.data() + (size_t)w * 48;
      for (uint32_t col = cb; col < ce; ++col)
        for (uint32_t lane = 0; lane < 32; ++lane) {
          uint32_t mypost = memb[col * 32 + lane];
          if (mypost == 0u) continue;
          uint32_t a[48] = {0};
          for (uint32_t s = 0; s < NSLOT; ++s) {
            bool isAff = s < inBr;
            if (sel == 0u && isAff) continue;
            if (sel == 1u && !isAff) continue;
            uint32_t g = conn[col * NSLOT + s];
            for (uint32_t j = 0; j < SLOT_U4; ++j)
              for (uint32_t q = 0; q < 4; ++q) {
                size_t ix = widx(col, s, j, lane, q);
                uint32_t a0 = W[0][ix], a1 = W[1][ix], a2 = W[2][ix], a3 = W[3][ix];
                uint32_t within = 0, anyp = 0;
                for (uint32_t qq = 0; qq < nstim; ++qq) {
                  uint32_t ap = asmSpk[(size_t)qq * NCOL + (size_t)g * 8 + j * 4 + q];
                  anyp |= ap;
                  if (((mypost >> qq) & 1u) != 0u) within |= ap;
                }
                uint32_t between = anyp & ~within;
                for (uint32_t v = 0; v < 16; ++v) {
                  uint32_t eq = ((v & 1u) ? a0 : ~a0) & ((v & 2u) ? a1 : ~a1) &
                                ((v & 4u) ? a2 : ~a2) & ((v & 8u) ? a3 : ~a3);
                  a[v] += popc(eq & within);
                  a[16 + v] += popc(eq & between);
                  a[32 + v] += popc(eq);
                }
              }
          }
          for (uint32_t i = 0; i < 48; ++i) hh[i] += a[i];
        }
    });
    for (unsigned w = 0; w < nt; ++w)
      for (uint32_t i = 0; i < 48; ++i) hist48[i] += part[(size_t)w * 48 + i];
  }
};

}  // namespace oracle
