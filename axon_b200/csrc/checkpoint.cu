// Network checkpoints: the trained state of one network in one file.
//
// The reference keeps no trained network: every run retrains from the seed
// (src/axon.mm:1001-1033). A checkpoint holds what training produces and what readouts
// use - the four counter planes, conn, bias and mult (src/axon.mm:749-768) - with the
// configuration and the training metadata (seed, load, pattern width, epochs; the patterns
// themselves follow from these, src/axon.mm:793-799), so trained networks can be served
// or compared without retraining.
//
// Layout (little-endian): "AXONCKPT", u32 version, u32 section count, the axon_cfg, the
// axon_ckpt_meta, one (u32 buffer id, u32 pad, u64 words, u64 FNV-1a-64 of the words) record
// per section, the sections' words in record order, and a final u64 FNV-1a-64 of every
// preceding byte.
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "engine.hpp"

using namespace axon;

namespace {

constexpr char kMagic[8] = {'A', 'X', 'O', 'N', 'C', 'K', 'P', 'T'};
constexpr uint32_t kVersion = 1;
const axon_buf kSections[] = {AXON_BUF_W0, AXON_BUF_W1, AXON_BUF_W2, AXON_BUF_W3,
                              AXON_BUF_CONN, AXON_BUF_BIAS, AXON_BUF_MULT};
constexpr uint32_t kNsec = sizeof(kSections) / sizeof(kSections[0]);

struct SecRec {
  uint32_t id, pad;
  uint64_t words, fnv;
};

struct Fnv {
  uint64_t h = 1469598103934665603ull;
  void add(const void* p, size_t n) {
    const unsigned char* b = (const unsigned char*)p;
    for (size_t i = 0; i < n; ++i) { h ^= b[i]; h *= 1099511628211ull; }
  }
};

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

}  // namespace

extern "C" axon_status axon_save(axon_net* net, const char* path, const axon_ckpt_meta* meta) {
  if (!net || !path || !meta) return set_error(AXON_EINVAL, "null argument");
  if (!net->initialized) return set_error(AXON_ESTATE, "save before init");
  std::vector<std::vector<uint32_t>> data(kNsec);
  std::vector<SecRec> recs(kNsec);
  for (uint32_t i = 0; i < kNsec; ++i) {
    data[i].resize(net->buf_words(kSections[i]));
    axon_status st = net->read(kSections[i], data[i].data(), data[i].size());
    if (st != AXON_OK) return st;
    Fnv f;
    f.add(data[i].data(), data[i].size() * 4);
    recs[i] = SecRec{(uint32_t)kSections[i], 0u, (uint64_t)data[i].size(), f.h};
  }
  File fh;
  fh.f = fopen(path, "wb");
  if (!fh.f) return set_error(AXON_EINVAL, std::string("cannot open for writing: ") + path);
  Fnv all;
  auto put = [&](const void* p, size_t n) {
    all.add(p, n);
    return fwrite(p, 1, n, fh.f) == n;
  };
  bool ok = put(kMagic, 8) && put(&kVersion, 4) && put(&kNsec, 4) && put(&net->cfg, sizeof(axon_cfg)) &&
            put(meta, sizeof(axon_ckpt_meta)) && put(recs.data(), recs.size() * sizeof(SecRec));
  for (uint32_t i = 0; ok && i < kNsec; ++i) ok = put(data[i].data(), data[i].size() * 4);
  if (ok) ok = fwrite(&all.h, 8, 1, fh.f) == 1;
  if (!ok || fflush(fh.f) != 0) return set_error(AXON_EINVAL, std::string("write failed: ") + path);
  return AXON_OK;
}

extern "C" axon_status axon_load(axon_net* net, const char* path, axon_ckpt_meta* meta) {
  if (!net || !path) return set_error(AXON_EINVAL, "null argument");
  File fh;
  fh.f = fopen(path, "rb");
  if (!fh.f) return set_error(AXON_EINVAL, std::string("cannot open: ") + path);
  Fnv all;
  auto get = [&](void* p, size_t n) {
    if (fread(p, 1, n, fh.f) != n) return false;
    all.add(p, n);
    return true;
  };
  char magic[8];
  uint32_t version = 0, nsec = 0;
  axon_cfg cfg;
  axon_ckpt_meta m;
  if (!get(magic, 8) || std::memcmp(magic, kMagic, 8) != 0) return set_error(AXON_EINVAL, "not an AXON checkpoint");
  if (!get(&version, 4) || version != kVersion) return set_error(AXON_EINVAL, "unsupported checkpoint version");
  if (!get(&nsec, 4) || nsec != kNsec) return set_error(AXON_EINVAL, "corrupt checkpoint header");
  if (!get(&cfg, sizeof(cfg)) || !get(&m, sizeof(m))) return set_error(AXON_EINVAL, "truncated checkpoint");
  if (std::memcmp(&cfg, &net->cfg, sizeof(axon_cfg)) != 0)
    return set_error(AXON_EINVAL, "checkpoint configuration differs from the network's");
  std::vector<SecRec> recs(kNsec);
  if (!get(recs.data(), recs.size() * sizeof(SecRec))) return set_error(AXON_EINVAL, "truncated checkpoint");
  std::vector<std::vector<uint32_t>> data(kNsec);
  for (uint32_t i = 0; i < kNsec; ++i) {
    if (recs[i].id != (uint32_t)kSections[i] || recs[i].words != net->buf_words(kSections[i]))
      return set_error(AXON_EINVAL, "checkpoint sections do not match the network");
    data[i].resize(recs[i].words);
    if (!get(data[i].data(), data[i].size() * 4)) return set_error(AXON_EINVAL, "truncated checkpoint");
    Fnv f;
    f.add(data[i].data(), data[i].size() * 4);
    if (f.h != recs[i].fnv) return set_error(AXON_EINVAL, "checkpoint checksum mismatch (corrupt data)");
  }
  uint64_t tail = 0;
  const uint64_t want = all.h;
  if (fread(&tail, 8, 1, fh.f) != 1 || tail != want) return set_error(AXON_EINVAL, "checkpoint checksum mismatch");
  // every check passed: only now does the network change
  for (uint32_t i = 0; i < kNsec; ++i) {
    axon_status st = net->write(kSections[i], data[i].data(), data[i].size());
    if (st != AXON_OK) return st;
  }
  std::vector<uint32_t> zeros(1024, 0u);
  axon_status st = net->write(AXON_BUF_STATS, zeros.data(), 1024);
  if (st != AXON_OK) return st;
  st = net->write(AXON_BUF_THETA, zeros.data(), 16);
  if (st != AXON_OK) return st;
  net->initialized = true;
  net->w3b_valid = false;
  if (meta) *meta = m;
  return AXON_OK;
}
