// Host protocol of the `axon` command line: the experiment of rakib-nyc/axon src/axon.mm
// (main, src/axon.mm:669-1911) on the B200 engine, printing the same lines.
//
// Structure on the GPU side: training presentations change the network and run in order,
// one persistent launch each (axon_present). Everything after training is a readout that
// changes no weight, so each analysis block submits all of its presentations at once as
// one batched recall (axon_recall) and then does its host-side set algebra on the
// returned spike vectors.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/axon_capi.h"

namespace axon {

// key=value tunables with the reference's defaults (src/axon.mm:688-735); the last
// occurrence of a key wins and values are read with atoi.
struct CliArgs {
  uint32_t nand = 4, target = 256, k = 6, dthr = 2, boost = 4, mode = 1, epochs = 30, T = 10, clampsteps = 5,
           stim = 12, quiet = 0, seed = 0, split = 0, unionchar = 0, biasup = 0, biasdown = 1, biasshift = 4,
           biasdownevery = 1, inbr = 8, stimcols = 128, incols = 512, ncol = 4096, diag = 0, profile = 0,
           topkpar = 1, vtopk = 0, contrast = 0, bandlo = 5, bandhi = 11, margingate = 1, hetero = 0, vbs = 0,
           ltdrep = 1, ltdevery = 1, ktest = 0, facil = 0, deep = 0, wave = 0, wavet = 35, trainclamp = 0,
           cueflip = 0;
  int device = 0;
  static CliArgs parse(int argc, char** argv);
  std::string check() const;  // empty when the run is supported
  axon_cfg engine_cfg() const;
};

int run_protocol(const CliArgs& a);

}  // namespace axon
