// AXON CPU oracle command line: `axon_oracle key=value ...` prints what
// rakib-nyc/axon's `build/axon` prints for the same arguments (src/axon.mm:669-1911).
// TEST INFRASTRUCTURE ONLY. Thread count: AXON_ORACLE_THREADS, else all host cores;
// it is reported on stderr so stdout stays line-comparable with the engine's CLI.
#include <cstdlib>
#include <thread>

#include "oracle_protocol.hpp"

int main(int argc, char** argv) {
  oracle::Cfg c = oracle::Cfg::parse(argc, argv);
  std::string why = c.reject_reason();
  if (c.profile) why = "profile=1 is not restated by the oracle";
  if (!why.empty()) { fprintf(stderr, "axon_oracle: invalid arguments: %s\n", why.c_str()); return 2; }
  unsigned threads = std::thread::hardware_concurrency();
  if (const char* e = std::getenv("AXON_ORACLE_THREADS")) threads = (unsigned)std::atoi(e);
  if (threads == 0) threads = 1;
  fprintf(stderr, "axon_oracle: %u host threads\n", threads);
  oracle::Protocol pr(c, threads);
  int rc = pr.run();
  fprintf(stderr, "axon_oracle: training wall %.3f s\n", pr.trainSeconds);
  return rc;
}
