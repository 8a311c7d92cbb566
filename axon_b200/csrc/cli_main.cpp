// `axon key=value ...`: command-line drop-in for rakib-nyc/axon's build/axon
// (src/axon.mm:669-1911) on the B200 engine. Same keys, same defaults, same printed lines.
// Extra key: device=<index> selects the GPU. Exit status: 0 ok, 2 unsupported or invalid
// arguments, 3 engine failure (message on stderr).
#include <cstdio>

#include "protocol.hpp"

int main(int argc, char** argv) {
  const axon::CliArgs a = axon::CliArgs::parse(argc, argv);
  const std::string why = a.check();
  if (!why.empty()) {
    fprintf(stderr, "axon: %s\n", why.c_str());
    return 2;
  }
  return axon::run_protocol(a);
}
