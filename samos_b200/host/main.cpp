// main.cpp -- `samos-gpu <conf file>`: the reference's `samos <conf file>`
// (src/samos.cpp:160-180) over the B200 engine.  `--check` parses and
// resolves every command without touching a GPU and prints the program.
#include <cstdio>
#include <cstring>
#include <exception>
#include <iostream>

#include "samos_host.hpp"

int main(int argc, char** argv) {
  samos_host::RunOptions opt;
  const char* conf = nullptr;
  for (int i = 1; i < argc; i++) {
    if (!std::strcmp(argv[i], "--check")) opt.check_only = true;
    else if (!std::strcmp(argv[i], "--quiet")) opt.quiet = true;
    else if (!std::strcmp(argv[i], "--device") && i + 1 < argc) opt.device = std::atoi(argv[++i]);
    else if (!std::strcmp(argv[i], "--params") && i + 1 < argc) {  // print one parsed parameter block
      samos_host::Params p;
      if (!samos_host::parse_params(argv[++i], p)) return 2;
      for (const auto& kv : p) std::cout << kv.first << "=" << kv.second << "\n";
      return 0;
    }
    else conf = argv[i];
  }
  if (!conf) {
    std::cerr << "Usage: " << std::endl << "    samos-gpu [--check] [--quiet] [--device N] <config file name>" << std::endl;
    return -1;
  }
  try {
    samos_host::Samos sim(opt);
    sim.execute_file(conf);
    if (opt.check_only) std::cout << sim.describe();
  } catch (const std::exception& e) {
    std::cerr << "ERROR: " << e.what() << std::endl;
    return 1;
  }
  return 0;
}
