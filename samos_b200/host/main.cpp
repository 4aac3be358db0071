// main.cpp -- `samos-gpu <conf file>`: the reference's `samos <conf file>`
// (src/samos.cpp:160-180) over the B200 engine.  `--check` parses and
// resolves every command without touching a GPU and prints the program;
// `--read-particles <file>` prints a particle file as the reader takes it.
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
    else if (!std::strcmp(argv[i], "--read-particles") && i + 1 < argc) {  // print a particle file as read
      try {
        samos_host::Particles P = samos_host::read_particles(argv[++i]);
        std::printf("id type radius x y z vx vy vz nx ny nz omega ix iy iz mass\n");
        for (size_t k = 0; k < P.size(); k++)
          std::printf("%d %d %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %.17g %d %d %d %.17g\n",
                      P.id[k], P.type[k], P.radius[k], P.x[k], P.y[k], P.z[k], P.vx[k], P.vy[k], P.vz[k], P.nx[k],
                      P.ny[k], P.nz[k], P.omega[k], P.ix[k], P.iy[k], P.iz[k], P.mass[k]);
      } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << std::endl;
        return 1;
      }
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
