// samos_host.hpp -- C++ host for the B200 engine: the `samos <conf file>`
// command loop of the reference (src/samos.cpp) for the hot-path commands,
// with the plugin factories' names, parameter keys, defaults and error
// behaviour, driving libsamos_gpu.so through the C ABI (samos_gpu.h).
#pragma once

#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "samos_gpu.h"

namespace samos_host {

// pairs_type of the reference (src/parser/parse_parameters.hpp:43): flags map to "".
using Params = std::map<std::string, std::string>;

// Messenger::ERROR + throw std::runtime_error, as the reference reports errors.
struct HostError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// ---- conf-file syntax (conf.cpp) ---------------------------------------------------
std::string trim(const std::string& s);
// "{ k = v; flag, k2 = v2; }" -> map (key_value_sequence, parse_parameters.hpp:47-52);
// returns false on a syntax error.
bool parse_params(const std::string& text, Params& out);
// "cmd rest" -> (cmd, rest)
void split_command(const std::string& line, std::string& cmd, std::string& rest);
// "name { ... }" -> (name, "{ ... }"); the brace part may be absent ("{}").
bool split_type_params(const std::string& rest, std::string& type, std::string& params,
                       bool file_name = false);

// ---- particles (particles.cpp) -------------------------------------------------------
struct Particles {
  std::vector<int32_t> id, type, ix, iy, iz, molecule;
  std::vector<double> radius, x, y, z, vx, vy, vz, nx, ny, nz, omega, mass;
  int ntypes = 0;  // distinct types (System::System, system.cpp:445)
  size_t size() const { return x.size(); }
};
// System::System input reader (src/system/system.cpp:76-450): `keys:` header,
// the deprecated `# id type radius ...` header, or the old positional format.
Particles read_particles(const std::string& path);
// numbers of a command's parameters; a malformed one stops with "Could not parse <what> command."
int64_t to_i64(const std::string& s, const char* what);
double to_dbl(const std::string& s, const char* what);

// ---- dumps (dump.cpp) -----------------------------------------------------------------
struct DumpSpec {
  std::string name, type, ext, dir, path;  // path: the single file when not `multi`
  int64_t start = 0, freq = 100, offset = 0;
  bool multi = false, header = false, keys = false;
  double scale = 1.0;
  Params p;
};
// What a dump reads: the particles (refreshed from the device), the box, and
// forces and surface normals when a dump asks for them.
struct DumpState {
  const Particles* parts = nullptr;
  double lx = 0.0, ly = 0.0, lz = 0.0;
  const std::vector<double> *fx = nullptr, *fy = nullptr, *fz = nullptr, *Nx = nullptr, *Ny = nullptr, *Nz = nullptr;
  const std::vector<int32_t>* coordination = nullptr;
};
// Dump ctor (src/dump/dump.cpp:45-340): validates, opens the single file
// (and writes the DCD header) as the reference does at construction.
DumpSpec make_dump(const std::string& name, const Params& p, int32_t n_particles);
bool dump_due(const DumpSpec& d, int64_t step);  // Dump::dump, dump.cpp:353-356
void write_dump(const DumpSpec& d, int64_t step, const DumpState& s);

// ---- plugins (plugins.cpp) -------------------------------------------------------------
struct PairSpec {
  std::string name;
  int kind = 0;
  double glob[SG_PAIR_NPARAM] = {0};
  std::vector<double> table;  // ntypes^2 * SG_PAIR_NPARAM
  bool use_radii = false, phase_in = false, shifted = false, has_pair_params = false;
  double phase_value[4] = {0.0, 0.0, 1.0, 1000.0};
};
struct AlignSpec {
  std::string name;
  int kind = 0;
  double J = 0.0, rcut = 0.0;
  std::vector<double> table;  // ntypes^2 * 2: {J, rcut}
  bool has_pair_params = false;
};
struct ExternalSpec {
  std::string name;
  int kind = 0;
  double alpha = 1.0;
  std::vector<double> type_alpha;
  bool has_params = false;
};
struct ConstraintSpec {
  int kind = 0;
  double params[10] = {0};  // the 9 values of sg_add_constraint
};
struct IntegratorSpec {
  std::string name;
  int kind = 0;
  double params[SG_INT_NPARAM] = {0};
  double temperature[4] = {0.0, 0.0, 1.0, 1000.0};
  std::string group = "all";  // integrator.hpp:67-109
};

PairSpec resolve_pair(const std::string& name, const Params& p, int ntypes, double nlist_rcut);
void apply_pair_param(PairSpec& s, const Params& p, int ntypes);
AlignSpec resolve_align(const std::string& name, const Params& p, int ntypes, double nlist_rcut);
void apply_align_param(AlignSpec& s, const Params& p, int ntypes);
ExternalSpec resolve_external(const std::string& name, const Params& p, int ntypes);
void apply_external_param(ExternalSpec& s, const Params& p, int ntypes);
ConstraintSpec resolve_constraint(const std::string& name, const Params& p);
IntegratorSpec resolve_integrator(const std::string& name, const Params& p, double dt_global);

// ---- the command loop (runner.cpp) --------------------------------------------------
struct RunOptions {
  bool check_only = false;  // parse and resolve every command, create no device state
  bool quiet = false;
  int device = 0;
};

class Samos {
 public:
  explicit Samos(RunOptions opt) : opt_(opt) {}
  ~Samos();
  void execute_file(const std::string& conf_path);
  void execute_line(const std::string& line, int line_no);
  // summary of the resolved program (used by --check)
  std::string describe() const;
  int64_t steps_run() const { return steps_run_; }

 private:
  void need_system(const char* what) const;
  void ensure_engine();
  void commit_forces();
  void cmd_run(int64_t steps);
  void cmd_dump(const std::string& rest);
  void cmd_log(const std::string& rest);
  void cmd_group(const std::string& name, const Params& p);
  void report(int64_t step);  // dumps and logs at the top of global step `step`
  void check(int rc, const char* what) const;

  RunOptions opt_;
  std::string base_dir_;
  sg_system* h_ = nullptr;
  bool has_box_ = false, periodic_ = false, has_input_ = false;
  double lx_ = 30.0, ly_ = 30.0, lz_ = 30.0;
  Particles parts_;
  bool has_nlist_ = false;
  double nl_rcut_ = 0.0, nl_pad_ = 0.0;
  double dt_ = 0.0;
  std::vector<ConstraintSpec> constraints_;
  std::map<std::string, PairSpec> pairs_;
  std::map<std::string, AlignSpec> aligns_;
  std::map<std::string, ExternalSpec> externals_;
  std::map<std::string, IntegratorSpec> integrators_;  // key type_group, as samos.cpp
  std::map<std::string, int> groups_;                   // `group` commands: name -> engine group index
  std::vector<std::string> committed_integ_;           // device order (map order)
  std::vector<DumpSpec> dumps_;
  struct Log { std::string name; int64_t freq = 1; std::vector<std::string> cols; };
  std::vector<Log> logs_;
  int64_t steps_run_ = 0;  // the reference's time_step
};

}  // namespace samos_host
