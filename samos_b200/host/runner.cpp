// runner.cpp -- the command loop of src/samos.cpp for the hot-path
// commands, over the C ABI.  Command order rules and error messages follow
// the reference (samos.cpp:176-1400): a box before `input`, `input` before
// constraints, potentials and integrators, a constraint before integrators,
// and a constraint plus an integrator before `run`.
//
// Plugins are kept in std::maps keyed as the reference keys them (pair and
// external potentials and aligners by type, integrators by type_group).
// Before each `run` the stateless force terms are handed to the engine in
// map order; integrators are inserted at their map position when created
// and removed by `disable`, so their noise streams persist across runs as the
// reference's RNG objects do.
#include <cctype>
#include <climits>
#include <cmath>
#include <cstdio>
#include <ctime>
#include <fstream>
#include <iostream>
#include <set>
#include <sstream>

#include "samos_host.hpp"

namespace samos_host {

int64_t to_i64(const std::string& s, const char* what) {
  char* end = nullptr;
  const long long v = std::strtoll(s.c_str(), &end, 10);
  if (s.empty() || *end != '\0') throw HostError(std::string("Could not parse ") + what + " command.");
  return v;
}
double to_dbl(const std::string& s, const char* what) {
  char* end = nullptr;
  const double v = std::strtod(s.c_str(), &end);
  if (s.empty() || *end != '\0') throw HostError(std::string("Could not parse ") + what + " command.");
  return v;
}

Samos::~Samos() {
  if (h_) sg_destroy(h_);
}

void Samos::check(int rc, const char* what) const {
  if (rc != SG_OK) {
    const std::string why = h_ ? sg_last_error(h_) : sg_error_string(rc);
    throw HostError(std::string(what) + ": " + sg_error_string(rc) + (why.empty() ? "" : " (" + why + ")"));
  }
}

void Samos::need_system(const char* what) const {
  if (!has_input_)
    throw HostError(std::string("System has not been defined. Please define system using \"input\" command before ") +
                    what + ".");
}

void Samos::ensure_engine() {
  if (h_ || opt_.check_only) return;
  check(sg_set_device(opt_.device), "sg_set_device");
  const int32_t n = (int32_t)parts_.size();
  check(sg_create(1, &n, parts_.ntypes, &h_), "sg_create");
  check(sg_set_box(h_, 0, lx_, ly_, lz_, periodic_ ? 1 : 0), "sg_set_box");
  auto up = [&](const char* f, const void* p) { check(sg_upload(h_, 0, f, p), "sg_upload"); };
  up("x", parts_.x.data()); up("y", parts_.y.data()); up("z", parts_.z.data());
  up("vx", parts_.vx.data()); up("vy", parts_.vy.data()); up("vz", parts_.vz.data());
  up("nx", parts_.nx.data()); up("ny", parts_.ny.data()); up("nz", parts_.nz.data());
  up("omega", parts_.omega.data()); up("radius", parts_.radius.data()); up("mass", parts_.mass.data());
  up("type", parts_.type.data());
  up("ix", parts_.ix.data()); up("iy", parts_.iy.data()); up("iz", parts_.iz.data());
}

void Samos::execute_file(const std::string& conf_path) {
  std::ifstream in(conf_path);
  if (!in) throw HostError("Could not open configuration file " + conf_path);
  const size_t slash = conf_path.find_last_of('/');
  base_dir_ = slash == std::string::npos ? "" : conf_path.substr(0, slash + 1);
  std::string line;
  int no = 1;
  while (std::getline(in, line)) {
    execute_line(line, no);
    no++;
  }
}

void Samos::execute_line(const std::string& raw, int line_no) {
  const std::string line = trim(raw);
  if (line.empty() || line[0] == '#') return;
  std::string cmd, rest, type, ptext;
  split_command(line, cmd, rest);
  Params p;
  auto params_of = [&](const std::string& text, const char* what) {
    if (!parse_params(text.empty() ? "{}" : text, p))
      throw HostError(std::string("Error parsing ") + what + " parameters at line " + std::to_string(line_no) + ".");
  };
  auto typed = [&](const char* what) {
    if (!split_type_params(rest, type, ptext))
      throw HostError(std::string("Error parsing ") + what + " command at line " + std::to_string(line_no) + ".");
    params_of(ptext, what);
  };

  if (cmd == "messages") {
    return;  // host messages go to stderr here
  } else if (cmd == "config") {  // the JSON record of parameters (samos.cpp, Messenger): not written here
    if (!opt_.quiet) std::fprintf(stderr, "config: the parameter record is not written by the GPU host.\n");
    return;
  } else if (cmd == "box") {  // samos.cpp:186-230
    typed("box");
    if (type == "periodic") periodic_ = true;
    else if (type == "fixed") periodic_ = false;
    else throw HostError("Unknown box type.");
    lx_ = p.count("lx") ? to_dbl(p["lx"], "box") : 10.0;  // DEFAULT_LX (defaults.hpp:36-38)
    ly_ = p.count("ly") ? to_dbl(p["ly"], "box") : 10.0;
    lz_ = p.count("lz") ? to_dbl(p["lz"], "box") : 10.0;
    has_box_ = true;
  } else if (cmd == "input") {  // samos.cpp:240-265
    if (!has_box_) throw HostError("Simulation box not defined.");
    const std::string name = trim(rest);
    parts_ = read_particles(name.size() && name[0] == '/' ? name : base_dir_ + name);
    has_input_ = true;
    ensure_engine();
  } else if (cmd == "nlist") {  // samos.cpp:540-560
    need_system("creating neighbour list");
    params_of(rest, "neighbour list");
    nl_rcut_ = p.count("rcut") ? to_dbl(p["rcut"], "nlist") : 3.0;  // DEFAULT_CUTOFF / DEFAULT_PADDING
    nl_pad_ = p.count("pad") ? to_dbl(p["pad"], "nlist") : 0.5;
    has_nlist_ = true;
    if (h_) check(sg_set_nlist(h_, nl_rcut_, nl_pad_), "sg_set_nlist");
  } else if (cmd == "constraint") {  // samos.cpp:498-530
    need_system("adding constraint");
    typed("constraint");
    ConstraintSpec c = resolve_constraint(type, p);
    constraints_.push_back(c);
    if (h_) check(sg_add_constraint(h_, c.kind, c.params), "sg_add_constraint");
  } else if (cmd == "pair_potential") {  // samos.cpp:332-380
    need_system("adding pair potential");
    typed("pair potential");
    if (!has_nlist_) {  // samos.cpp:347-352: a default neighbour list
      nl_rcut_ = 3.0; nl_pad_ = 0.5; has_nlist_ = true;
      if (h_) check(sg_set_nlist(h_, nl_rcut_, nl_pad_), "sg_set_nlist");
    }
    pairs_[type] = resolve_pair(type, p, parts_.ntypes, nl_rcut_);
  } else if (cmd == "pair_param") {
    if (pairs_.empty()) throw HostError("No pair potentials defined.");
    typed("pair parameters");
    auto it = pairs_.find(type);
    if (it == pairs_.end()) throw HostError("Pair potential " + type + " has not been defined.");
    apply_pair_param(it->second, p, parts_.ntypes);
  } else if (cmd == "pair_align") {
    need_system("adding pair alignment");
    typed("pair alignment");
    if (!has_nlist_) {
      nl_rcut_ = 3.0; nl_pad_ = 0.5; has_nlist_ = true;
      if (h_) check(sg_set_nlist(h_, nl_rcut_, nl_pad_), "sg_set_nlist");
    }
    aligns_[type] = resolve_align(type, p, parts_.ntypes, nl_rcut_);
  } else if (cmd == "align_param") {
    if (aligns_.empty()) throw HostError("No pair alignment defined.");
    typed("alignment parameters");
    auto it = aligns_.find(type);
    if (it == aligns_.end()) throw HostError("Pair alignment " + type + " has not been defined.");
    apply_align_param(it->second, p, parts_.ntypes);
  } else if (cmd == "external") {
    need_system("adding external potential");
    typed("external potential");
    externals_[type] = resolve_external(type, p, parts_.ntypes);
  } else if (cmd == "external_param") {
    typed("external potential parameters");
    auto it = externals_.find(type);
    if (it == externals_.end()) throw HostError("External potential " + type + " has not been defined.");
    apply_external_param(it->second, p, parts_.ntypes);
  } else if (cmd == "timestep") {  // samos.cpp:1332-1350
    need_system("setting the integrator time step");
    dt_ = to_dbl(trim(rest), "timestep");
    if (h_) check(sg_set_timestep(h_, dt_), "sg_set_timestep");
  } else if (cmd == "integrator") {  // samos.cpp:640-700
    need_system("adding integrator");
    if (constraints_.empty()) throw HostError("Constraint not defined.");
    typed("integrator");
    const std::string key = type + "_" + (p.count("group") ? p["group"] : std::string("all"));
    if (integrators_.count(key))
      throw HostError("Integrator of type " + type + " (for group " + key.substr(type.size() + 1) +
                      ") already exists. You need to disable the old one first.");
    IntegratorSpec s = resolve_integrator(type, p, dt_);
    int group = 0;
    if (s.group != "all") {
      auto g = groups_.find(s.group);
      if (g == groups_.end()) throw HostError("Group " + s.group + " is not defined.");
      group = g->second;
    }
    integrators_[key] = s;
    int pos = 0;
    for (const auto& kv : integrators_) {
      if (kv.first == key) break;
      pos++;
    }
    committed_integ_.insert(committed_integ_.begin() + pos, key);
    if (h_) check(sg_insert_integrator(h_, pos, s.kind, s.params, s.temperature), "sg_insert_integrator");
    if (h_ && group) check(sg_set_integrator_group(h_, pos, group), "sg_set_integrator_group");
  } else if (cmd == "disable") {  // samos.cpp:1143-1180
    if (integrators_.empty()) throw HostError("Integrator not defined.");
    typed("disable");
    const std::string key = type + "_" + (p.count("group") ? p["group"] : std::string("all"));
    auto it = integrators_.find(key);
    if (it == integrators_.end()) throw HostError("Trying to disable non-existent integrator.");
    int pos = 0;
    for (const auto& k : committed_integ_) {
      if (k == key) break;
      pos++;
    }
    integrators_.erase(it);
    committed_integ_.erase(committed_integ_.begin() + pos);
    if (h_) check(sg_disable_integrator(h_, pos), "sg_disable_integrator");
  } else if (cmd == "run") {  // samos.cpp:837-972
    need_system("running");
    if (constraints_.empty()) throw HostError("Constraint not defined.");
    if (integrators_.empty()) throw HostError("Integrator not defined.");
    cmd_run(to_i64(trim(rest), "run"));
  } else if (cmd == "dump") {
    need_system("adding dumps");
    cmd_dump(rest);
  } else if (cmd == "log") {
    need_system("adding logs");
    cmd_log(rest);
  } else if (cmd == "group") {  // samos.cpp:1108-1140, System::make_group (system.cpp:462-572)
    need_system("adding any particle groups");
    typed("group");
    cmd_group(type, p);
  } else {
    throw HostError("Command " + cmd + " (line " + std::to_string(line_no) + ") is not part of the GPU path.");
  }
}

void Samos::commit_forces() {
  if (!h_) return;
  check(sg_clear_forces(h_), "sg_clear_forces");
  for (const auto& kv : pairs_) {
    const PairSpec& s = kv.second;
    check(sg_add_pair(h_, s.kind, s.glob, s.table.data(), s.use_radii, s.phase_in, s.shifted, s.has_pair_params,
                      s.phase_value),
          "sg_add_pair");
  }
  for (const auto& kv : aligns_) {
    const AlignSpec& s = kv.second;
    check(sg_add_align(h_, s.kind, s.J, s.rcut, s.table.data(), s.has_pair_params), "sg_add_align");
  }
  for (const auto& kv : externals_) {
    const ExternalSpec& s = kv.second;
    check(sg_add_external(h_, s.kind, s.alpha, s.type_alpha.data(), s.has_params), "sg_add_external");
  }
}

void Samos::cmd_run(int64_t steps) {
  if (!opt_.quiet) std::fprintf(stderr, "Starting simulation run for %lld steps.\n", (long long)steps);
  if (opt_.check_only) { steps_run_ += steps + 1; return; }
  commit_forces();
  // Iterations t = 0..steps (samos.cpp:878) with the global step counter
  // time_step = steps_run_ + t.  Dumps and logs act at the top of an
  // iteration (samos.cpp:895-898), so the run is split there: sg_run for the
  // first segment, sg_run_continue for the others (same bits as one sg_run).
  auto next_due = [&](int64_t T) {  // first global step > T with a dump or log
    int64_t best = INT64_MAX;
    for (const auto& d : dumps_) {
      int64_t a = std::max(d.start, T + 1);
      a = (a + d.freq - 1) / d.freq * d.freq;
      best = std::min(best, a);
    }
    for (const auto& l : logs_) best = std::min(best, (T + 1 + l.freq - 1) / l.freq * l.freq);
    return best;
  };
  auto due = [&](int64_t T) { return next_due(T - 1) == T; };
  const int64_t total = steps + 1;
  int64_t t = 0, builds = 0;
  double ms = 0.0;
  bool started = false;
  while (t < total) {
    if (due(steps_run_)) report(steps_run_);
    const int64_t nd = next_due(steps_run_);
    const int64_t len = std::min(total - t, nd - steps_run_);
    sg_run_stats st{};
    if (!started) check(sg_run(h_, len - 1, &st), "sg_run");
    else check(sg_run_continue(h_, len, &st), "sg_run_continue");
    started = true;
    builds += st.nlist_builds;
    ms += st.device_ms;
    steps_run_ += len;
    t += len;
  }
  if (!opt_.quiet)
    std::fprintf(stderr, "Run of %lld steps done: %lld neighbour-list builds, %.3f ms on the device.\n",
                 (long long)total, (long long)builds, ms);
}

// Members: the particles meeting every given criterion on the state at this
// command, in index order.
void Samos::cmd_group(const std::string& name, const Params& p) {
  if (name == "boundary" || name == "tissue")
    throw HostError("Groups \"tissue\" and \"boundary\" are reserved and cannot be used.");
  if (groups_.count(name))
    throw HostError("Group " + name + " is already defined (adding to a group is not part of the GPU path).");
  if (groups_.size() >= 7) throw HostError("More than 7 particle groups are not part of the GPU path.");
  static const std::set<std::string> crit = {"type", "not_type", "r_eq", "r_le", "r_ge", "x_le",
                                             "x_ge", "y_le", "y_ge", "z_le", "z_ge"};
  bool positions = false;
  for (const auto& kv : p) {
    if (!crit.count(kv.first)) throw HostError("Group criterion " + kv.first + " is not part of the GPU path.");
    positions = positions || kv.first[0] == 'x' || kv.first[0] == 'y' || kv.first[0] == 'z';
  }
  if (positions && h_) {  // the current positions, not the input's
    check(sg_download(h_, 0, "x", parts_.x.data()), "sg_download");
    check(sg_download(h_, 0, "y", parts_.y.data()), "sg_download");
    check(sg_download(h_, 0, "z", parts_.z.data()), "sg_download");
  }
  std::vector<uint8_t> member(parts_.size(), 1);
  for (const auto& kv : p) {
    const std::string& k = kv.first;
    for (size_t i = 0; i < parts_.size(); i++) {
      bool ok = true;
      if (k == "type") ok = parts_.type[i] == (int)to_i64(kv.second, "group");
      else if (k == "not_type") ok = parts_.type[i] != (int)to_i64(kv.second, "group");
      else {
        const double v = to_dbl(kv.second, "group");
        const double q = k[0] == 'r' ? parts_.radius[i] : k[0] == 'x' ? parts_.x[i] : k[0] == 'y' ? parts_.y[i] : parts_.z[i];
        const std::string op = k.substr(2);
        ok = op == "eq" ? q == v : op == "le" ? q <= v : q >= v;
      }
      member[i] = member[i] && ok;
    }
  }
  const int idx = (int)groups_.size() + 1;
  groups_[name] = idx;
  if (h_) check(sg_define_group(h_, 0, idx, member.data()), "sg_define_group");
}

void Samos::cmd_dump(const std::string& rest) {
  std::string name, ptext;
  if (!split_type_params(rest, name, ptext, true)) throw HostError("Error parsing dump command.");
  Params p;
  if (!parse_params(ptext, p)) throw HostError("Error parsing dump parameters.");
  dumps_.push_back(make_dump(name, p, (int32_t)parts_.size()));
}

// Logger ctor (logger.cpp:40-124): `step` always first, then every
// parameter key other than freq (std::map order) naming a quantity; freq
// defaults to 100; the header names the file, the time and the columns.
void Samos::cmd_log(const std::string& rest) {
  std::string name, ptext;
  if (!split_type_params(rest, name, ptext, true)) throw HostError("Error parsing log command.");
  Params p;
  if (!parse_params(ptext, p)) throw HostError("Error parsing log parameters.");
  Log l;
  l.name = name;
  l.freq = p.count("freq") ? to_i64(p["freq"], "log") : 100;
  if (l.freq <= 0) throw HostError("Log frequency has to be positive.");
  static const std::set<std::string> here = {"step", "velocity", "vec_velocity", "kinetic_energy", "size",
                                             "soft_energy", "lj_energy", "morse_energy", "gaussian_energy",
                                             "polar_align", "nematic_align"};
  static const std::set<std::string> elsewhere = {
      "soft_attractive_energy", "rod_energy", "ljrod_energy", "vp_energy", "line_tension_energy",
      "boundary_bending_energy", "boundary_attraction_energy", "coulomb_energy", "bare_coulomb_energy",
      "coulomb3_energy", "yukawa_energy", "harmonic_bond_energy", "harmonic_angle_energy", "cosine_angle_energy",
      "external_gravity_energy", "external_harmonic_energy", "area", "avg_perim"};
  l.cols.push_back("step");
  for (const auto& kv : p) {
    std::string q = kv.first;
    for (auto& ch : q) ch = (char)std::tolower((unsigned char)ch);
    if (q == "freq") continue;
    if (here.count(q)) l.cols.push_back(q);
    else if (elsewhere.count(q)) throw HostError("Log quantity " + q + " is not part of the GPU path.");
    else throw HostError("Unknown log quantity : " + q + ".");
  }
  logs_.push_back(l);
  std::FILE* f = std::fopen(l.name.c_str(), "w");
  if (!f) throw HostError("Cannot open log file " + l.name);
  char when[64];
  std::time_t now = std::time(nullptr);
  std::strftime(when, sizeof when, "%Y-%b-%d %H:%M:%S", std::localtime(&now));
  std::fprintf(f, "# Log file : %s\n# Generated on : %s\n# ", l.name.c_str(), when);
  for (size_t i = 0; i < l.cols.size(); i++) std::fprintf(f, "(%zu) %s ", i + 1, l.cols[i].c_str());
  std::fprintf(f, "\n");
  std::fclose(f);
}

void Samos::report(int64_t step) {
  check(sg_begin_step(h_), "sg_begin_step");
  bool energies = false;
  for (const auto& l : logs_)
    if (step % l.freq == 0)
      for (const auto& c : l.cols)
        energies = energies || c == "soft_energy" || c == "lj_energy" || c == "morse_energy" || c == "gaussian_energy" ||
                   c == "polar_align" || c == "nematic_align";
  if (energies) check(sg_compute(h_, dt_), "sg_compute");
  auto down = [&](const char* f, void* p) { check(sg_download(h_, 0, f, p), "sg_download"); };
  down("x", parts_.x.data()); down("y", parts_.y.data()); down("z", parts_.z.data());
  down("vx", parts_.vx.data()); down("vy", parts_.vy.data()); down("vz", parts_.vz.data());
  down("nx", parts_.nx.data()); down("ny", parts_.ny.data()); down("nz", parts_.nz.data());
  down("omega", parts_.omega.data());
  down("ix", parts_.ix.data()); down("iy", parts_.iy.data()); down("iz", parts_.iz.data());
  DumpState ds;
  ds.parts = &parts_;
  ds.lx = lx_; ds.ly = ly_; ds.lz = lz_;
  std::vector<double> F[3], N[3];
  std::vector<int32_t> coord;
  for (const auto& d : dumps_) {
    if (!dump_due(d, step)) continue;
    if (d.type == "vtp" && coord.empty()) {
      coord.resize(parts_.size());
      check(sg_coordination(h_, 0, coord.data()), "sg_coordination");
    }
    if (((d.type == "full" && d.p.count("force")) || d.type == "vtp") && F[0].empty()) {
      const char* names[3] = {"fx", "fy", "fz"};
      for (int c = 0; c < 3; c++) { F[c].resize(parts_.size()); down(names[c], F[c].data()); }
    }
    if (d.type == "full" && d.p.count("normal") && N[0].empty()) {
      const char* names[3] = {"Nx", "Ny", "Nz"};
      for (int c = 0; c < 3; c++) { N[c].resize(parts_.size()); down(names[c], N[c].data()); }
    }
    ds.fx = &F[0]; ds.fy = &F[1]; ds.fz = &F[2];
    ds.Nx = &N[0]; ds.Ny = &N[1]; ds.Nz = &N[2];
    ds.coordination = &coord;
    write_dump(d, step, ds);
  }
  for (const auto& l : logs_) {  // Logger::log (logger.cpp:128-139): each column then a space
    if (step % l.freq) continue;
    std::FILE* f = std::fopen(l.name.c_str(), "a");
    if (!f) throw HostError("Cannot open log file " + l.name);
    const double N = (double)parts_.size();
    for (const auto& c : l.cols) {
      if (c == "step") { std::fprintf(f, "%8lld  ", (long long)step); continue; }       // log_step.hpp:55
      if (c == "size") { std::fprintf(f, "%6lld  ", (long long)parts_.size()); continue; }  // log_size.hpp:55
      double v = 0.0;
      if (c == "velocity") {  // log_velocity.hpp:56-65: mean speed
        for (size_t i = 0; i < parts_.size(); i++)
          v += std::sqrt(parts_.vx[i] * parts_.vx[i] + parts_.vy[i] * parts_.vy[i] + parts_.vz[i] * parts_.vz[i]);
        v /= N;
      } else if (c == "vec_velocity") {  // log_vec_velocity.hpp:56-68: |sum v| / N
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (size_t i = 0; i < parts_.size(); i++) { sx += parts_.vx[i]; sy += parts_.vy[i]; sz += parts_.vz[i]; }
        v = std::sqrt(sx * sx + sy * sy + sz * sz) / N;
      } else if (c == "kinetic_energy") {  // log_kinetic_eng.hpp:56-66: sum v^2 / (2 m), / N
        for (size_t i = 0; i < parts_.size(); i++) {
          const double v2 = parts_.vx[i] * parts_.vx[i] + parts_.vy[i] * parts_.vy[i] + parts_.vz[i] * parts_.vz[i];
          v += 0.5 * v2 / parts_.mass[i];
        }
        v /= N;
      } else {  // the term's total energy from the last force evaluation (log_pair_eng.hpp, log_pair_align.hpp)
        const bool align = c == "polar_align" || c == "nematic_align";
        const std::string want = c.substr(0, c.find('_'));
        int comp = 0;
        bool found = false;
        if (align) {
          for (const auto& kv : aligns_) { if (kv.first == want) { found = true; break; } comp++; }
        } else {
          for (const auto& kv : pairs_) { if (kv.first == want) { found = true; break; } comp++; }
        }
        if (!found)
          throw HostError(std::string(align ? "Pair alignment" : "Pair potential") + " of type " + want + " not defined.");
        check(sg_energy(h_, 0, align ? 1 : 0, comp, &v), "sg_energy");
      }
      std::fprintf(f, "%12.6e  ", v);
    }
    std::fprintf(f, "\n");
    std::fclose(f);
  }
}

std::string Samos::describe() const {
  std::ostringstream o;
  o << "particles " << parts_.size() << " ntypes " << parts_.ntypes << "\n";
  o << "box " << (periodic_ ? "periodic" : "fixed") << " " << lx_ << " " << ly_ << " " << lz_ << "\n";
  if (has_nlist_) o << "nlist " << nl_rcut_ << " " << nl_pad_ << "\n";
  for (const auto& c : constraints_) o << "constraint " << c.kind << " " << c.params[0] << "\n";
  for (const auto& kv : pairs_) {
    o << "pair " << kv.first << " " << kv.second.kind;
    for (int i = 0; i < SG_PAIR_NPARAM; i++) o << " " << kv.second.glob[i];
    o << " radii " << kv.second.use_radii << "\n";
  }
  for (const auto& kv : aligns_) o << "align " << kv.first << " " << kv.second.J << " " << kv.second.rcut << "\n";
  for (const auto& kv : externals_) o << "external " << kv.first << " " << kv.second.alpha << "\n";
  for (const auto& key : committed_integ_) {
    const IntegratorSpec& s = integrators_.at(key);
    o << "integrator " << key << " " << s.kind;
    for (int i = 0; i < 12; i++) o << " " << s.params[i];
    o << "\n";
  }
  o << "steps " << steps_run_ << "\n";
  return o.str();
}

}  // namespace samos_host
