// plugins.cpp -- the plugin constructors of the hot path, restated: factory
// names (src/utils/register_*.cpp), parameter keys, defaults, the
// known-parameter checks (PairPotential::params_ok, pair_potential.hpp:123-129)
// and the per-type tables, producing the numeric vectors of the C ABI.
#include <algorithm>
#include <cstdlib>

#include "samos_host.hpp"

namespace samos_host {

namespace {

double to_double(const std::string& key, const std::string& v) {
  char* end = nullptr;
  const double d = std::strtod(v.c_str(), &end);
  if (v.empty() || *end != '\0') throw HostError("Parameter " + key + " = \"" + v + "\" is not a number.");
  return d;
}
int to_int(const std::string& key, const std::string& v) {
  char* end = nullptr;
  const long l = std::strtol(v.c_str(), &end, 10);
  if (v.empty() || *end != '\0') throw HostError("Parameter " + key + " = \"" + v + "\" is not an integer.");
  return (int)l;
}
double get(const Params& p, const std::string& key, double def) {
  auto it = p.find(key);
  return it == p.end() ? def : to_double(key, it->second);
}
bool has(const Params& p, const std::string& key) { return p.count(key) != 0; }

void known(const Params& p, std::vector<std::string> keys, const std::string& what) {
  for (const auto& kv : p)
    if (std::find(keys.begin(), keys.end(), kv.first) == keys.end())
      throw HostError("Unknown parameter \"" + kv.first + "\" in " + what + ".");
}

// Value object (src/system/value.hpp:59-178): {kind, min_val, max_val, steps}
void value_of(const std::string& kind, const Params& p, double out[4]) {
  if (kind != "constant" && kind != "linear") throw HostError("Unknown value type " + kind + ".");
  const double vmin = get(p, "min_val", 0.0), vmax = get(p, "max_val", 1.0);
  const int steps = has(p, "steps") ? to_int("steps", p.at("steps")) : 1000;
  if (kind == "linear") {
    if (vmax < vmin) throw HostError("Value parameters are not properly set.");
    if (steps <= 0) throw HostError("Value parameters. Zero steps given.");
  }
  out[0] = kind == "constant" ? SG_VALUE_CONSTANT : SG_VALUE_LINEAR;
  out[1] = vmin; out[2] = vmax; out[3] = steps;
}

int type_index(const Params& p, const char* key, int ntypes) {
  const int t = to_int(key, p.at(key));
  if (t < 1 || t > ntypes) throw HostError(std::string(key) + " outside 1..ntypes.");
  return t - 1;
}

const std::vector<std::string> kPairBase = {"min_val", "max_val", "ntypes", "steps"};
const std::vector<std::string> kIntBase = {"dt", "group", "temperature_control", "min_val", "max_val", "steps"};
const double kWcaFactor = 1.122462048309373;  // 2^(1/6), pair_lj_potential.hpp

std::vector<std::string> plus(std::vector<std::string> a, std::initializer_list<const char*> b) {
  for (const char* s : b) a.emplace_back(s);
  return a;
}

const std::vector<std::string>& table_keys(const std::string& name) {
  static const std::map<std::string, std::vector<std::string>> k = {
      {"soft", {"k", "a"}},
      {"lj", {"epsilon", "sigma", "rcut"}},
      {"morse", {"D", "a", "re", "rcut"}},
      {"gaussian", {"A", "B", "alpha", "beta", "rA", "rB", "rcut"}}};
  return k.at(name);
}

}  // namespace

PairSpec resolve_pair(const std::string& name, const Params& p, int ntypes, double nlist_rcut) {
  (void)nlist_rcut;
  PairSpec s;
  s.name = name;
  s.use_radii = has(p, "use_particle_radii");
  s.phase_in = has(p, "phase_in");
  s.shifted = has(p, "shifted");
  double* g = s.glob;
  if (name == "soft") {  // pair_soft_potential.hpp:63-121
    known(p, plus(kPairBase, {"k", "a", "use_particle_radii", "phase_in"}), "soft potential");
    s.kind = SG_PAIR_SOFT;
    g[0] = get(p, "k", 1.0); g[1] = get(p, "a", 2.0);
    s.shifted = false;
  } else if (name == "lj") {  // pair_lj_potential.hpp:61-159
    known(p, plus(kPairBase, {"epsilon", "sigma", "rcut", "use_particle_radii", "phase_in", "shifted", "WCA"}),
          "Lennard-Jones potential");
    s.kind = SG_PAIR_LJ;
    g[0] = get(p, "epsilon", 1.0); g[1] = get(p, "sigma", 1.0); g[2] = get(p, "rcut", 3.0);
    if (has(p, "WCA")) { g[2] = kWcaFactor * g[1]; s.shifted = true; }
  } else if (name == "morse") {  // pair_morse_potential.hpp:61-160
    known(p, plus(kPairBase, {"D", "a", "re", "rcut", "use_particle_radii", "phase_in", "shifted"}), "Morse potential");
    s.kind = SG_PAIR_MORSE;
    g[0] = get(p, "D", 1.0); g[1] = get(p, "a", 1.0); g[2] = get(p, "re", 1.0); g[3] = get(p, "rcut", 2.5 * g[2]);
  } else if (name == "gaussian") {  // pair_gaussian_potential.hpp:66-194 (no params_ok there)
    s.kind = SG_PAIR_GAUSSIAN;
    g[0] = get(p, "A", 2.0); g[1] = get(p, "B", -1.0); g[2] = get(p, "alpha", 1.0); g[3] = get(p, "beta", 3.0);
    g[4] = get(p, "rA", 0.0); g[5] = get(p, "rB", 1.5); g[6] = get(p, "rcut", 3.0);
  } else {
    throw HostError("Unknown pair potential " + name + ".");
  }
  if (has(p, "ntypes")) ntypes = std::max(ntypes, to_int("ntypes", p.at("ntypes")));
  s.table.assign((size_t)ntypes * ntypes * SG_PAIR_NPARAM, 0.0);
  for (int a = 0; a < ntypes * ntypes; a++)
    for (int i = 0; i < SG_PAIR_NPARAM; i++) s.table[(size_t)a * SG_PAIR_NPARAM + i] = g[i];
  if (name == "gaussian")  // per-type default B = A (pair_gaussian_potential.hpp:174)
    for (int a = 0; a < ntypes * ntypes; a++) s.table[(size_t)a * SG_PAIR_NPARAM + 1] = g[0];
  if (s.phase_in) {
    const std::string kind = p.at("phase_in").empty() ? "constant" : p.at("phase_in");
    value_of(kind, p, s.phase_value);
  }
  return s;
}

void apply_pair_param(PairSpec& s, const Params& p, int ntypes) {
  if (!has(p, "type_1") || !has(p, "type_2")) throw HostError("Missing key for pair potential parameters.");
  const int t1 = type_index(p, "type_1", ntypes), t2 = type_index(p, "type_2", ntypes);
  const auto& keys = table_keys(s.name);
  for (size_t slot = 0; slot < keys.size(); slot++) {
    double v = get(p, keys[slot], s.glob[slot]);
    if (s.name == "lj" && keys[slot] == "rcut" && has(p, "WCA")) {
      v = kWcaFactor * get(p, "sigma", s.glob[1]);
      s.shifted = true;
    }
    s.table[((size_t)t1 * ntypes + t2) * SG_PAIR_NPARAM + slot] = v;
    s.table[((size_t)t2 * ntypes + t1) * SG_PAIR_NPARAM + slot] = v;
  }
  s.has_pair_params = true;
}

AlignSpec resolve_align(const std::string& name, const Params& p, int ntypes, double nlist_rcut) {
  AlignSpec s;
  s.name = name;
  if (name == "polar") s.kind = SG_ALIGN_POLAR;
  else if (name == "nematic") s.kind = SG_ALIGN_NEMATIC;
  else if (name == "vicsek") s.kind = SG_ALIGN_VICSEK;
  else throw HostError("Unknown pair aligner " + name + ".");
  if (has(p, "exclude_boundary")) throw HostError("exclude_boundary (tissue boundaries) is not part of the GPU path.");
  s.J = name == "vicsek" ? 0.0 : get(p, "J", 1.0);
  s.rcut = get(p, "rcut", nlist_rcut);  // pair_polar_aligner.hpp:80-84
  s.table.assign((size_t)ntypes * ntypes * 2, 0.0);
  for (int a = 0; a < ntypes * ntypes; a++) { s.table[2 * a] = s.J; s.table[2 * a + 1] = s.rcut; }
  return s;
}

void apply_align_param(AlignSpec& s, const Params& p, int ntypes) {
  if (s.name == "vicsek") return;  // pair_vicsek_aligner.hpp:69-72 ignores per-pair parameters
  if (!has(p, "type_1") || !has(p, "type_2")) throw HostError("Missing key for pair alignment parameters.");
  const int t1 = type_index(p, "type_1", ntypes), t2 = type_index(p, "type_2", ntypes);
  const double J = get(p, "J", s.J), rc = get(p, "rcut", s.rcut);
  for (const auto& ab : {std::make_pair(t1, t2), std::make_pair(t2, t1)}) {
    s.table[((size_t)ab.first * ntypes + ab.second) * 2] = J;
    s.table[((size_t)ab.first * ntypes + ab.second) * 2 + 1] = rc;
  }
  s.has_pair_params = true;
}

ExternalSpec resolve_external(const std::string& name, const Params& p, int ntypes) {
  if (name != "self_propulsion") throw HostError("External potential " + name + " is not part of the GPU path.");
  ExternalSpec s;  // external_self_propulsion.hpp:51-63
  s.name = name;
  s.kind = SG_EXT_SELF_PROPULSION;
  s.alpha = get(p, "alpha", 1.0);
  s.type_alpha.assign(ntypes, s.alpha);
  return s;
}

void apply_external_param(ExternalSpec& s, const Params& p, int ntypes) {
  if (!has(p, "type")) throw HostError("Missing type for external potential parameters.");
  const int t = type_index(p, "type", ntypes);
  s.type_alpha[t] = get(p, "alpha", s.alpha);
  s.has_params = true;
}

ConstraintSpec resolve_constraint(const std::string& name, const Params& p) {
  ConstraintSpec s;
  if (name == "none") s.kind = SG_CONS_NONE;
  else if (name == "plane") s.kind = SG_CONS_PLANE;
  else if (name == "sphere") s.kind = SG_CONS_SPHERE;
  else if (name == "cylinder") s.kind = SG_CONS_CYLINDER;
  else if (name == "torus") s.kind = SG_CONS_TORUS;
  else if (name == "ellipsoid") s.kind = SG_CONS_ELLIPSOID;
  else if (name == "peanut") s.kind = SG_CONS_PEANUT;
  else if (name == "gyroid") s.kind = SG_CONS_GYROID;
  else if (name == "hourglass") s.kind = SG_CONS_HOURGLASS;
  else if (name == "gaussian_bump") s.kind = SG_CONS_GAUSSIAN_BUMP;
  else if (name == "slab") s.kind = SG_CONS_SLAB;
  else if (name == "walls") s.kind = SG_CONS_PLANE_WALLS;
  else if (name == "tetrahedron") s.kind = SG_CONS_TETRAHEDRON;
  else throw HostError("Constraint " + name + " is not part of the GPU path.");
  if (has(p, "group") && p.at("group") != "all") throw HostError("Constraint groups other than 'all' are not part of the GPU path.");
  // Constraint base (constraint.hpp:56-120); tol is parsed as an int there (82)
  const double maxiter = has(p, "maxiter") ? to_int("maxiter", p.at("maxiter")) : 100.0;
  const double tol = has(p, "tol") ? (double)to_int("tol", p.at("tol")) : 1e-6;
  double first = 0.0, unlimited = 0.0, second = 0.0, third = 0.0;
  if (name == "plane") { first = get(p, "zpos", 0.0); unlimited = has(p, "unlimited") ? 1.0 : 0.0; }
  else if (name == "sphere" || name == "cylinder") first = get(p, "r", 1.0);
  else if (name == "torus") { first = get(p, "c", 1.0); second = get(p, "a", 0.5); }  // constraint_torus.hpp
  else if (name == "ellipsoid") { first = get(p, "a", 1.0); second = get(p, "b", 1.0); third = get(p, "c", 1.0); }
  else if (name == "peanut") {  // constraint_peanut.hpp:62-88
    first = get(p, "a", 10.0); second = get(p, "b", 8.0);
    if (second <= first)
      throw HostError("Parameter b has to be larger than parameter a. Otherwise the surface will be disconnected.");
  } else if (name == "hourglass") {  // constraint_hourglass.hpp:64-102 (A checked only when given)
    first = get(p, "R", 10.0); second = get(p, "A", 1.0); third = get(p, "n", 1.0);
    if (has(p, "A") && second > first) throw HostError("Hourglass constraint. Amplitude has to be smaller than the radius.");
  } else if (name == "gaussian_bump") {  // constraint_gaussian_bump.hpp: the widths a, b are stored squared
    first = get(p, "A", 1.0); second = get(p, "a", 1.0); third = get(p, "b", 1.0);
    second *= second;
    third *= third;
  } else if (name == "slab") {  // constraint_slab.hpp:56-78
    first = get(p, "z_lo", 0.0); second = get(p, "z_hi", 1.0);
  } else if (name == "walls") {  // constraint_plane_walls.hpp:56-74 (the engine moves l to the box edge)
    first = get(p, "l", 1.0);
  } else if (name == "tetrahedron") {  // constraint_tetrahedron.hpp:62-88
    first = get(p, "scale", 10.0); second = get(p, "value", 1.0);
  }
  const double v[9] = {first, unlimited, maxiter, tol, get(p, "rescale", 1.0), get(p, "rescale_steps", 1000.0),
                       get(p, "rescale_freq", 10.0), second, third};
  for (int i = 0; i < 9; i++) s.params[i] = v[i];
  return s;
}

IntegratorSpec resolve_integrator(const std::string& name, const Params& p, double dt_global) {
  IntegratorSpec s;
  s.name = name;
  double* q = s.params;
  const double dt = get(p, "dt", dt_global);
  if (!(dt > 0.0)) throw HostError("Integrator step has not been set.");
  s.group = has(p, "group") ? p.at("group") : std::string("all");
  q[0] = dt;
  auto seed = [&]() { return has(p, "seed") ? (double)to_int("seed", p.at("seed")) : 0.0; };
  if (name == "brownian") {  // integrator_brownian.hpp:55-160
    known(p, plus(kIntBase, {"v0", "nu", "mu", "mur", "seed", "nematic", "tau", "velocity_align"}), "brownian integrator");
    s.kind = SG_INT_BROWNIAN;
    q[1] = get(p, "v0", 1.0); q[2] = get(p, "nu", 1.0); q[3] = get(p, "mu", 1.0); q[4] = get(p, "mur", 1.0);
    q[5] = seed(); q[6] = has(p, "nematic") ? 1.0 : 0.0; q[7] = get(p, "tau", 1.0);
    q[8] = has(p, "velocity_align") ? 1.0 : 0.0;
  } else if (name == "brownian_pos") {  // integrator_brownian_pos.hpp:55-90
    known(p, plus(kIntBase, {"mu", "seed"}), "brownian_pos integrator");
    s.kind = SG_INT_BROWNIAN_POS;
    q[3] = get(p, "mu", 1.0); q[5] = seed();
  } else if (name == "brownian_align") {  // integrator_brownian_align.hpp:55-127
    known(p, plus(kIntBase, {"nu", "mur", "seed", "nematic", "tau"}), "brownian_align integrator");
    s.kind = SG_INT_BROWNIAN_ALIGN;
    q[2] = get(p, "nu", 1.0); q[4] = get(p, "mur", 1.0); q[5] = seed();
    q[6] = has(p, "nematic") ? 1.0 : 0.0; q[7] = get(p, "tau", 1.0);
  } else if (name == "langevin") {  // integrator_langevin.hpp:64-116
    known(p, plus(kIntBase, {"gamma", "seed", "method"}), "langevin integrator");
    s.kind = SG_INT_LANGEVIN;
    q[5] = seed(); q[9] = get(p, "gamma", 1.0);
    std::string m = has(p, "method") ? p.at("method") : "baoab";
    std::transform(m.begin(), m.end(), m.begin(), ::tolower);
    if (m == "baoab") q[10] = 0; else if (m == "spv") q[10] = 1; else if (m == "bbk") q[10] = 2;
    else throw HostError("Unknown integration method");
  } else if (name == "fire") {  // integrator_fire.hpp:58-154 (no params_ok there)
    s.kind = SG_INT_FIRE;
    q[1] = get(p, "alpha", 0.1); q[2] = get(p, "alpha_scale", 0.99);
    q[3] = get(p, "f_tolerance", 1e-4); q[4] = get(p, "e_tolerance", 1e-6);
    q[6] = get(p, "dt_inc", 1.1); q[7] = get(p, "dt_dec", 0.5); q[8] = get(p, "dt_max", 1.0);
    q[9] = has(p, "min_neg_steps") ? (double)to_int("min_neg_steps", p.at("min_neg_steps")) : 5.0;
    q[11] = get(p, "fmax_tolerance", 0.0);
  } else if (name == "vicsek") {  // integrator_vicsek.hpp:55-105 (no params_ok there)
    s.kind = SG_INT_VICSEK;
    q[1] = get(p, "v0", 1.0); q[2] = get(p, "eta", 0.1); q[3] = get(p, "mu", 0.0); q[5] = seed();
  } else if (name == "nve") {  // integrator_nve.hpp:59-75 (no params_ok there)
    s.kind = SG_INT_NVE;
    if (has(p, "limit")) { q[12] = 1.0; q[13] = get(p, "limit", 0.0); }
    if (has(p, "angle_limit")) { q[14] = 1.0; q[15] = get(p, "angle_limit", 0.0); }
  } else {
    throw HostError("Integrator " + name + " is not part of the GPU path.");
  }
  value_of(has(p, "temperature_control") ? p.at("temperature_control") : "constant", p, s.temperature);
  return s;
}

}  // namespace samos_host
