// ref_driver.cpp -- C entry points over SAMoS's OWN hot-path classes.
//
// TEST INFRASTRUCTURE ONLY.  oracle/build_ref.sh compiles this file together
// with the reference's unmodified sources (src/system, src/potentials,
// src/aligner, src/constraints, src/integrators, src/utils/rng.cpp,
// src/messenger) into oracle/_ref/.  It is the pin for the CPU oracle
// (oracle/samos_oracle.c) and the timed reference CPU baseline.  Only
// tests/, bench.py's reference arm and cpu_baseline leg load it.
//
// Each rs_* call performs what one conf-file command does in the reference's
// command loop (src/samos.cpp:176-1400), with the parameter block given as
// "key=value;flag;..." text (a flag maps to "", as the reference's
// key_value_sequence grammar makes it).  The plugin objects are the
// reference's own classes, constructed by name the way its class factories
// construct them (src/utils/register_*.cpp).  rs_run is the `run` command's
// loop (src/samos.cpp:864-972) without dumps, logs and populations.
//
// Noise: gsl/gsl_rng.h in oracle/ref_shim makes RNG draw the project's
// counter-based stream, so the reference's integrators consume the same
// noise as the oracle and the CUDA path.

#include <cstring>
#include <exception>
#include <functional>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "aligner.hpp"
#include "box.hpp"
#include "constrainer.hpp"
#include "constraint_cylinder.hpp"
#include "constraint_ellipsoid.hpp"
#include "constraint_gaussian_bump.hpp"
#include "constraint_gyroid.hpp"
#include "constraint_hourglass.hpp"
#include "constraint_none.hpp"
#include "constraint_peanut.hpp"
#include "constraint_plane.hpp"
#include "constraint_plane_walls.hpp"
#include "constraint_slab.hpp"
#include "constraint_sphere.hpp"
#include "constraint_tetrahedron.hpp"
#include "constraint_torus.hpp"
#include "external_self_propulsion.hpp"
#include "integrator_brownian.hpp"
#include "integrator_brownian_align.hpp"
#include "integrator_brownian_pos.hpp"
#include "integrator_fire.hpp"
#include "integrator_langevin.hpp"
#include "integrator_nve.hpp"
#include "integrator_vicsek.hpp"
#include "messenger.hpp"
#include "neighbour_list.hpp"
#include "pair_gaussian_potential.hpp"
#include "pair_lj_potential.hpp"
#include "pair_morse_potential.hpp"
#include "pair_nematic_aligner.hpp"
#include "pair_polar_aligner.hpp"
#include "pair_soft_potential.hpp"
#include "pair_vicsek_aligner.hpp"
#include "potential.hpp"
#include "system.hpp"
#include "value.hpp"

namespace {

const double kDefaultCutoff = 3.0;   // src/system/defaults.hpp
const double kDefaultPadding = 0.5;

struct Session {
  MessengerPtr msg;
  BoxPtr box;
  bool periodic = false;
  SystemPtr sys;
  NeighbourListPtr nlist;
  PotentialPtr pot;
  AlignerPtr aligner;
  ConstrainerPtr constraint;
  std::map<std::string, IntegratorPtr> integrator;  // keyed type_group, as samos.cpp keys them
  int time_step = 0;                                // samos.cpp:127
  int nlist_builds = 0;
  std::string error;
};

// "k=10;use_particle_radii" -> {"k": "10", "use_particle_radii": ""}
pairs_type parse_block(const char* text) {
  pairs_type out;
  if (!text) return out;
  std::stringstream ss(text);
  std::string item;
  while (std::getline(ss, item, ';')) {
    if (item.empty()) continue;
    std::size_t eq = item.find('=');
    if (eq == std::string::npos) out[item] = "";
    else out[item.substr(0, eq)] = item.substr(eq + 1);
  }
  return out;
}

ValuePtr make_value(const std::string& kind, MessengerPtr msg, pairs_type& p) {
  if (kind == "constant") return std::make_shared<ValueConstant>(msg, p);
  if (kind == "linear") return std::make_shared<ValueLinear>(msg, p);
  throw std::runtime_error("unknown value type " + kind);
}

template <class F>
int guarded(Session* s, F&& f) {
  try {
    f();
    return 0;
  } catch (std::exception& e) {
    s->error = e.what();
  } catch (...) {
    s->error = "unknown exception";
  }
  return -1;
}

void require(bool ok, const char* what) {
  if (!ok) throw std::runtime_error(what);
}

}  // namespace

extern "C" {

void* rs_create(const char* messages) {
  Session* s = new Session();
  s->msg = std::make_shared<Messenger>(std::string(messages && *messages ? messages : "/dev/null"));
  return s;
}

void rs_destroy(void* h) { delete static_cast<Session*>(h); }

const char* rs_error(void* h) { return static_cast<Session*>(h)->error.c_str(); }

// box periodic|fixed {lx; ly; lz}
int rs_box(void* h, double lx, double ly, double lz, int periodic) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    s->box = std::make_shared<Box>(Box(lx, ly, lz));
    s->periodic = periodic != 0;
  });
}

// input <file>: System reads the particle file with its own reader
int rs_input(void* h, const char* path) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    require(s->box != nullptr, "Simulation box not defined.");
    s->sys = std::make_shared<System>(System(std::string(path), s->msg, s->box));
    s->sys->set_periodic(s->periodic);
  });
}

int rs_size(void* h) {
  Session* s = static_cast<Session*>(h);
  return s->sys ? s->sys->size() : 0;
}

// nlist {rcut; pad}
int rs_nlist(void* h, const char* params) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    require(s->sys != nullptr, "System not defined.");
    pairs_type p = parse_block(params);
    double rcut = kDefaultCutoff, pad = kDefaultPadding;
    if (p.count("rcut")) rcut = lexical_cast<double>(p["rcut"]);
    if (p.count("pad")) pad = lexical_cast<double>(p["pad"]);
    s->nlist = std::make_shared<NeighbourList>(NeighbourList(s->sys, s->msg, rcut, pad, p));
  });
}

// constraint <name> {...}: added, then enforced on every particle
int rs_constraint(void* h, const char* name, const char* params) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    require(s->sys != nullptr, "System not defined.");
    pairs_type p = parse_block(params);
    std::string n(name);
    ConstraintPtr c;
    SystemPtr sys = s->sys;
    MessengerPtr msg = s->msg;
    if (n == "sphere") c = std::make_shared<ConstraintSphere>(sys, msg, p);
    else if (n == "plane") c = std::make_shared<ConstraintPlane>(sys, msg, p);
    else if (n == "walls") c = std::make_shared<ConstraintPlaneWalls>(sys, msg, p);
    else if (n == "cylinder") c = std::make_shared<ConstraintCylinder>(sys, msg, p);
    else if (n == "peanut") c = std::make_shared<ConstraintPeanut>(sys, msg, p);
    else if (n == "torus") c = std::make_shared<ConstraintTorus>(sys, msg, p);
    else if (n == "ellipsoid") c = std::make_shared<ConstraintEllipsoid>(sys, msg, p);
    else if (n == "gyroid") c = std::make_shared<ConstraintGyroid>(sys, msg, p);
    else if (n == "hourglass") c = std::make_shared<ConstraintHourglass>(sys, msg, p);
    else if (n == "gaussian_bump") c = std::make_shared<ConstraintGaussianBump>(sys, msg, p);
    else if (n == "none") c = std::make_shared<ConstraintNone>(sys, msg, p);
    else if (n == "tetrahedron") c = std::make_shared<ConstraintTetrahedron>(sys, msg, p);
    else if (n == "slab") c = std::make_shared<ConstraintSlab>(sys, msg, p);
    else throw std::runtime_error("unknown constraint " + n);
    if (!s->constraint) s->constraint = std::make_shared<Constrainer>(Constrainer(sys, msg));
    s->constraint->add_constraint(n, c);
    for (int i = 0; i < sys->size(); i++) s->constraint->enforce(sys->get_particle(i));
  });
}

static void default_nlist(Session* s, pairs_type& p) {
  if (!s->nlist) s->nlist = std::make_shared<NeighbourList>(NeighbourList(s->sys, s->msg, kDefaultCutoff, kDefaultPadding, p));
}

// group <name> {...}: System::make_group on the current state
int rs_group(void* h, const char* name, const char* params) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    require(s->sys != nullptr, "System not defined.");
    pairs_type p = parse_block(params);
    s->sys->make_group(std::string(name), p);
  });
}

// pair_potential <name> {...}
int rs_pair_potential(void* h, const char* name, const char* params) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    require(s->sys != nullptr, "System not defined.");
    pairs_type p = parse_block(params);
    if (!s->pot) s->pot = std::make_shared<Potential>(Potential(s->sys, s->msg));
    default_nlist(s, p);
    std::string phase_in = p.count("phase_in") ? p["phase_in"] : std::string("constant");
    ValuePtr val = make_value(phase_in, s->msg, p);
    std::string n(name);
    PairPotentialPtr pp;
    if (n == "soft") pp = std::make_shared<PairSoftPotential>(s->sys, s->msg, s->nlist, val, p);
    else if (n == "lj") pp = std::make_shared<PairLJPotential>(s->sys, s->msg, s->nlist, val, p);
    else if (n == "morse") pp = std::make_shared<PairMorsePotential>(s->sys, s->msg, s->nlist, val, p);
    else if (n == "gaussian") pp = std::make_shared<PairGaussianPotential>(s->sys, s->msg, s->nlist, val, p);
    else throw std::runtime_error("unknown pair potential " + n);
    s->pot->add_pair_potential(n, pp);
  });
}

// pair_param <name> {type_1; type_2; ...}
int rs_pair_param(void* h, const char* name, const char* params) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    require(s->pot != nullptr, "No pair potential defined.");
    pairs_type p = parse_block(params);
    s->pot->add_pair_potential_parameters(std::string(name), p);
  });
}

// external <name> {...}
int rs_external(void* h, const char* name, const char* params) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    require(s->sys != nullptr, "System not defined.");
    pairs_type p = parse_block(params);
    if (!s->pot) s->pot = std::make_shared<Potential>(Potential(s->sys, s->msg));
    std::string n(name);
    require(n == "self_propulsion", "only the self_propulsion external potential is built here");
    s->pot->add_external_potential(n, std::make_shared<ExternalSelfPropulsion>(s->sys, s->msg, p));
  });
}

// external_param <name> {type; alpha}
int rs_external_param(void* h, const char* name, const char* params) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    require(s->pot != nullptr, "No external potential defined.");
    pairs_type p = parse_block(params);
    s->pot->add_external_potential_parameters(std::string(name), p);
  });
}

// pair_align <name> {...}
int rs_pair_align(void* h, const char* name, const char* params) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    require(s->sys != nullptr, "System not defined.");
    pairs_type p = parse_block(params);
    if (!s->aligner) s->aligner = std::make_shared<Aligner>(Aligner(s->sys, s->msg));
    default_nlist(s, p);
    std::string n(name);
    PairAlignPtr a;
    if (n == "polar") a = std::make_shared<PairPolarAlign>(s->sys, s->msg, s->nlist, p);
    else if (n == "nematic") a = std::make_shared<PairNematicAlign>(s->sys, s->msg, s->nlist, p);
    else if (n == "vicsek") a = std::make_shared<PairVicsekAlign>(s->sys, s->msg, s->nlist, p);
    else throw std::runtime_error("unknown pair aligner " + n);
    s->aligner->add_pair_align(n, a);
  });
}

// align_param <name> {...}
int rs_align_param(void* h, const char* name, const char* params) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    require(s->aligner != nullptr, "No aligner defined.");
    pairs_type p = parse_block(params);
    s->aligner->add_pair_align_parameters(std::string(name), p);
  });
}

// timestep <dt>
int rs_timestep(void* h, double dt) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    require(s->sys != nullptr, "System not defined.");
    s->sys->set_integrator_step(dt);
  });
}

// integrator <name> {...}
int rs_integrator(void* h, const char* name, const char* params) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    require(s->sys != nullptr, "System not defined.");
    require(s->constraint != nullptr, "Constraint not defined.");
    pairs_type p = parse_block(params);
    std::string group = p.count("group") ? p["group"] : std::string("all");
    std::string n(name);
    std::string key = n + "_" + group;
    require(s->integrator.find(key) == s->integrator.end(), "Integrator already exists.");
    std::string tc = p.count("temperature_control") ? p["temperature_control"] : std::string("constant");
    ValuePtr temp = make_value(tc, s->msg, p);
    IntegratorPtr it;
    if (n == "brownian")
      it = std::make_shared<IntegratorBrownian>(s->sys, s->msg, s->pot, s->aligner, s->nlist, s->constraint, temp, p);
    else if (n == "brownian_pos")
      it = std::make_shared<IntegratorBrownianPos>(s->sys, s->msg, s->pot, s->aligner, s->nlist, s->constraint, temp, p);
    else if (n == "brownian_align")
      it = std::make_shared<IntegratorBrownianAlign>(s->sys, s->msg, s->pot, s->aligner, s->nlist, s->constraint, temp, p);
    else if (n == "langevin")
      it = std::make_shared<IntegratorLangevin>(s->sys, s->msg, s->pot, s->aligner, s->nlist, s->constraint, temp, p);
    else if (n == "fire")
      it = std::make_shared<IntegratorFIRE>(s->sys, s->msg, s->pot, s->aligner, s->nlist, s->constraint, temp, p);
    else if (n == "nve")
      it = std::make_shared<IntegratorNVE>(s->sys, s->msg, s->pot, s->aligner, s->nlist, s->constraint, temp, p);
    else if (n == "vicsek")
      it = std::make_shared<IntegratorVicsek>(s->sys, s->msg, s->pot, s->aligner, s->nlist, s->constraint, temp, p);
    else
      throw std::runtime_error("unknown integrator " + n);
    s->integrator[key] = it;
  });
}

// disable {name; group}
int rs_disable(void* h, const char* name, const char* group) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    std::string key = std::string(name) + "_" + std::string(group && *group ? group : "all");
    require(s->integrator.erase(key) == 1, "No such integrator.");
  });
}

// One force and torque evaluation as at the top of a step (reset, then
// potentials, then aligners): samos.cpp:889-894.
int rs_compute(void* h) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    s->sys->reset_forces();
    s->sys->reset_torques();
    if (s->pot) s->pot->compute(s->sys->get_integrator_step());
    if (s->aligner) s->aligner->compute();
  });
}

// run <steps>: steps+1 integration steps (samos.cpp:864-972)
int rs_run(void* h, int steps) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    require(s->sys != nullptr, "System not defined.");
    require(s->constraint != nullptr, "Constraint not defined.");
    require(!s->integrator.empty(), "Integrator not defined.");
    SystemPtr sys = s->sys;
    if (s->pot) s->pot->compute(sys->get_integrator_step());
    if (s->aligner) s->aligner->compute();
    for (int t = 0; t <= steps; t++) {
      sys->set_step(s->time_step);
      sys->set_run_step(t);
      if (s->constraint->rescale()) {
        s->nlist->build();
        s->nlist_builds++;
      }
      for (int i = 0; i < sys->size(); i++) s->constraint->enforce(sys->get_particle(i));
      sys->reset_forces();
      sys->reset_torques();
      if (s->pot) s->pot->compute(sys->get_integrator_step());
      if (s->aligner) s->aligner->compute();
      for (auto& kv : s->integrator) kv.second->integrate();
      if ((s->pot && s->pot->need_nlist()) || (s->aligner && s->aligner->need_nlist())) {
        bool rebuild = false;
        if (sys->get_force_nlist_rebuild()) {
          rebuild = true;
          sys->set_force_nlist_rebuild(false);
        } else {
          for (int i = 0; i < sys->size(); i++)
            if (s->nlist->need_update(sys->get_particle(i))) {
              rebuild = true;
              break;
            }
        }
        if (rebuild) {
          s->nlist->build();
          s->nlist_builds++;
        }
      }
      s->time_step++;
    }
  });
}

int rs_nlist_builds(void* h) { return static_cast<Session*>(h)->nlist_builds; }

int rs_build_nlist(void* h) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    require(s->nlist != nullptr, "No neighbour list.");
    s->nlist->build();
  });
}

// Per-particle field in particle index order.  Doubles: x y z vx vy vz fx fy
// fz tau_x tau_y tau_z nx ny nz Nx Ny Nz omega age radius mass; ints (as
// doubles): ix iy iz type.
int rs_get(void* h, const char* field, double* out) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    std::string f(field);
    int n = s->sys->size();
    std::function<double(Particle&)> get;
    if (f == "x") get = [](Particle& p) { return p.x; };
    else if (f == "y") get = [](Particle& p) { return p.y; };
    else if (f == "z") get = [](Particle& p) { return p.z; };
    else if (f == "vx") get = [](Particle& p) { return p.vx; };
    else if (f == "vy") get = [](Particle& p) { return p.vy; };
    else if (f == "vz") get = [](Particle& p) { return p.vz; };
    else if (f == "fx") get = [](Particle& p) { return p.fx; };
    else if (f == "fy") get = [](Particle& p) { return p.fy; };
    else if (f == "fz") get = [](Particle& p) { return p.fz; };
    else if (f == "tau_x") get = [](Particle& p) { return p.tau_x; };
    else if (f == "tau_y") get = [](Particle& p) { return p.tau_y; };
    else if (f == "tau_z") get = [](Particle& p) { return p.tau_z; };
    else if (f == "nx") get = [](Particle& p) { return p.nx; };
    else if (f == "ny") get = [](Particle& p) { return p.ny; };
    else if (f == "nz") get = [](Particle& p) { return p.nz; };
    else if (f == "Nx") get = [](Particle& p) { return p.Nx; };
    else if (f == "Ny") get = [](Particle& p) { return p.Ny; };
    else if (f == "Nz") get = [](Particle& p) { return p.Nz; };
    else if (f == "omega") get = [](Particle& p) { return p.omega; };
    else if (f == "age") get = [](Particle& p) { return p.age; };
    else if (f == "radius") get = [](Particle& p) { return p.get_radius(); };
    else if (f == "mass") get = [](Particle& p) { return p.mass; };
    else if (f == "ix") get = [](Particle& p) { return (double)p.ix; };
    else if (f == "iy") get = [](Particle& p) { return (double)p.iy; };
    else if (f == "iz") get = [](Particle& p) { return (double)p.iz; };
    else if (f == "type") get = [](Particle& p) { return (double)p.get_type(); };
    else throw std::runtime_error("unknown field " + f);
    for (int i = 0; i < n; i++) out[i] = get(s->sys->get_particle(i));
  });
}

// The half neighbour list in its storage order: for each particle i, the
// entries of get_neighbours(i) in order.  Returns the pair count, or
// -count when cap is too small.
int rs_pairs(void* h, int* out_i, int* out_j, int cap) {
  Session* s = static_cast<Session*>(h);
  int count = 0;
  int n = s->sys->size();
  for (int i = 0; i < n; i++) count += (int)s->nlist->get_neighbours(i).size();
  if (count > cap || !out_i) return -count;
  int k = 0;
  for (int i = 0; i < n; i++)
    for (int j : s->nlist->get_neighbours(i)) {
      out_i[k] = i;
      out_j[k] = j;
      k++;
    }
  return count;
}

// Energies of the last evaluation: the named pair potential (cls 0) or pair
// aligner (cls 1).
int rs_energy(void* h, int cls, const char* name, double* out) {
  Session* s = static_cast<Session*>(h);
  return guarded(s, [&] {
    if (cls == 0) *out = s->pot->compute_pair_potential_energy_of_type(std::string(name));
    else *out = s->aligner->compute_pair_alignment_energy_of_type(std::string(name));
  });
}

}  // extern "C"
