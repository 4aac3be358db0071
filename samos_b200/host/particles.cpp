// particles.cpp -- particle input files, as System::System reads them
// (src/system/system.cpp:76-450): lines are trimmed and lower-cased, split
// on whitespace or commas; a `keys:` line (or the deprecated `# id type ...`
// line) names the columns, otherwise the positional format
// id type radius x y z vx vy vz nx ny nz [omega [length]] is read, with at
// least NUM_PART_ATTRIB = 10 columns (particle.hpp:49).
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <fstream>
#include <set>
#include <sstream>

#include "samos_host.hpp"

namespace samos_host {

namespace {

// split_line (system.cpp:40-45): separators are a run of whitespace or a
// single comma, as regex "\\s+|,|\\t" splits; the line is already trimmed.
std::vector<std::string> split_fields(const std::string& line) {
  std::vector<std::string> out;
  std::string cur;
  size_t i = 0;
  while (i < line.size()) {
    const char c = line[i];
    if (c == ',') {
      out.push_back(cur); cur.clear(); i++;
    } else if (std::isspace((unsigned char)c)) {
      out.push_back(cur); cur.clear();
      while (i < line.size() && std::isspace((unsigned char)line[i])) i++;
    } else {
      cur += c; i++;
    }
  }
  out.push_back(cur);
  return out;
}

double num(const std::string& s, const char* what) {
  char* end = nullptr;
  const double v = std::strtod(s.c_str(), &end);
  if (s.empty() || *end != '\0') throw HostError(std::string("Bad ") + what + " value \"" + s + "\" in input file.");
  return v;
}
int inum(const std::string& s, const char* what) {
  char* end = nullptr;
  const long v = std::strtol(s.c_str(), &end, 10);
  if (s.empty() || *end != '\0') throw HostError(std::string(what) + " has to be an integer (\"" + s + "\").");
  return (int)v;
}

const char* kOldKeys[] = {"id", "type", "radius", "x", "y", "z", "vx", "vy", "vz", "nx", "ny", "nz",
                          "omega", "length", "ix", "iy", "iz"};

}  // namespace

Particles read_particles(const std::string& path) {
  std::ifstream in(path);
  if (!in) throw HostError("Problem opening file " + path);
  Particles P;
  std::map<std::string, int> col;
  bool has_keys = false;
  int id = -1;
  std::set<int> types;
  std::string line;
  while (std::getline(in, line)) {
    line = trim(line);
    std::transform(line.begin(), line.end(), line.begin(), ::tolower);
    if (line.empty()) continue;
    const std::vector<std::string> f = split_fields(line);
    if (f.empty()) continue;
    if (f[0] == "#") {
      if (f.size() > 1 && std::find(std::begin(kOldKeys), std::end(kOldKeys), f[1]) != std::end(kOldKeys)) {
        has_keys = true;
        col.clear();
        for (size_t c = 1; c < f.size(); c++) col[f[c]] = (int)c - 1;
      }
      continue;
    }
    if (f[0][0] == '#') continue;
    if (f[0] == "keys:") {
      has_keys = true;
      col.clear();
      for (size_t c = 1; c < f.size(); c++) col[f[c]] = (int)c - 1;
      continue;
    }
    if (!has_keys && f.size() < 10)
      throw HostError("Insufficient number of parameters to define a particle. " + std::to_string(f.size()) +
                      " given, but 10 expected.");
    auto field = [&](const char* key, int pos, bool& found) -> const std::string* {
      if (has_keys) {
        auto it = col.find(key);
        found = it != col.end() && it->second < (int)f.size();
        return found ? &f[it->second] : nullptr;
      }
      found = pos >= 0 && pos < (int)f.size();
      return found ? &f[pos] : nullptr;
    };
    bool ok;
    const std::string* s;
    s = field("id", 0, ok);
    id = ok ? inum(*s, "Particle id") : id + 1;
    s = field("type", 1, ok);
    const int tp = ok ? inum(*s, "Particle type") : 1;
    if (tp < 1) throw HostError("Particle type has to be positive integer.");
    types.insert(tp);
    s = field("radius", 2, ok);
    const double r = ok ? num(*s, "radius") : 1.0;
    auto dbl = [&](const char* key, int pos, double def) {
      bool found;
      const std::string* v = field(key, pos, found);
      return found ? num(*v, key) : def;
    };
    P.id.push_back(id);
    P.type.push_back(tp);
    P.radius.push_back(r);
    P.x.push_back(dbl("x", 3, 0.0)); P.y.push_back(dbl("y", 4, 0.0)); P.z.push_back(dbl("z", 5, 0.0));
    P.vx.push_back(dbl("vx", 6, 0.0)); P.vy.push_back(dbl("vy", 7, 0.0)); P.vz.push_back(dbl("vz", 8, 0.0));
    P.nx.push_back(dbl("nx", 9, 1.0)); P.ny.push_back(dbl("ny", 10, 0.0)); P.nz.push_back(dbl("nz", 11, 0.0));
    P.omega.push_back(dbl("omega", 12, 0.0));
    P.mass.push_back(has_keys ? dbl("mass", -1, 1.0) : 1.0);
    P.ix.push_back(has_keys ? (int)dbl("ix", -1, 0.0) : 0);
    P.iy.push_back(has_keys ? (int)dbl("iy", -1, 0.0) : 0);
    P.iz.push_back(has_keys ? (int)dbl("iz", -1, 0.0) : 0);
    P.molecule.push_back(has_keys ? (int)dbl("molecule", -1, 0.0) : 0);
  }
  if (P.x.empty()) throw HostError("No particles read from " + path);
  P.ntypes = (int)types.size();
  // The engine addresses particles by their position in the file, which is
  // the reference's particle index; type tables need types 1..ntypes.
  if (*types.rbegin() != P.ntypes) throw HostError("Particle types must be 1..ntypes without gaps.");
  return P;
}


}  // namespace samos_host
