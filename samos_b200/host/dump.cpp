// Dumps of the conf-file host, following Dump (src/dump/dump.cpp): types
// input, full, xyz, velocity, director, xyzv, dcd and vtp with the
// reference's extensions, file naming, headers and number formats; vtp as a
// VTK XML PolyData file (ASCII) with the point arrays Dump::dump_vtp adds for
// particles without mesh or bonds (dump.cpp:1109-1230).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>

#include "samos_host.hpp"

namespace samos_host {

namespace {

const char* ext_of(const std::string& type) {  // m_type_ext, dump.cpp:65-79
  if (type == "velocity") return "vel";
  if (type == "xyz") return "xyz";
  if (type == "full") return "dat";
  if (type == "input") return "inp";
  if (type == "dcd") return "dcd";
  if (type == "director") return "dir";
  if (type == "xyzv") return "xyzv";
  if (type == "vtp") return "vtp";
  return nullptr;
}

void write_int(std::FILE* f, int32_t v) { std::fwrite(&v, 4, 1, f); }

// DCD header, dump.cpp:274-338 (frame count left 0, as there)
void dcd_header(std::FILE* f, const DumpSpec& d, int32_t n) {
  write_int(f, 84);
  std::fwrite("CORD", 1, 4, f);
  write_int(f, 0);
  write_int(f, (int32_t)d.start);
  write_int(f, (int32_t)d.freq);
  for (int i = 0; i < 6; i++) write_int(f, 0);
  write_int(f, 0);  // timestep (unused)
  write_int(f, 1);  // include unit cell
  for (int i = 0; i < 8; i++) write_int(f, 0);
  write_int(f, 24);  // CHARMM version 24
  write_int(f, 84);
  write_int(f, 164);
  write_int(f, 2);
  char title[80] = {0};
  std::strncpy(title, "Created by SAMoS", 79);
  std::fwrite(title, 1, 80, f);
  char when[80] = {0};
  std::time_t now = std::time(nullptr);
  std::strftime(when, sizeof when, "REMARKS Created  %d %B, %Y at %H:%M", std::localtime(&now));
  std::fwrite(when, 1, 80, f);
  write_int(f, 164);
  write_int(f, 4);
  write_int(f, n);
  write_int(f, 4);
}

std::string scale_text(double s) {  // operator<< of a double (6 significant digits)
  char b[64];
  std::snprintf(b, sizeof b, "%g", s);
  return b;
}

}  // namespace

DumpSpec make_dump(const std::string& name, const Params& p, int32_t n) {
  DumpSpec d;
  d.name = name;
  auto it = p.find("type");
  if (it == p.end()) throw HostError("No dump type specified.");
  d.type = it->second;
  const char* ext = ext_of(d.type);
  if (!ext) {
    static const char* others[] = {"xyzc", "mol2", "contact", "face", "mesh", "boundary", "ajm"};
    for (const char* o : others)
      if (d.type == o) throw HostError("Dump type " + d.type + " is not part of the GPU path.");
    throw HostError("Unsupported dump type " + d.type + ".");
  }
  d.ext = ext;
  d.p = p;
  d.dir = p.count("directory") ? p.at("directory") : ".";
  d.start = p.count("start") ? to_i64(p.at("start"), "dump") : 0;
  d.freq = p.count("freq") ? to_i64(p.at("freq"), "dump") : 100;
  if (d.freq <= 0) throw HostError("Dump frequency has to be positive.");
  d.offset = p.count("step_offset") ? to_i64(p.at("step_offset"), "dump") : 0;
  d.multi = p.count("multi") != 0;
  d.header = p.count("header") != 0;
  d.keys = p.count("keys") != 0;
  if (p.count("compress")) throw HostError("Compressed dumps are not part of the GPU path.");
  if (p.count("group") && p.at("group") != "all") throw HostError("Dump groups other than 'all' are not part of the GPU path.");
  if (d.type == "full")
    for (const char* q : {"area", "single_particle"})
      if (p.count(q)) throw HostError(std::string("Dump quantity ") + q + " is not part of the GPU path.");
  if (d.type == "dcd" && d.multi) throw HostError("DCD files cannot be split. mulifile flag is not permitted.");
  d.scale = p.count("scale") ? to_dbl(p.at("scale"), "dump") : 1.0;
  if (!d.multi) {  // one file for the whole run, opened now (dump.cpp:160-170; a vtp one stays empty)
    d.path = d.dir + "/" + d.name + "." + d.ext;
    std::FILE* f = std::fopen(d.path.c_str(), d.type == "dcd" ? "wb" : "w");
    if (!f) throw HostError("Cannot open dump file " + d.path);
    if (d.type == "dcd") dcd_header(f, d, n);
    std::fclose(f);
  }
  return d;
}

bool dump_due(const DumpSpec& d, int64_t step) { return step >= d.start && step % d.freq == 0; }

namespace {

// Dump::dump_vtp (dump.cpp:1109-1230): one file per dump, <name>_<step>.vtp;
// Pressure is the trace of the particle stress, which none of the GPU path's
// potentials sets (zero, as in the reference); NumNeigh is the coordination.
void write_vtp(const DumpSpec& d, int64_t step, const DumpState& s) {
  char num[32];
  std::snprintf(num, sizeof num, "%010lld", (long long)step);
  const std::string path = d.dir + "/" + d.name + "_" + num + "." + d.ext;
  std::FILE* f = std::fopen(path.c_str(), "w");
  if (!f) throw HostError("Cannot open dump file " + path);
  const Particles& P = *s.parts;
  const size_t N = P.size();
  std::fprintf(f, "<?xml version=\"1.0\"?>\n<VTKFile type=\"PolyData\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
                  "  <PolyData>\n    <Piece NumberOfPoints=\"%zu\" NumberOfVerts=\"0\" NumberOfLines=\"0\" "
                  "NumberOfStrips=\"0\" NumberOfPolys=\"0\">\n      <PointData>\n", N);
  auto ints = [&](const char* name, auto get) {
    std::fprintf(f, "        <DataArray type=\"Int32\" Name=\"%s\" format=\"ascii\">\n", name);
    for (size_t i = 0; i < N; i++) std::fprintf(f, "%d\n", (int)get(i));
    std::fprintf(f, "        </DataArray>\n");
  };
  auto reals = [&](const char* name, int comps, auto get) {
    std::fprintf(f, "        <DataArray type=\"Float64\" Name=\"%s\" NumberOfComponents=\"%d\" format=\"ascii\">\n",
                 name, comps);
    for (size_t i = 0; i < N; i++) {
      for (int c = 0; c < comps; c++) std::fprintf(f, c ? " %.17g" : "%.17g", get(i, c));
      std::fputs("\n", f);
    }
    std::fprintf(f, "        </DataArray>\n");
  };
  ints("Id", [&](size_t i) { return P.id[i]; });
  ints("Type", [&](size_t i) { return P.type[i]; });
  reals("Radius", 1, [&](size_t i, int) { return P.radius[i]; });
  reals("NativeArea", 1, [&](size_t i, int) { return 3.14159265359 * P.radius[i] * P.radius[i]; });  // particle.hpp:81
  reals("Pressure", 1, [&](size_t, int) { return 0.0; });
  reals("Velocity", 3, [&](size_t i, int c) { return c == 0 ? P.vx[i] : c == 1 ? P.vy[i] : P.vz[i]; });
  reals("Force", 3, [&](size_t i, int c) { return c == 0 ? (*s.fx)[i] : c == 1 ? (*s.fy)[i] : (*s.fz)[i]; });
  reals("Director", 3, [&](size_t i, int c) { return c == 0 ? P.nx[i] : c == 1 ? P.ny[i] : P.nz[i]; });
  reals("NDirector", 3, [&](size_t i, int c) { return c == 0 ? -P.nx[i] : c == 1 ? -P.ny[i] : -P.nz[i]; });
  reals("NumNeigh", 1, [&](size_t i, int) { return (double)(*s.coordination)[i]; });
  std::fprintf(f, "      </PointData>\n      <Points>\n"
                  "        <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n");
  for (size_t i = 0; i < N; i++) std::fprintf(f, "%.17g %.17g %.17g\n", P.x[i], P.y[i], P.z[i]);
  std::fprintf(f, "        </DataArray>\n      </Points>\n    </Piece>\n  </PolyData>\n</VTKFile>\n");
  std::fclose(f);
}

}  // namespace

void write_dump(const DumpSpec& d, int64_t step, const DumpState& s) {
  if (d.type == "vtp") { write_vtp(d, step, s); return; }
  std::string path = d.path;
  const char* mode = d.type == "dcd" ? "ab" : "a";
  if (d.multi) {
    char num[32];
    std::snprintf(num, sizeof num, "%010lld", (long long)(step + d.offset));
    path = d.dir + "/" + d.name + "_" + num + "." + d.ext;
    mode = "w";
  }
  std::FILE* f = std::fopen(path.c_str(), mode);
  if (!f) throw HostError("Cannot open dump file " + path);
  const Particles& P = *s.parts;
  const size_t N = P.size();
  const double a = d.scale;
  auto has = [&](const char* k) { return d.p.count(k) != 0; };
  if (d.type == "xyz") {  // dump.cpp:490-502
    std::fprintf(f, "%zu\nGenerated by SAMoS code.\n", N);
    for (size_t i = 0; i < N; i++) std::fprintf(f, "%3d\t%10.6f\t%10.6f\t%10.6f\n", P.type[i], P.x[i], P.y[i], P.z[i]);
  } else if (d.type == "velocity" || d.type == "director") {  // dump.cpp:710-756
    const bool vel = d.type == "velocity";
    const char* c = vel ? "v" : "n";
    if (d.header)
      std::fprintf(f, "# scale a = %s\n# x-0.5*a*%sx  y-0.5*a*%sy z-0.5*a*%sz  a*%sx  a*%sy  a*%sz\n",
                   scale_text(a).c_str(), c, c, c, c, c, c);
    for (size_t i = 0; i < N; i++) {
      const double ux = vel ? P.vx[i] : P.nx[i], uy = vel ? P.vy[i] : P.ny[i], uz = vel ? P.vz[i] : P.nz[i];
      std::fprintf(f, "%12.7e\t%12.7e\t%12.7e\t%12.7e\t%12.7e\t%12.7e\n", P.x[i] - 0.5 * a * ux, P.y[i] - 0.5 * a * uy,
                   P.z[i] - 0.5 * a * uz, a * ux, a * uy, a * uz);
    }
  } else if (d.type == "xyzv") {  // dump.cpp:758-785
    const bool vel = has("velocity");
    std::fprintf(f, "%zu\nGenerated by SAMoS code. Vectors are %s scaled by %s\n", N, vel ? "velocities" : "directors",
                 scale_text(a).c_str());
    for (size_t i = 0; i < N; i++) {
      const double ux = vel ? P.vx[i] : P.nx[i], uy = vel ? P.vy[i] : P.ny[i], uz = vel ? P.vz[i] : P.nz[i];
      std::fprintf(f, "%c\t%12.7e\t%12.7e\t%12.7e\t%12.7e\t%12.7e\t%12.7e\n", (char)(64 + P.type[i]), P.x[i], P.y[i],
                   P.z[i], a * ux, a * uy, a * uz);
    }
  } else if (d.type == "input") {  // dump.cpp:690-708 (the `length` column carries omega, as there)
    if (d.header) {
      std::fprintf(f, "#  Lx = %10.6f, Ly = %10.6f, Lz = %10.6f\n", s.lx, s.ly, s.lz);
      std::fprintf(f, "# id type  radius x y z vx vy vz nx ny nz  omega length ix iy iz\n");
    }
    std::fprintf(f, "keys: id molecule type radius  x   y   z   vx   vy   vz   nx   ny   nz  length ix iy iz\n");
    for (size_t i = 0; i < N; i++)
      std::fprintf(f,
                   "%5d  %3d  %2d  %8.4f  %10.6f  %10.6f  %10.6f  %10.6f  %10.6f  %10.6f  %10.6f  %10.6f  %10.6f  "
                   "%10.6f  %3d  %3d  %3d\n",
                   P.id[i], P.molecule[i], P.type[i], P.radius[i], P.x[i], P.y[i], P.z[i], P.vx[i], P.vy[i], P.vz[i],
                   P.nx[i], P.ny[i], P.nz[i], P.omega[i], P.ix[i], P.iy[i], P.iz[i]);
  } else if (d.type == "full") {  // dump.cpp:504-688 (no mesh, no contacts on this path)
    static const char* const cols[][2] = {
        {"id", " id "}, {"tp", " type "}, {"flag", " flag "}, {"radius", " radius "}, {"coordinate", " x  y  z "},
        {"velocity", " vx  vy  vz "}, {"force", " fx  fy  fz "}, {"director", " nx  ny  nz "}, {"omega", " omega "},
        {"image_flags", " ix  iy  iz "}, {"normal", " nvx  nvy  nvz "}, {"parent", " parent "},
        {"cell_area", " cell_area "}, {"cell_perim", " cell_perim "}, {"cont_num", " cont_num "},
        {"boundary", " boundary "}, {"in_tissue", " in_tissue "}, {"molecule", " molecule "}};
    if (d.header) {
      std::fprintf(f, "# ");
      for (const auto& c : cols)
        if (has(c[0])) std::fputs(c[1], f);
      if (has("shape_param")) std::fputs(" shape_param", f);
      std::fputs("\n", f);
    }
    if (d.keys) {
      std::fprintf(f, "keys: ");
      for (const auto& c : cols)
        if (has(c[0])) std::fputs(c[1], f);
      std::fputs("\n", f);
    }
    const bool unwrap = has("unwrap");
    for (size_t i = 0; i < N; i++) {
      if (has("id")) std::fprintf(f, "%5d ", P.id[i]);
      if (has("tp")) std::fprintf(f, "%2d ", P.type[i]);
      if (has("flag")) std::fprintf(f, "%5d ", (int)i);  // the position in the input file (system.cpp:392-393)
      if (has("radius")) std::fprintf(f, "%8.5f ", P.radius[i]);
      if (has("coordinate")) {
        if (unwrap)
          std::fprintf(f, " %16.10e  %16.10e  %16.10e", P.x[i] + P.ix[i] * s.lx, P.y[i] + P.iy[i] * s.ly,
                       P.z[i] + P.iz[i] * s.lz);
        else
          std::fprintf(f, " %16.10e  %16.10e  %16.10e", P.x[i], P.y[i], P.z[i]);
      }
      if (has("velocity")) std::fprintf(f, " %12.7e  %12.7e  %12.7e", P.vx[i], P.vy[i], P.vz[i]);
      if (has("force")) std::fprintf(f, " %12.7e  %12.7e  %12.7e", (*s.fx)[i], (*s.fy)[i], (*s.fz)[i]);
      if (has("director")) std::fprintf(f, " %10.6f  %10.6f  %10.6f", P.nx[i], P.ny[i], P.nz[i]);
      if (has("omega")) std::fprintf(f, "%8.5f ", P.omega[i]);
      if (has("image_flags")) std::fprintf(f, " %3d  %3d  %3d ", P.ix[i], P.iy[i], P.iz[i]);
      if (has("normal")) std::fprintf(f, " %10.6f  %10.6f  %10.6f", (*s.Nx)[i], (*s.Ny)[i], (*s.Nz)[i]);
      if (has("parent")) std::fprintf(f, " %3d ", 0);
      if (has("boundary")) std::fputs(" 0 ", f);
      if (has("in_tissue")) std::fputs(" 0 ", f);
      if (has("molecule")) std::fprintf(f, "%2d ", P.molecule[i]);
      std::fputs("\n", f);
    }
  } else if (d.type == "dcd") {  // dump.cpp:419-488: unit cell record, then x, y, z as floats
    double cell[6] = {100.0, 0.0, 100.0, 0.0, 0.0, 100.0};
    write_int(f, 48);
    std::fwrite(cell, 8, 6, f);
    write_int(f, 48);
    const bool unwrap = has("unwrap");
    std::vector<float> buf(N);
    const std::vector<double>* X[3] = {&P.x, &P.y, &P.z};
    const std::vector<int32_t>* I[3] = {&P.ix, &P.iy, &P.iz};
    const double L[3] = {s.lx, s.ly, s.lz};
    for (int c = 0; c < 3; c++) {
      for (size_t i = 0; i < N; i++)
        buf[i] = unwrap ? (float)((*X[c])[i] + (*I[c])[i] * L[c]) : (float)(*X[c])[i];
      write_int(f, (int32_t)(N * sizeof(float)));
      std::fwrite(buf.data(), sizeof(float), N, f);
      write_int(f, (int32_t)(N * sizeof(float)));
    }
  }
  std::fclose(f);
}

}  // namespace samos_host
